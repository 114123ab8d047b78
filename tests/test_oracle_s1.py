"""The S1 oracle (oracle/stitch_oracle.c) against the reference's own S1
acceptance test (tests/test_s1_cuda.cu:107-200, :226-270, :272-330): the same
synthetic RGB patterns, resolutions and scales, the test's CPU reference
(float64 box filter, lround), and its tolerances (exact, except +-1 at
S = 0.75 where the reference's float kernel and its float64 check differ);
and the test's gradient known answers."""
import math

import numpy as np
import pytest

from oracle import c_oracle


def gray15(rgb):
    r, g, b = (rgb[..., i].astype(np.int64) for i in range(3))
    return ((9798 * r + 19235 * g + 3735 * b + 16384) >> 15).astype(np.int64)


def test_reference_cpu_s1(rgb, w, h, ww, wh):
    """Restatement of cpu_reference_s1 in tests/test_s1_cuda.cu:107-200."""
    gray = gray15(rgb)
    if (w, h) == (ww, wh):
        return gray.astype(np.uint8)
    if (w, h) == (2 * ww, 2 * wh):
        s = gray[0::2, 0::2] + gray[0::2, 1::2] + gray[1::2, 0::2] + gray[1::2, 1::2]
        return ((s + 2) >> 2).astype(np.uint8)
    if (w, h) == (4 * ww, 4 * wh):
        s = sum(gray[dy::4, dx::4] for dy in range(4) for dx in range(4))
        return np.vectorize(lambda v: int(math.floor(v * 0.0625 + 0.5)))(s).astype(np.uint8)
    isx, isy = w / ww, h / wh
    area = 1.0 / (isx * isy)
    out = np.zeros((wh, ww), np.uint8)
    for yd in range(wh):
        fy1, fy2 = yd * isy, (yd + 1) * isy
        for xd in range(ww):
            fx1, fx2 = xd * isx, (xd + 1) * isx
            t = 0.0
            for ys in range(int(math.floor(fy1)), min(int(math.ceil(fy2)), h)):
                wy = max(0.0, min(ys + 1.0, fy2) - max(float(ys), fy1))
                if wy <= 0:
                    continue
                for xs in range(int(math.floor(fx1)), min(int(math.ceil(fx2)), w)):
                    wx = max(0.0, min(xs + 1.0, fx2) - max(float(xs), fx1))
                    if wx > 0:
                        t += gray[ys, xs] * (wx * wy)
            out[yd, xd] = int(math.floor(t * area + 0.5))
    return out


test_reference_cpu_s1.__test__ = False


def pattern(w, h, mul, add):
    i = np.arange(w * h * 3, dtype=np.int64)
    return ((i * mul + add) % 256).astype(np.uint8).reshape(h, w, 3)


def work_size(w, h, s):
    return max(1, int(math.floor(w * s + 0.5))), max(1, int(math.floor(h * s + 0.5)))


@pytest.mark.parametrize("scale", [1.0, 0.5, 0.25, 0.75])
@pytest.mark.parametrize("size", [(64, 64), (128, 96), (640, 480)])
def test_oracle_matches_reference_test(scale, size):
    w, h = size
    ww, wh = work_size(w, h, scale)
    tol = 1 if scale == 0.75 else 0
    for mul, add in ((17, 23), (31, 97)):
        rgb = pattern(w, h, mul, add)
        got = c_oracle.s1(rgb, ww, wh).astype(int)
        want = test_reference_cpu_s1(rgb, w, h, ww, wh).astype(int)
        assert np.abs(got - want).max() <= tol


def test_gradient_known_answers():
    w, h = 64, 48
    assert c_oracle.s1_gradient(np.full((h, w), 128, np.uint8)) == 0.0
    checker = (((np.arange(w)[None, :] + np.arange(h)[:, None]) % 2) * 255).astype(np.uint8)
    assert abs(c_oracle.s1_gradient(checker) - 1.0) < 1e-9
    tex = ((np.arange(w * h) * 37 + 11) % 256).astype(np.uint8).reshape(h, w).astype(np.int64)
    s = np.abs(np.diff(tex, axis=1)).sum() + np.abs(np.diff(tex, axis=0)).sum()
    want = s / (255.0 * (h * (w - 1) + w * (h - 1)))
    assert abs(c_oracle.s1_gradient(tex.astype(np.uint8)) - want) < 1e-12

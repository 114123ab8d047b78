"""The C S5 oracle: host-side known answers of the reference
(tests/test_s5_math.cpp:21-88, tests/test_s5_cuda.cu:99-116) and bit-for-bit
agreement with the reference's own src/s5/s5_math.hpp compiled from the
reference tree (oracle/_ref/libref_s5math.so, when present)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import c_oracle

REF_MATH = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libref_s5math.so"
TRUTH = np.array([1.02, 0.03, 11, -0.02, 0.98, 7, 0.0002, -0.0001, 1], np.float64)


def p(a):
    return C.c_void_p(a.ctypes.data)


def project(h, bx, by):
    z = h[6] * bx + h[7] * by + h[8]
    return (h[0] * bx + h[1] * by + h[2]) / z, (h[3] * bx + h[4] * by + h[5]) / z


def hdiff(a, b):
    a = np.asarray(a).reshape(9)
    b = np.asarray(b).reshape(9)
    return np.max(np.abs(a / a[8] - b / b[8]))


def test_fit_recovers_projective_truth():
    pts = []
    for y in range(6):
        for x in range(8):
            bx, by = 11 + x * 80, 13 + y * 70
            ax, ay = project(TRUTH, bx, by)
            pts.append((ax, ay, bx, by))
    pts = np.array(pts, np.float64)
    out = np.zeros(9)
    assert c_oracle.lib().oracle_fit(len(pts), p(pts), None, p(out))
    assert hdiff(out, TRUTH) < 1e-8
    for q in pts:
        assert c_oracle.lib().oracle_residual2(p(out), *q) < 1e-16
    assert c_oracle.lib().oracle_valid_domain(p(out), 640, 480)


def test_degenerate_samples():
    rect = np.array([[3, 7, 0, 0], [103, 7, 100, 0], [103, 107, 100, 100], [3, 107, 0, 100]], np.float64)
    line = np.array([[1, 1, 1, 1], [2, 2, 2, 2], [3, 3, 3, 3], [4, 4, 4, 4]], np.float64)
    L = c_oracle.lib()
    out = np.zeros(9)
    assert L.oracle_nondegenerate(p(rect)) and L.oracle_fit(4, p(rect), None, p(out))
    assert not L.oracle_nondegenerate(p(line)) and not L.oracle_fit(4, p(line), None, p(out))
    dup = np.ascontiguousarray(rect[[0, 1, 2, 0]])
    assert not L.oracle_nondegenerate(p(dup))
    assert not L.oracle_fit(3, p(rect), None, p(out))


@pytest.mark.parametrize("n", [4, 5, 17, 101])
def test_counter_samples_distinct(n):
    out = np.zeros(4, np.int32)
    for h in range(4096):
        c_oracle.lib().oracle_sample_four(n, 20261022, h, p(out))
        assert len(set(out.tolist())) == 4 and out.min() >= 0 and out.max() < n


def known_answer_points(outliers=True, line=False):
    pts = []
    for i in range(80):
        x = 20 + (i % 10) * 50
        y = 2 * x if line else 20 + (i // 10) * 45
        x, y = float(np.float32(x)), float(np.float32(y))
        z = 0.0002 * x - 0.0001 * y + 1
        u = float(np.float32((1.02 * x + 0.03 * y + 11) / z))
        v = float(np.float32((-0.02 * x + 0.98 * y + 7) / z))
        if outliers and i % 4 == 0:
            u, v = float(600 - i), float(400 - i * 2)
        pts.append((u, v, x, y))
    return np.array(pts, np.float64)


def test_known_h_and_outliers():
    pts = known_answer_points()
    sa = c_oracle.make_scale_info(640, 480)
    res, mask, _ = c_oracle.s5(pts, 80, 257, 0.5, 20261022, 2, sa, sa)
    assert res["status"] == 0 and res["num_matches"] == 80 and res["num_inliers"] == 60
    assert abs(res["inlier_ratio"] - 0.75) < 1e-12
    assert 0 < res["inlier_coverage"] <= 1 and res["reproj_residual"] < 1e-3
    assert hdiff(res["H_s"], TRUTH) < 1e-3 and hdiff(res["H"], TRUTH) < 1e-3
    assert np.array_equal(mask, np.array([i % 4 != 0 for i in range(80)], np.uint8))


def test_incremental_equals_full():
    pts = known_answer_points()
    sa = c_oracle.make_scale_info(640, 480)
    full, fmask, _ = c_oracle.s5(pts, 80, 257, 0.5, 20261022, 2, sa, sa)
    _, _, best = c_oracle.s5(pts, 80, 17, 0.5, 20261022, 2, sa, sa)
    split, smask, _ = c_oracle.s5(pts, 80, 257, 0.5, 20261022, 2, sa, sa, previous=best, first=17)
    assert np.array_equal(full["H"], split["H"]) and np.array_equal(fmask, smask)


def test_collinear_is_degenerate():
    sa = c_oracle.make_scale_info(640, 480)
    res, mask, _ = c_oracle.s5(known_answer_points(False, True), 80, 257, 0.5, 20261022, 2, sa, sa)
    assert res["status"] == 5 and not mask.any()


@pytest.fixture(scope="module")
def refmath():
    if not REF_MATH.exists():
        pytest.skip("reference s5_math checker not built (oracle/_ref)")
    L = C.CDLL(str(REF_MATH))
    L.ref_fit.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ref_sample_four.argtypes = [C.c_int, C.c_uint64, C.c_int, C.c_void_p]
    L.ref_residual2.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double]
    L.ref_residual2.restype = C.c_double
    L.ref_nondegenerate.argtypes = [C.c_void_p]
    L.ref_valid_domain.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.ref_mat3_inverse.argtypes = [C.c_void_p, C.c_void_p]
    return L


def test_math_bitwise_vs_reference(refmath):
    rng = np.random.default_rng(5)
    L = c_oracle.lib()
    for trial in range(3000):
        n = 4 if trial % 3 else int(rng.integers(4, 60))
        b = rng.uniform(0, 640, (n, 2))
        h = TRUTH + rng.normal(0, [0.02, 0.02, 5, 0.02, 0.02, 5, 1e-4, 1e-4, 0])
        a = np.array([project(h, *q) for q in b]) + rng.normal(0, 0.5, (n, 2)) * (trial % 2)
        pts = np.ascontiguousarray(np.hstack([a, b]).astype(np.float32).astype(np.float64))
        keep = (rng.random(n) > 0.2).astype(np.uint8) if n > 4 else None
        o1, o2 = np.zeros(9), np.zeros(9)
        r1 = L.oracle_fit(n, p(pts), None if keep is None else p(keep), p(o1))
        r2 = refmath.ref_fit(n, p(pts), None if keep is None else p(keep), p(o2))
        assert r1 == r2
        if r1:
            assert np.array_equal(o1.view(np.uint64), o2.view(np.uint64))
            for q in pts[:5]:
                e1 = L.oracle_residual2(p(o1), *q)
                e2 = refmath.ref_residual2(p(o2), *q)
                assert e1 == e2
            assert L.oracle_valid_domain(p(o1), 640, 480) == refmath.ref_valid_domain(p(o2), 640, 480)
        if n == 4:
            assert L.oracle_nondegenerate(p(pts)) == refmath.ref_nondegenerate(p(pts))


def test_samples_vs_reference(refmath):
    a, b = np.zeros(4, np.int32), np.zeros(4, np.int32)
    for n in (4, 5, 17, 101, 1000, 65536):
        for h in range(0, 20000, 7):
            c_oracle.lib().oracle_sample_four(n, 0x1234567890abcdef, h, p(a))
            refmath.ref_sample_four(n, 0x1234567890abcdef, h, p(b))
            assert np.array_equal(a, b)


def test_inverse_vs_reference(refmath):
    rng = np.random.default_rng(2)
    for _ in range(200):
        m = rng.normal(size=9)
        o1, o2 = np.zeros(9), np.zeros(9)
        assert c_oracle.lib().oracle_mat3_inverse(p(m), p(o1)) == refmath.ref_mat3_inverse(p(m), p(o2))
        assert np.array_equal(o1, o2)

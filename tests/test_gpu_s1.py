"""S1 on the GPU: RGB8 -> GRAY8 with area resizing, bit for bit against the
oracle and against the reference's own S1 kernel built for sm_100a, at the
reference test's scales plus others; single-image and pair calls agree; the
gradient probe equals the oracle."""
import ctypes as C
import math

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi
from crossstage_stitch_b200._abi import ImageView, ScaleInfo
from oracle import c_oracle

from .gpu_util import REF_STAGES, stream

pytestmark = pytest.mark.gpu
ref = C.byref
PAD = 19


def rgb_view(rgb):
    h, w, _ = rgb.shape
    t = torch.full((h, 3 * w + PAD), 0xee, dtype=torch.uint8, device="cuda")
    t[:, :3 * w] = torch.from_numpy(rgb.reshape(h, 3 * w)).cuda()
    return t, ImageView(t.data_ptr(), w, h, t.stride(0), 0)


def gray_view(w, h):
    t = torch.full((h, w + PAD), 0x55, dtype=torch.uint8, device="cuda")
    return t, ImageView(t.data_ptr(), w, h, t.stride(0), 1)


def work(w, h, s):
    return max(1, int(math.floor(w * s + 0.5))), max(1, int(math.floor(h * s + 0.5)))


def ref_lib():
    if not REF_STAGES.exists():
        pytest.skip("reference stage build not present (oracle/_ref)")
    L = C.CDLL(str(REF_STAGES))
    L.ref_s1_preprocess.argtypes = _abi.PROTOTYPES["stitch_s1_preprocess"][1]
    L.ref_s1_compute_gradient.argtypes = _abi.PROTOTYPES["stitch_s1_compute_gradient"][1]
    return L


def run_pair(fn, rgb_a, rgb_b, scale):
    ta, va = rgb_view(rgb_a)
    tb, vb = rgb_view(rgb_b)
    wa, ha = work(rgb_a.shape[1], rgb_a.shape[0], scale)
    wb, hb = work(rgb_b.shape[1], rgb_b.shape[0], scale)
    ga, oa = gray_view(wa, ha)
    gb, ob = gray_view(wb, hb)
    sa, sb = ScaleInfo(), ScaleInfo()
    st = fn(ref(va), ref(vb), scale, ref(oa), ref(ob), ref(sa), ref(sb), stream())
    torch.cuda.synchronize()
    assert st == 0
    assert (sa.work_w, sa.work_h, sb.work_w, sb.work_h) == (wa, ha, wb, hb)
    pad_ok = bool((ga[:, wa:] == 0x55).all() and (gb[:, wb:] == 0x55).all())
    return ga[:, :wa].cpu().numpy(), gb[:, :wb].cpu().numpy(), pad_ok


SIZES = [(64, 64), (128, 96), (640, 480), (333, 257), (1920, 1080)]


@pytest.mark.parametrize("scale", [1.0, 0.5, 0.25, 0.75, 0.6, 0.3])
def test_s1_vs_oracle_and_reference(cuda, scale):
    L = _abi.load()
    R = ref_lib()
    rng = np.random.default_rng(int(scale * 1000))
    for (w, h) in SIZES:
        a = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        b = rng.integers(0, 256, (h + 2, w - 1, 3), dtype=np.uint8)
        ga, gb, pad_ok = run_pair(L.stitch_s1_preprocess, a, b, scale)
        assert pad_ok  # nothing written past the working width
        assert np.array_equal(ga, c_oracle.s1(a, *work(w, h, scale)))
        assert np.array_equal(gb, c_oracle.s1(b, *work(w - 1, h + 2, scale)))
        ra, rb, _ = run_pair(R.ref_s1_preprocess, a, b, scale)
        assert np.array_equal(ga, ra) and np.array_equal(gb, rb)
        # single-image call equals the pair call
        ta, va = rgb_view(a)
        g1, o1 = gray_view(*work(w, h, scale))
        si = ScaleInfo()
        assert L.stitch_s1_preprocess_single(ref(va), scale, ref(o1), ref(si), stream()) == 0
        torch.cuda.synchronize()
        assert np.array_equal(g1[:, :o1.width].cpu().numpy(), ga)


def test_s1_argument_checks(cuda):
    L = _abi.load()
    rgb = np.zeros((8, 8, 3), np.uint8)
    t, v = rgb_view(rgb)
    g, o = gray_view(4, 4)
    si = ScaleInfo()
    assert L.stitch_s1_preprocess_single(ref(v), 0.0, ref(o), ref(si), stream()) == 1
    assert L.stitch_s1_preprocess_single(ref(v), 1.5, ref(o), ref(si), stream()) == 1
    assert L.stitch_s1_preprocess_single(ref(v), 1.0, ref(o), ref(si), stream()) == 1  # out is 4x4, needs 8x8
    bad = ImageView(v.data, 8, 8, 8, 0)  # pitch below 3 * width
    assert L.stitch_s1_preprocess_single(ref(bad), 0.5, ref(o), ref(si), stream()) == 1


def test_gradient(cuda):
    L = _abi.load()
    R = ref_lib()
    ws = torch.zeros(64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, pin_memory=True)
    pa = C.cast(out.data_ptr(), C.POINTER(C.c_double))
    pb = C.cast(out.data_ptr() + 8, C.POINTER(C.c_double))
    rng = np.random.default_rng(3)
    w, h = 64, 48
    checker = (((np.arange(w)[None, :] + np.arange(h)[:, None]) % 2) * 255).astype(np.uint8)
    cases = [np.full((h, w), 128, np.uint8), checker, rng.integers(0, 256, (h, w), dtype=np.uint8),
             rng.integers(0, 256, (1080, 1920), dtype=np.uint8)]
    for a in cases:
        b = np.ascontiguousarray(a[::-1, :])
        ga, va = gray_view(a.shape[1], a.shape[0])
        gb, vb = gray_view(b.shape[1], b.shape[0])
        ga[:, :a.shape[1]] = torch.from_numpy(a).cuda()
        gb[:, :b.shape[1]] = torch.from_numpy(b).cuda()
        assert L.stitch_s1_compute_gradient(ref(va), ref(vb), C.c_void_p(ws.data_ptr()), pa, pb, stream()) == 0
        torch.cuda.synchronize()
        mine = out.clone()
        assert mine[0].item() == c_oracle.s1_gradient(a) and mine[1].item() == c_oracle.s1_gradient(b)
        assert R.ref_s1_compute_gradient(ref(va), ref(vb), C.c_void_p(ws.data_ptr()), pa, pb, stream()) == 0
        torch.cuda.synchronize()
        assert out[0].item() == mine[0].item() and out[1].item() == mine[1].item()
    assert c_oracle.s1_gradient(checker) == pytest.approx(1.0, abs=1e-9)

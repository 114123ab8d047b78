"""S6 feather render on the GPU through the C ABI: bit for bit against the
oracle (panorama, mask, union/overlap counters) on the golden cases and on
seeded random pairs up to 1920x1080; canvas and mask exact and RGB within 2
of the reference's FP64 NumPy render (the reference's own bar,
tests/test_s6_cuda.cu:443-448); mask and counters exact and RGB within 1 of
the reference's own kernel built for sm_100a (its nvcc build contracts
products into FMAs, this one rounds each operation); nothing written past
the row width; the argument checks of tests/test_s6_cuda.cu:192-262."""
import ctypes as C
import math

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi, render
from crossstage_stitch_b200._abi import ImageView, S6Geometry
from oracle import c_oracle

from .gpu_util import REF_STAGES, stream
from .test_oracle_s6 import GOLDEN_CASES, IDENTITY

pytestmark = pytest.mark.gpu
ref = C.byref
PAD = 13
OK, INVALID = 0, 1


def rgb_dev(img):
    h, w, _ = img.shape
    t = torch.full((h, 3 * w + PAD), 0xa5, dtype=torch.uint8, device="cuda")
    t[:, :3 * w] = torch.from_numpy(np.ascontiguousarray(img).reshape(h, 3 * w)).cuda()
    return t, ImageView(t.data_ptr(), w, h, t.stride(0), 0)


def canvas(g):
    out = torch.full((g.height, 3 * g.width + PAD), 0xa5, dtype=torch.uint8, device="cuda")
    mask = torch.full((g.height, g.width + PAD), 0xa5, dtype=torch.uint8, device="cuda")
    return (out, ImageView(out.data_ptr(), g.width, g.height, out.stride(0), 0),
            mask, ImageView(mask.data_ptr(), g.width, g.height, mask.stride(0), 1))


class Renderer:
    def __init__(self, which):
        if which == "ours":
            self.L = _abi.load()
            self.render = self.L.stitch_s6_render
            self.prepare = self.L.stitch_s6_prepare_geometry
        else:
            if not REF_STAGES.exists():
                pytest.skip("reference stage build not present (oracle/_ref)")
            self.L = C.CDLL(str(REF_STAGES))
            self.render = self.L.ref_s6_render
            self.render.argtypes = _abi.PROTOTYPES["stitch_s6_render"][1]
            self.prepare = self.L.ref_s6_prepare_geometry
            self.prepare.argtypes = _abi.PROTOTYPES["stitch_s6_prepare_geometry"][1]
        self.render.restype = C.c_int
        self.prepare.restype = C.c_int

    def geometry(self, a, b, h):
        g = S6Geometry()
        p = render.default_policy()
        st = self.prepare(a.shape[1], a.shape[0], b.shape[1], b.shape[0],
                          (C.c_double * 9)(*np.asarray(h, np.float64).ravel()), ref(p), ref(g))
        return st, g

    def __call__(self, a, b, h):
        st, g = self.geometry(a, b, h)
        assert st == OK
        ta, va = rgb_dev(a)
        tb, vb = rgb_dev(b)
        out, vo, mask, vm = canvas(g)
        stats = torch.full((2,), -1, dtype=torch.int64, device="cuda")
        sp = C.cast(stats.data_ptr(), C.POINTER(C.c_uint64))
        assert self.render(ref(va), ref(vb), ref(g), 0, ref(vo), ref(vm), None, 0, stream(), sp) == OK
        torch.cuda.synchronize()
        assert (out[:, 3 * g.width:] == 0xa5).all().item() and (mask[:, g.width:] == 0xa5).all().item()
        pano = out[:, :3 * g.width].cpu().numpy().reshape(g.height, g.width, 3)
        return g, pano, mask[:, :g.width].cpu().numpy(), tuple(int(v) for v in stats.cpu())


def smooth(w, h, seed):
    yy, xx = np.indices((h, w), dtype=np.float64)
    rng = np.random.default_rng(seed)
    ch = []
    for _ in range(3):
        f = rng.uniform(0.01, 0.3, 4)
        v = np.sin(f[0] * xx + f[1] * yy + rng.uniform(0, 6)) + np.cos(f[2] * xx - f[3] * yy)
        ch.append(np.clip(np.round(127.5 + 63 * v + rng.normal(0, 8, v.shape)), 0, 255))
    return np.stack(ch, -1).astype(np.uint8)


def random_pairs():
    rng = np.random.default_rng(2024)
    sizes = [(1, 1), (2, 1), (1, 5), (7, 3), (64, 48), (333, 257), (640, 480)]
    for i, (w, h) in enumerate(sizes * 2):
        wb, hb = max(1, w + int(rng.integers(-3, 4))), max(1, h + int(rng.integers(-3, 4)))
        ang, s = rng.uniform(-0.3, 0.3), rng.uniform(0.7, 1.4)
        H = np.array([[s * math.cos(ang), -s * math.sin(ang), rng.uniform(-0.4, 0.4) * w],
                      [s * math.sin(ang), s * math.cos(ang), rng.uniform(-0.4, 0.4) * h],
                      [rng.normal(0, 3e-4), rng.normal(0, 3e-4), 1.0]])
        if i % 3 == 0:
            H = np.array([[1, 0, float(rng.integers(-w, w + 1))], [0, 1, float(rng.integers(-h, h + 1))], [0, 0, 1]])
        yield f"{w}x{h}_{i}", smooth(w, h, i), smooth(wb, hb, 100 + i), H
    yield "snap_near_integer", smooth(40, 30, 7), smooth(40, 30, 8), np.array(
        [[1, 0, -2 - 5e-11], [0, 1, 3 + 4e-11], [0, 0, 1.0]])
    yield "strong_perspective", smooth(200, 150, 9), smooth(200, 150, 10), np.array(
        [[1, 0.1, 5], [0.05, 1, -3], [2.5e-3, 1e-3, 1.0]])
    yield "noise_1080p", np.random.default_rng(5).integers(0, 256, (1080, 1920, 3), dtype=np.uint8), \
        np.random.default_rng(6).integers(0, 256, (1080, 1920, 3), dtype=np.uint8), np.array(
            [[0.98, 0.02, 310.5], [-0.015, 1.01, 22.25], [1e-5, -2e-5, 1.0]])


RANDOM = list(random_pairs())


@pytest.mark.parametrize("name,case", GOLDEN_CASES, ids=[n for n, _ in GOLDEN_CASES])
def test_golden_vs_oracle_and_reference_fp64(cuda, name, case):
    a, b, h = case["a"], case["b"], case["H"]
    g, pano, mask, stats = Renderer("ours")(a, b, h)
    assert [g.width, g.height, g.origin_x, g.origin_y] == case["canvas"].tolist()
    _, og = c_oracle.s6_geometry(a.shape[1], a.shape[0], b.shape[1], b.shape[0], h)
    opano, omask, ostats = c_oracle.s6_feather(a, b, og)
    assert np.array_equal(pano, opano) and np.array_equal(mask, omask) and stats == ostats
    np.testing.assert_array_equal(mask, case["mask"])
    assert np.abs(pano.astype(int) - case["panorama"].astype(int)).max() <= 2


@pytest.mark.parametrize("name,a,b,h", RANDOM, ids=[r[0] for r in RANDOM])
def test_random_vs_oracle_and_reference_kernel(cuda, name, a, b, h):
    g, pano, mask, stats = Renderer("ours")(a, b, h)
    st, og = c_oracle.s6_geometry(a.shape[1], a.shape[0], b.shape[1], b.shape[0], h)
    assert st == OK and [og.w, og.h, og.ox, og.oy] == [g.width, g.height, g.origin_x, g.origin_y]
    assert list(og.inv) == list(g.inverse)
    opano, omask, ostats = c_oracle.s6_feather(a, b, og)
    assert np.array_equal(mask, omask) and stats == ostats
    assert np.array_equal(pano, opano), int(np.abs(pano.astype(int) - opano.astype(int)).max())
    rg, rpano, rmask, rstats = Renderer("reference")(a, b, h)
    assert list(rg.inverse) == list(g.inverse)
    assert np.array_equal(mask, rmask) and stats == rstats
    assert np.abs(pano.astype(int) - rpano.astype(int)).max() <= 1


def test_repeat_resets_counters_and_python_wrapper(cuda):
    a = torch.zeros((3, 4, 3), dtype=torch.uint8, device="cuda")
    b = torch.full((3, 4, 3), 255, dtype=torch.uint8, device="cuda")
    g = render.prepare_geometry(4, 3, 4, 3, [1, 0, 7, 0, 1, 0, 0, 0, 1.0])
    assert (g.width, g.height) == (11, 3)
    stats = torch.full((2,), 123, dtype=torch.int64, device="cuda")
    first = None
    for _ in range(2):
        out, mask = render.render(a, b, g, statistics=stats)
        torch.cuda.synchronize()
        assert stats.tolist() == [24, 0]
        xs = torch.arange(11, device="cuda")
        assert torch.equal(mask, ((xs < 4) | (xs >= 7)).to(torch.uint8).expand(3, 11))
        assert torch.equal(out, torch.where(xs >= 7, 255, 0).to(torch.uint8)[None, :, None].expand(3, 11, 3))
        if first is not None:
            assert torch.equal(first, out)
        first = out.clone()
    # many blocks: each valid pixel counted once (tests/test_s6_cuda.cu:269-275)
    big = torch.zeros((3, 259, 3), dtype=torch.uint8, device="cuda")
    render.render(big, big, render.prepare_geometry(259, 3, 259, 3, IDENTITY), statistics=stats)
    torch.cuda.synchronize()
    assert stats.tolist() == [777, 777]


def test_argument_checks(cuda):
    L = _abi.load()
    a = np.zeros((3, 5, 3), np.uint8)
    _, g = Renderer("ours").geometry(a, a, [1, 0, -2, 0, 1, -1, 0, 0, 1.0])
    ta, va = rgb_dev(a)
    tb, vb = rgb_dev(a)
    out, vo, mask, vm = canvas(g)
    counters = torch.zeros(4, dtype=torch.int64, device="cuda")
    cp = C.cast(counters.data_ptr(), C.POINTER(C.c_uint64))
    s = stream()

    def call(va_=va, vb_=vb, g_=g, mode=0, vo_=vo, vm_=vm, ws=None, n=0, stats=None):
        return L.stitch_s6_render(ref(va_), ref(vb_), ref(g_), mode, ref(vo_), ref(vm_), ws, n, s, stats)

    assert call(stats=cp) == OK
    torch.cuda.synchronize()
    assert counters[:2].tolist() == [24, 6]
    b = C.c_size_t(123)
    assert L.stitch_s6_workspace_bytes(ref(g), 0, ref(b)) == OK and b.value == 0
    assert L.stitch_s6_workspace_bytes(ref(g), 17, ref(b)) == INVALID
    assert L.stitch_s6_workspace_bytes(ref(g), 0, None) == INVALID
    broken = S6Geometry.from_buffer_copy(g)
    broken.inverse[0] = float("nan")
    assert L.stitch_s6_workspace_bytes(ref(broken), 0, ref(b)) == INVALID
    assert call(g_=broken) == INVALID
    for mode in (1, 2):  # multiband is not built
        assert L.stitch_s6_workspace_bytes(ref(g), mode, ref(b)) == INVALID
        assert call(mode=mode) == INVALID
    assert call(vo_=va) == INVALID  # output aliases an input
    assert call(vo_=ImageView(vo.data, vo.width, vo.height, 3 * vo.width - 1, 0)) == INVALID  # pitch short
    assert call(vo_=ImageView(None, vo.width, vo.height, vo.pitch_bytes, 0)) == INVALID
    assert call(vm_=ImageView(vo.data, vm.width, vm.height, vm.pitch_bytes, 1)) == INVALID  # mask aliases output
    assert call(vm_=ImageView(vm.data, vm.width, vm.height, vm.pitch_bytes, 0)) == INVALID  # mask not GRAY8
    assert call(vo_=ImageView(vo.data, vo.width - 1, vo.height, vo.pitch_bytes, 0)) == INVALID  # wrong size
    assert call(va_=vb, vb_=vb, stats=cp) == OK  # inputs may alias each other
    for bad in (va.data, vo.data, vm.data):
        assert call(stats=C.cast(bad, C.POINTER(C.c_uint64))) == INVALID
    assert call(stats=C.cast(counters.data_ptr() + 1, C.POINTER(C.c_uint64))) == INVALID  # misaligned
    ws = C.c_void_p(counters.data_ptr())
    assert call(ws=ws, n=32, stats=cp) == INVALID  # counters inside a supplied workspace
    assert call(vo_=ImageView(None, vo.width, vo.height, vo.pitch_bytes, 0), stats=cp) == INVALID
    torch.cuda.synchronize()
    assert counters[:2].tolist() == [24, 6]  # failed calls wrote nothing

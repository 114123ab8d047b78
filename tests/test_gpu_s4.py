"""S4 on the GPU through the C ABI: the reference's own edge, tile and tie
cases (tests/test_s4_cuda.cu:185-315) against the CPU oracle, the popc path
against the oracle on random and planted-partner descriptors (the matching
microbenchmark's recipe), and agreement with the reference's kernels."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import c_oracle
from tests import gpu_util as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ours(cuda):
    """The __popc matcher (the tensor-core one has its own module)."""
    from crossstage_stitch_b200 import _abi
    L = _abi.load()
    before = L.stitch_s4_matcher()
    assert L.stitch_s4_set_matcher(0) == 0
    yield G.Lib("ours")
    L.stitch_s4_set_matcher(before)


def check(lib, a, b, ratio=0.8, cross=False, ca=None, cb=None, l2=False, pad_a=3, pad_b=7):
    dtype = G.FLOAT32 if l2 else G.BINARY_U8
    top, ia, ib, d, st = G.match(lib, a, b, ratio, cross, ca, cb, pad_a, pad_b, dtype)
    assert st == (0, 0)
    fwd = c_oracle.top2(a, b, ca, cb, l2)
    assert np.array_equal(top["first_index"], fwd["first_index"])
    assert np.array_equal(top["second_index"], fwd["second_index"])
    assert np.array_equal(top["first_distance"], fwd["first_distance"])
    assert np.array_equal(top["second_distance"], fwd["second_distance"])
    rev = c_oracle.top2(b, a, cb, ca, l2) if cross and b.shape[0] else None
    wa, wb, wd = c_oracle.accept(fwd, rev, ratio, l2)
    assert np.array_equal(ia, wa) and np.array_equal(ib, wb)
    assert np.array_equal(d, wd)
    return ia, ib, d


def u8(*v):
    return np.array(v, np.uint8).reshape(-1, 1)


def f32(*v):
    return np.array(v, np.float32).reshape(-1, 1)


@pytest.mark.parametrize("cross", [False, True])
def test_edges(ours, cross):
    assert check(ours, np.zeros((0, 1), np.uint8), u8(0, 255), cross=cross)[0].size == 0
    assert check(ours, u8(0, 1), np.zeros((0, 1), np.uint8), cross=cross)[0].size == 0
    assert check(ours, f32(0, 1), f32(0), cross=cross, l2=True)[0].size == 0
    assert check(ours, f32(0), f32(0, 0), cross=cross, l2=True)[0].size == 0
    assert check(ours, u8(0), u8(0, 0), cross=cross)[0].size == 0
    assert check(ours, u8(0), u8(0), cross=cross)[0].size == 0
    assert check(ours, u8(0), u8(1, 2), cross=cross)[0].size == 0
    assert check(ours, f32(0), f32(1, 2), 0.5, cross, l2=True)[0].size == 0
    assert check(ours, u8(0), u8(1, 3), 0.5, cross)[0].size == 0
    assert check(ours, f32(0), f32(0, 2), float(np.nextafter(0, 1)), cross, l2=True)[0].size == 1
    assert check(ours, f32(0, 99), f32(1, -1, 9), 0.9, cross, ca=1, l2=True)[0].size == 0
    assert check(ours, u8(0, 1), u8(0, 255), cross=cross, ca=0)[0].size == 0
    assert check(ours, u8(0, 1), u8(0, 255), cross=cross, cb=0)[0].size == 0
    assert check(ours, u8(0, 1), u8(0, 255), cross=cross, ca=3)[0].size == 0
    assert check(ours, u8(0, 1), u8(0, 255), cross=cross, cb=-1)[0].size == 0


def test_mutual_and_overflow(ours):
    assert check(ours, f32(0, 0), f32(0, 10), l2=True)[0].size == 2
    ia, _, _ = check(ours, f32(0, 0), f32(0, 10), cross=True, l2=True)
    assert list(ia) == [0]
    ia, _, _ = check(ours, u8(0, 0), u8(0, 255), cross=True)
    assert list(ia) == [0]
    ia, ib, d = check(ours, np.zeros((1, 2), np.float32), np.array([[3, 4], [30, 40]], np.float32), l2=True)
    assert d[0] == 5
    big = np.finfo(np.float32).max
    _, _, d = check(ours, f32(-big), f32(big / 2, big), 0.9, l2=True)
    assert np.isinf(d[0])


@pytest.mark.parametrize("dim", [1, 31, 32, 33, 65])
@pytest.mark.parametrize("cross", [False, True])
def test_tiles(ours, dim, cross):
    i = np.arange(263 * dim)
    a = ((i * 73 + i // dim * 19) % 256).astype(np.uint8).reshape(263, dim)
    j = np.arange(259 * dim)
    b = a.reshape(-1)[(j + 3 * dim) % a.size].reshape(259, dim)
    check(ours, a, b, cross=cross, ca=257, cb=253)
    fa = ((((i * 13 + i // dim * 11) % 101) - 50) / 8 + (i // dim) * 0.25).astype(np.float32).reshape(263, dim)
    fb = (fa.reshape(-1)[(j + 5 * dim) % fa.size] + 0.125).astype(np.float32).reshape(259, dim)
    check(ours, fa, fb, cross=cross, ca=257, cb=253, l2=True)


def test_ties_across_training_tiles(ours):
    train = np.full((260, 1), 20, np.float32)
    train[[3, 129, 258]] = 1
    check(ours, np.zeros((1, 1), np.float32), train, cross=True, l2=True)
    q = (np.arange(263) * 4.0).astype(np.float32).reshape(-1, 1)
    r = (np.arange(259) * 4.0 + 0.25).astype(np.float32).reshape(-1, 1)
    assert check(ours, q, r, cross=True, ca=257, cb=253, l2=True)[0].size == 253
    assert check(ours, q, r, cross=False, ca=257, cb=253, l2=True)[0].size == 257


def planted(nq, nt, seed=20261203):
    """Uniform 256-bit rows; 30 % of queries get a planted partner at
    Binomial(256, 0.05) distance and 5 % a second partner at the same
    distance (ties go to the lower train index)."""
    rng = np.random.default_rng(seed)
    q = rng.integers(0, 256, (nq, 32), dtype=np.uint8)
    t = rng.integers(0, 256, (nt, 32), dtype=np.uint8)
    partners = rng.choice(nq, size=int(0.3 * nq), replace=False)
    for qi in partners:
        d = rng.binomial(256, 0.05)
        for rep in range(2 if rng.random() < 0.05 / 0.3 else 1):
            row = np.unpackbits(q[qi]).copy()
            flip = rng.choice(256, size=d, replace=False)
            row[flip] ^= 1
            t[rng.integers(0, nt)] = np.packbits(row)
    return q, t


@pytest.mark.parametrize("shape", [(1000, 1000), (2000, 3000), (300, 20000), (4096, 64)])
@pytest.mark.parametrize("cross", [False, True])
def test_popc_planted_vs_oracle(ours, shape, cross):
    q, t = planted(*shape)
    check(ours, q, t, cross=cross, pad_a=0, pad_b=0)


def test_popc_active_counts_below_capacity(ours):
    q, t = planted(700, 900, seed=3)
    check(ours, q, t, cross=True, ca=650, cb=811, pad_a=16, pad_b=16)


def test_matching_microbenchmark_full_size(ours):
    """8192 x 8192 planted descriptors, the full microbenchmark size."""
    q, t = planted(8192, 8192)
    ia, ib, d = check(ours, q, t, pad_a=0, pad_b=0)
    assert ia.size > 0.2 * 8192


def test_validation_writes_nothing(ours):
    a = np.zeros((2, 2), np.float32)
    b = np.array([[0, 0], [9, 9]], np.float32)
    L = ours
    ra = torch.zeros((2, 3), dtype=torch.float32, device="cuda")
    rb = torch.zeros((2, 4), dtype=torch.float32, device="cuda")
    na = torch.tensor([2], dtype=torch.int32, device="cuda")
    ka = G.Keypoints(0, 0, 0, 2, na.data_ptr())
    da = G.Descriptors(1, 2, 12, ra.data_ptr())
    db = G.Descriptors(1, 2, 16, rb.data_ptr())
    cfg = G.S4Config()
    cfg.ratio_threshold = 0.8
    cfg.cross_check = 1
    b_ = C.c_size_t()
    assert L.s4_workspace_bytes(2, 2, G.ref(cfg), G.ref(b_)) == 0
    ws = G.workspace(b_.value)
    cnt = torch.full((1,), 0x5a5a5a5a, dtype=torch.int32, device="cuda")
    idx = torch.zeros(2, dtype=torch.int32, device="cuda")
    out = G.Matches(idx.data_ptr(), idx.data_ptr(), idx.data_ptr(), 2, cnt.data_ptr())
    s = G.stream()
    call = lambda kA, dA, kB, dB, c, o, w, n: L.s4_match(G.ref(kA), G.ref(dA), G.ref(kB), G.ref(dB), G.ref(c),
                                                       G.ref(o), w, n, s)
    wp = C.c_void_p(ws.data_ptr())
    assert call(ka, da, ka, db, cfg, out, wp, b_.value - 1) == 2
    assert call(ka, da, ka, db, cfg, out, None, b_.value) == 2
    assert call(ka, da, ka, db, cfg, out, C.c_void_p(ws.data_ptr() + 1), b_.value) == 1
    for field, value in (("row_stride_bytes", 4), ("row_stride_bytes", 9), ("type", 0), ("dim", 2 ** 31 - 1),
                         ("data", None), ("type", 9), ("dim", 0)):
        bad = G.Descriptors(1, 2, 12, ra.data_ptr())
        setattr(bad, field, value)
        assert call(ka, bad, ka, db, cfg, out, wp, b_.value) == 1, field
    bad_k = G.Keypoints(0, 0, 0, -1, na.data_ptr())
    assert call(bad_k, da, ka, db, cfg, out, wp, b_.value) == 1
    small = G.Matches(idx.data_ptr(), idx.data_ptr(), idx.data_ptr(), 1, cnt.data_ptr())
    assert call(ka, da, ka, db, cfg, small, wp, b_.value) == 1
    c0 = G.S4Config()
    c0.ratio_threshold = 0.0
    assert call(ka, da, ka, db, c0, out, wp, b_.value) == 1
    torch.cuda.synchronize()
    assert cnt.item() == 0x5a5a5a5a


def test_vs_reference_kernels(ours):
    if not G.ref_available():
        pytest.skip("reference stage build not present")
    theirs = G.Lib("ref")
    for shape, cross in (((1500, 1700), False), ((1500, 1700), True), ((257, 253), True)):
        q, t = planted(*shape, seed=9)
        A = G.match(ours, q, t, 0.8, cross)
        B = G.match(theirs, q, t, 0.8, cross)
        assert np.array_equal(A[0], B[0])
        for x, y in zip(A[1:4], B[1:4]):
            assert np.array_equal(x, y)

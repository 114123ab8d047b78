"""S2/S3 on the GPU through the C ABI: the reference's golden cases bit for
bit (tests/test_s2_s3_cuda.cu:22-39 with exact instead of toleranced
descriptors), contract and reuse checks (:64-194), the large-K fallback, and
agreement with the reference's own kernels built for sm_100a."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import s2s3
from tests import gpu_util as G

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((GOLDEN / "s2s3_manifest.json").read_text())


@pytest.fixture(scope="module")
def ours(cuda):
    return G.Lib("ours")


@pytest.mark.parametrize("name", sorted(MANIFEST["cases"]))
def test_golden_bit_exact(ours, name):
    z = np.load(GOLDEN / MANIFEST["cases"][name]["file"])
    thr, k = (int(v) for v in z["knobs"])
    hk = float(z["harris_k"][0])
    kp, desc, blurred, (st2, st3, n) = G.detect_describe(ours, z["gray"], thr, k, hk)
    assert (st2, st3) == (0, 0)
    assert n == z["keypoints"].shape[0]
    assert np.array_equal(kp, z["keypoints"])
    assert np.array_equal(desc, z["descriptors"])
    if k > 0 and blurred is not None:
        assert np.array_equal(blurred, z["blurred"])
    again = G.detect_describe(ours, z["gray"], thr, k, hk)
    assert np.array_equal(again[0], kp) and np.array_equal(again[1], desc)


def pattern_image(w, h):
    g = np.zeros((h, w), np.uint8)
    state = 12345
    for y in range(h):
        for x in range(w):
            state = (state * 1664525 + 1013904223) & 0xffffffff
            square = x % 20 < 11 and y % 16 < 9
            g[y, x] = (190 if square else 50) + (state >> 28)
    return g


def test_contract_checks(ours):
    w, h = 160, 120
    gray = pattern_image(w, h)
    kp, desc, _, (st2, st3, n) = G.detect_describe(ours, gray, 20, 200)
    assert n > 0 and np.all(np.diff(kp[:, 2]) <= 0)
    assert np.all((kp[:, 0] >= 31) & (kp[:, 0] < w - 31) & (kp[:, 1] >= 31) & (kp[:, 1] < h - 31))
    want_kp, want_desc = s2s3.detect_and_describe(gray, 20, 200)
    assert np.array_equal(kp, want_kp) and np.array_equal(desc, want_desc)
    L = ours
    img = G.pitched(gray)
    iv = G.ImageView(img.data_ptr(), w, h, img.stride(0), 1)
    x = torch.zeros(200, device="cuda")
    cnt = torch.full((1,), 0x7f7f7f7f, dtype=torch.int32, device="cuda")
    kpv = G.Keypoints(x.data_ptr(), x.data_ptr(), 0, 200, cnt.data_ptr())
    cfg = G.S2Config(20, 200, 0.04)
    b = C.c_size_t()
    L.s2_workspace_bytes(w, h, G.ref(cfg), G.ref(b))
    ws = G.workspace(b.value)
    s = G.stream()
    p = C.c_void_p(ws.data_ptr())
    assert L.s2_detect(G.ref(iv), G.ref(cfg), G.ref(kpv), p, b.value - 1, s) == 2
    assert L.s2_detect(G.ref(iv), G.ref(cfg), G.ref(kpv), C.c_void_p(ws.data_ptr() + 1), b.value, s) == 1
    assert L.s2_detect(G.ref(iv), G.ref(G.S2Config(0, 200, 0.04)), G.ref(kpv), p, b.value, s) == 1
    small = G.Keypoints(x.data_ptr(), x.data_ptr(), 0, 199, cnt.data_ptr())
    assert L.s2_detect(G.ref(iv), G.ref(cfg), G.ref(small), p, b.value, s) == 1
    rgb = G.ImageView(img.data_ptr(), w, h, img.stride(0), 0)
    assert L.s2_detect(G.ref(rgb), G.ref(cfg), G.ref(kpv), p, b.value, s) == 1
    torch.cuda.synchronize()
    assert cnt.item() == 0x7f7f7f7f, "failed calls must not write the count"
    d = G.Descriptors(0, 31, 48, x.data_ptr())
    b3 = C.c_size_t()
    L.s3_workspace_bytes(w, h, G.ref(b3))
    ws3 = G.workspace(b3.value)
    assert L.s3_describe(G.ref(iv), G.ref(kpv), G.ref(d), C.c_void_p(ws3.data_ptr()), b3.value, s) == 1
    d = G.Descriptors(1, 32, 48, x.data_ptr())
    assert L.s3_describe(G.ref(iv), G.ref(kpv), G.ref(d), C.c_void_p(ws3.data_ptr()), b3.value, s) == 1
    d = G.Descriptors(0, 32, 48, x.data_ptr())
    assert L.s3_describe(G.ref(iv), G.ref(kpv), G.ref(d), C.c_void_p(ws3.data_ptr()), b3.value - 1, s) == 2
    # K = 0 and images without an interior report zero keypoints
    none = G.Keypoints(0, 0, 0, 0, cnt.data_ptr())
    assert L.s2_detect(G.ref(iv), G.ref(G.S2Config(20, 0, 0.04)), G.ref(none), None, 0, s) == 0
    torch.cuda.synchronize()
    assert cnt.item() == 0
    cnt.fill_(0x7f7f7f7f)
    thin = G.ImageView(img.data_ptr(), w, 62, img.stride(0), 1)
    assert L.s2_detect(G.ref(thin), G.ref(cfg), G.ref(kpv), p, b.value, s) == 0
    torch.cuda.synchronize()
    assert cnt.item() == 0


def test_reuse_buffers_across_sizes(ours):
    """One buffer set sized for (1000x700, K=4000) serves attempts of other
    sizes and K bit-identically (tests/test_s2_s3_cuda.cu:135-194)."""
    attempts = [(1000, 700, 4000), (1000, 700, 500), (500, 350, 2000), (250, 175, 1000), (750, 525, 500),
                (40, 30, 1000), (1000, 700, 1)]
    for w, h, k in attempts:
        gray = pattern_image(w, h)
        exact = G.detect_describe(ours, gray, 20, k)
        big = G.detect_describe(ours, gray, 20, k, capacity=4000)
        assert np.array_equal(exact[0], big[0]) and np.array_equal(exact[1], big[1])
        want_kp, want_desc = s2s3.detect_and_describe(gray, 20, k)
        assert np.array_equal(exact[0], want_kp) and np.array_equal(exact[1], want_desc)


def test_many_candidates_use_fallback_rank(ours):
    """More than 16384 pre-selected points: the global rank path."""
    rng = np.random.default_rng(11)
    gray = rng.integers(0, 256, (1100, 1100), dtype=np.uint8)
    kp, desc, _, (st2, st3, n) = G.detect_describe(ours, gray, 10, 10000)
    want_kp, want_desc = s2s3.detect_and_describe(gray, 10, 10000)
    assert n == want_kp.shape[0] and n == 10000
    assert np.array_equal(kp, want_kp) and np.array_equal(desc, want_desc)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_synthetic_scenes_vs_oracle(ours, seed):
    from crossstage_stitch_b200 import synth
    p = synth.config0_pair(seed)
    for g in (p.gray_a, p.gray_b):
        for thr, k in ((20, 1000), (10, 2000)):
            kp, desc, blurred, _ = G.detect_describe(ours, g, thr, k)
            want_kp, want_desc = s2s3.detect_and_describe(g, thr, k)
            assert np.array_equal(kp, want_kp) and np.array_equal(desc, want_desc)
            assert np.array_equal(blurred, s2s3.blur(g))


def test_vs_reference_kernels(ours):
    """Same inputs through the reference's own S2/S3 kernels (sm_100a build)."""
    if not G.ref_available():
        pytest.skip("reference stage build not present")
    theirs = G.Lib("ref")
    from crossstage_stitch_b200 import synth
    rng = np.random.default_rng(3)
    images = [synth.config0_pair(5).gray_a, rng.integers(0, 256, (333, 257), dtype=np.uint8),
              pattern_image(300, 200)]
    for g in images:
        for thr, k in ((20, 500), (10, 3000), (40, 1)):
            a = G.detect_describe(ours, g, thr, k)
            b = G.detect_describe(theirs, g, thr, k)
            assert a[3][2] == b[3][2]
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])

"""Scale-pyramid S2/S3 (levels > 1) on the GPU against the pyramid oracle:
keypoints (level-0 coordinates, responses) and descriptors bit for bit, per
image through stitch_pyramid_detect_describe, per pair through the plain
chain, and in the batched form against the per-pair path. Parity here is
with the oracle's restatement of OpenCV's layer semantics; the reference
itself is single-level."""
import ctypes as C

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi, batch, stages, synth
from crossstage_stitch_b200._abi import Descriptors, ImageView, Keypoints, PyramidConfig, S2Config
from oracle import chain, pyramid, s2s3

from .gpu_util import pitched, stream, workspace

pytestmark = pytest.mark.gpu
ref = C.byref


def run_pyramid(gray, thr, k, levels, factor, stride=48, capacity=None, pad=None):
    L = _abi.load()
    h, w = gray.shape
    img = pitched(gray) if pad is None else pitched(gray, pad)
    iv = ImageView(img.data_ptr(), w, h, img.stride(0), 1)
    cap = k if capacity is None else capacity
    n = max(cap, 1)
    x = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
    y = torch.full_like(x, -1.0)
    r = torch.full_like(x, -1.0)
    cnt = torch.full((1,), 0x7f7f7f7f, dtype=torch.int32, device="cuda")
    desc = torch.full((n, stride), 0xcd, dtype=torch.uint8, device="cuda")
    cfg, pyr = S2Config(thr, k, 0.04), PyramidConfig(levels, factor)
    b = C.c_size_t()
    assert L.stitch_pyramid_workspace_bytes(w, h, ref(cfg), ref(pyr), ref(b)) == 0
    ws = workspace(b.value)
    kp = Keypoints(x.data_ptr(), y.data_ptr(), r.data_ptr(), cap, cnt.data_ptr())
    ds = Descriptors(0, 32, stride, desc.data_ptr())
    st = L.stitch_pyramid_detect_describe(ref(iv), ref(cfg), ref(pyr), ref(kp), ref(ds), C.c_void_p(ws.data_ptr()),
                                          b.value, stream())
    torch.cuda.synchronize()
    if st != 0:
        return st, None, None
    m = int(cnt.item())
    out_kp = torch.stack([x[:m], y[:m], r[:m]], 1).cpu().numpy() if m else np.zeros((0, 3), np.float32)
    out_desc = desc[:m].cpu().numpy()
    assert (out_desc[:, 32:] == 0xcd).all()  # bytes past the descriptor are untouched
    return st, out_kp, out_desc[:, :32]


def image(kind):
    if kind == "c0a":
        return synth.config0_pair(0).gray_a
    if kind == "c0b":
        return synth.config0_pair(1).gray_b
    if kind == "vga":
        return synth.make_pair(21, 640, 480, overlap=(0.15, 0.7), corrupt=(0.2, 0.7)).gray_b
    if kind == "odd":
        return synth.make_pair(22, 333, 257).gray_a
    if kind == "hd":
        return synth.make_pair(23, 1920, 1080, overlap=(0.15, 0.7)).gray_a
    raise KeyError(kind)


CASES = [
    ("c0a", 20, 1000, 8, 1.2),
    ("c0b", 20, 2000, 8, 1.2),
    ("vga", 10, 500, 4, 1.5),
    ("odd", 20, 300, 8, 1.2),
    ("c0a", 20, 7, 8, 1.2),      # budgets clamped to K
    ("c0a", 40, 20000, 3, 2.0),  # every layer short of its budget
    ("hd", 20, 8000, 8, 1.2),
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-t{c[1]}-k{c[2]}-l{c[3]}-s{c[4]}" for c in CASES])
def test_pyramid_vs_oracle(cuda, case):
    kind, thr, k, levels, factor = case
    gray = image(kind)
    st, kp, desc = run_pyramid(gray, thr, k, levels, factor)
    assert st == 0
    want_kp, want_desc = pyramid.detect_and_describe(gray, thr, k, levels, factor)
    assert kp.shape == want_kp.shape
    assert np.array_equal(kp, want_kp)
    assert np.array_equal(desc, want_desc)


# The resize of layer 1 reads the caller's image: a 16-byte aligned pitch
# takes the staged-window path, the default odd pitch the byte path; layer
# ratios of 3 and 4 leave lanes whose four columns do not fit two 8-byte
# pools (per-lane byte path) and windows beyond the staging buffer.
RESIZE_CASES = [
    ("odd", 1.2), ("odd", 1.45), ("vga", 2.0), ("odd", 3.0), ("vga", 4.0),
]


@pytest.mark.parametrize("case", RESIZE_CASES, ids=[f"{c[0]}-s{c[1]}" for c in RESIZE_CASES])
@pytest.mark.parametrize("aligned", [True, False], ids=["pitch16", "pitch-odd"])
def test_pyramid_resize_paths_vs_oracle(cuda, case, aligned):
    kind, factor = case
    gray = image(kind)
    w = gray.shape[1]
    pad = (-w) % 16 + 16 if aligned else None
    st, kp, desc = run_pyramid(gray, 20, 800, 4, factor, pad=pad)
    assert st == 0
    want_kp, want_desc = pyramid.detect_and_describe(gray, 20, 800, 4, factor)
    assert np.array_equal(kp, want_kp)
    assert np.array_equal(desc, want_desc)


def test_single_level_equals_stage_path(cuda):
    gray = image("c0a")
    st, kp, desc = run_pyramid(gray, 20, 1000, 1, 1.2)
    assert st == 0
    want_kp, want_desc = s2s3.detect_and_describe(gray, 20, 1000)
    assert np.array_equal(kp, want_kp) and np.array_equal(desc, want_desc)


def test_empty_and_small(cuda):
    gray = image("c0a")
    st, kp, _ = run_pyramid(gray, 20, 0, 8, 1.2)
    assert st == 0 and kp.shape == (0, 3)
    rng = np.random.default_rng(4)
    tiny = rng.integers(0, 256, (60, 200), dtype=np.uint8)
    st, kp, _ = run_pyramid(tiny, 20, 100, 8, 1.2)
    assert st == 0 and kp.shape == (0, 3)
    flat = np.full((300, 300), 77, np.uint8)
    st, kp, _ = run_pyramid(flat, 20, 100, 8, 1.2)
    assert st == 0 and kp.shape == (0, 3)


def test_capacity_below_k_is_rejected(cuda):
    st, _, _ = run_pyramid(image("c0a"), 20, 100, 8, 1.2, capacity=50)
    assert st == 1


@pytest.mark.parametrize("index", range(2))
def test_chain_vs_oracle(cuda, index):
    p = synth.config0_pair(index)
    knobs = stages.Knobs(max_keypoints=1000, hypotheses=2000, seed=synth.BASE_SEED + index, levels=8,
                         scale_factor=1.2)
    runner = stages.PairRunner(512, 512, 1000, max_r=2000)
    res = runner.run(p.gray_a, p.gray_b, knobs)
    got = runner.download()
    want = chain.run_pair(p.gray_a, p.gray_b, knobs)
    for tag in "ab":
        assert np.array_equal(got[f"kp_{tag}"], want[f"kp_{tag}"])
        assert np.array_equal(got[f"desc_{tag}"], want[f"desc_{tag}"])
    assert np.array_equal(got["idx_a"], want["idx_a"]) and np.array_equal(got["idx_b"], want["idx_b"])
    assert np.array_equal(got["mask"], want["mask"])
    assert int(res["status"]) == want["status"]
    if want["status"] == 0:
        assert synth.max_corner_error(res["H"], want["H"], 512, 512) < 1e-3
        assert res["num_inliers"] == want["num_inliers"]


def test_batch_mixed_levels_equals_per_pair(cuda):
    cases = []
    for i in range(3):
        p = synth.config0_pair(i)
        cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=2000, seed=100 + i, levels=8)))
    p = synth.make_pair(7, 640, 480, overlap=(0.15, 0.7), corrupt=(0.2, 0.7))
    cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=500, fast_threshold=10, hypotheses=500,
                                                    cross_check=True, seed=5, levels=5, scale_factor=1.5)))
    p = synth.config0_pair(4)
    cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=1000, seed=9)))  # single level
    rng = np.random.default_rng(4)
    tiny = rng.integers(0, 256, (60, 200), dtype=np.uint8)
    cases.append((tiny, tiny.copy(), stages.Knobs(max_keypoints=100, hypotheses=64, seed=2, levels=8)))
    p = synth.config0_pair(5)
    cases.append((p.gray_a, p.gray_b[:300, :420].copy(), stages.Knobs(max_keypoints=7, hypotheses=64, seed=3,
                                                                      levels=8)))
    W = max(max(a.shape[1], b.shape[1]) for a, b, _ in cases)
    H = max(max(a.shape[0], b.shape[0]) for a, b, _ in cases)
    runner = stages.PairRunner(W, H, 2000, max_r=2000, cross_check=True)
    want = []
    for a, b, k in cases:
        res = runner.run(a, b, k)
        want.append((res, runner.download()))
    imgs = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b, _ in cases]
    bt = batch.Batch([batch.pair_desc(ia, ib, k) for (ia, ib), (_, _, k) in zip(imgs, cases)])
    bt.capture()
    bt.ws.fill_(0xcd)
    for _ in range(2):
        bt.launch()
        torch.cuda.synchronize()
        for i, (res, dl) in enumerate(want):
            got = bt.outputs(i)
            for key in ("kp_a", "kp_b", "desc_a", "desc_b", "idx_a", "idx_b", "distance", "mask"):
                assert np.array_equal(got[key], dl[key]), (i, key)
            r = bt.result(i)
            assert r["status"] == res["status"] and r["num_inliers"] == res["num_inliers"]
            np.testing.assert_array_equal(r["H"], res["H"])


@pytest.mark.parametrize("kind,k", [("c0a", 1000), ("c0b", 1000), ("c1", 2000)])
def test_pyramid_layers_equal_reference_kernels(cuda, kind, k):
    """Each pyramid layer runs the reference's single-level S2/S3 unchanged.
    The reference's own S2/S3 kernels (src/s2_s3/s2.cu:333-385,
    src/s2_s3/s3.cu:168-195, built for sm_100a into oracle/_ref as a
    checker), run on each layer image of the pyramid oracle with that layer's
    budget, give this library's pyramid output layer by layer: the same
    counts, responses and descriptors bit for bit, and x and y equal to the
    reference's layer coordinates times s_l in float32 (the one step the
    pyramid adds)."""
    from . import gpu_util as G
    if not G.ref_available():
        pytest.skip("reference stage build not present (oracle/_ref)")
    gray = synth.config0_pair(2).gray_a if kind == "c1" else image(kind)
    levels, factor, thr = 8, 1.2, 20
    st, kp, desc = run_pyramid(gray, thr, k, levels, factor)
    assert st == 0
    budgets = pyramid.level_budgets(k, levels, factor)
    scales = pyramid.layer_scales(levels, factor)
    lib = G.Lib("ref")
    off = 0
    layers = pyramid.build_layers(gray, levels, factor)
    assert len(layers) == levels
    for l, layer in enumerate(layers):
        rk, rd, _, (s2, s3, n) = G.detect_describe(lib, layer, thr, budgets[l])
        assert (s2, s3) == (0, 0) and n == rk.shape[0] > 0, l
        span = slice(off, off + n)
        assert np.array_equal(kp[span, 0], rk[:, 0] * scales[l]), l
        assert np.array_equal(kp[span, 1], rk[:, 1] * scales[l]), l
        assert np.array_equal(kp[span, 2], rk[:, 2]), l
        assert np.array_equal(desc[span], rd), l
        off += n
    assert off == kp.shape[0]

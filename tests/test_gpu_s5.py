"""S5 on the GPU through the C ABI: the reference's own known-answer and
contract tests (tests/test_s5_cuda.cu:99-186), bit-for-bit agreement with the
CPU oracle (same hypothesis sequence -> same winner, same inlier mask,
identical H), and agreement with the reference's kernels (identical inlier
set, corners within 1e-3 px)."""
import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import synth
from oracle import c_oracle
from tests import gpu_util as G
from tests.test_oracle_s5 import TRUTH, hdiff, known_answer_points

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ours(cuda):
    return G.Lib("ours")


def load_known(f, outliers=True, line=False):
    pts = known_answer_points(outliers, line)
    f.set_points(pts[:, 0:2], pts[:, 2:4])


def test_known_h_and_outliers(ours):
    f = G.S5Fixture(ours, 80)
    load_known(f)
    r = f.run()
    assert r["status"] == 0 and r["num_matches"] == 80 and r["num_inliers"] == 60
    assert abs(r["inlier_ratio"] - 0.75) < 1e-12
    assert 0 < r["inlier_coverage"] <= 1 and r["reproj_residual"] < 1e-3
    assert hdiff(r["H_s"], TRUTH) < 1e-3 and hdiff(r["H"], TRUTH) < 1e-3
    assert np.array_equal(f.mask_host(), np.array([i % 4 != 0 for i in range(80)], np.uint8))


def test_incremental_equals_full(ours):
    f = G.S5Fixture(ours, 80)
    load_known(f)
    full = f.run()
    full_mask = f.mask_host()
    f.config.hypotheses = 17
    assert f.run()["status"] == 0
    f.config.previous_hypotheses, f.config.hypotheses = 17, 257
    split = f.run()
    assert full["status"] == split["status"] and full["num_inliers"] == split["num_inliers"]
    assert np.array_equal(full["H"], split["H"]) and np.array_equal(full["H_s"], split["H_s"])
    assert full["inlier_ratio"] == split["inlier_ratio"] and full["inlier_coverage"] == split["inlier_coverage"]
    assert full["reproj_residual"] == split["reproj_residual"]
    assert np.array_equal(full_mask, f.mask_host())


def test_resize_and_repeatability(ours):
    f = G.S5Fixture(ours, 80)
    load_known(f, outliers=False)
    L = G._abi.load()
    assert L.stitch_make_scale_info(1281, 961, 0.5, G.ref(f.sa)) == 0
    assert L.stitch_make_scale_info(1281, 961, 0.75, G.ref(f.sb)) == 0
    first, second = f.run(), f.run()
    assert first["status"] == 0 and second["status"] == 0
    sa = np.array(f.sa.D[:])
    sb = np.array(f.sb.D[:])
    expected = np.linalg.inv(sa.reshape(3, 3)) @ first["H_s"].reshape(3, 3) @ sb.reshape(3, 3)
    assert hdiff(first["H"], expected) < 1e-10
    assert np.array_equal(first["H"], second["H"])


def test_failed_data_and_stale_state(ours):
    f = G.S5Fixture(ours, 80)
    load_known(f, outliers=False)
    f.nm.fill_(3)
    assert f.run()["status"] == 4
    assert not f.mask.cpu().numpy()[:80].any()
    f.nm.fill_(80)
    load_known(f, outliers=False, line=True)
    assert f.run()["status"] == 5
    load_known(f, outliers=False)
    assert f.run()["status"] == 0
    f.config.previous_hypotheses = f.config.hypotheses
    f.config.generation += 1
    stale = f.run()
    assert stale["status"] == 1 and np.isnan(stale["H"][0])
    f.config.previous_hypotheses = 0
    assert f.run()["status"] == 0
    f.ia[:80] = 80
    assert f.run()["status"] == 1
    load_known(f, outliers=False)
    f.nm.fill_(81)
    assert f.run()["status"] == 1


def test_host_boundary_errors(ours):
    f = G.S5Fixture(ours, 80)
    load_known(f)
    assert f.call(ws_bytes=f.bytes - 1) == 2
    assert f.call(ws_offset=1) == 1
    f.config.threshold = float("inf")
    assert f.call() == 1


def oracle_s5(f, a, b, ia, ib, hyp, tau, seed, refine, prev=None, first=0):
    pts = np.stack([a[ia, 0], a[ia, 1], b[ib, 0], b[ib, 1]], 1).astype(np.float32).astype(np.float64)
    sa = c_oracle.make_scale_info(f.sa.orig_w, f.sa.orig_h, f.sa.work_w / f.sa.orig_w)
    sb = c_oracle.make_scale_info(f.sb.orig_w, f.sb.orig_h, f.sb.work_w / f.sb.orig_w)
    sa["D"], sb["D"] = np.array(f.sa.D[:]), np.array(f.sb.D[:])
    return c_oracle.s5(pts, f.cap, hyp, tau, seed, refine, sa, sb, 0 if len(ia) >= 4 else 4, prev, first)


def synthetic_matches(seed, n, outlier_frac, w=640, h=480):
    rng = np.random.default_rng(seed)
    H = synth.random_homography(rng, w, h, (0.5, 0.8))
    b = rng.uniform([0, 0], [w - 1, h - 1], (n, 2))
    z = H[2, 0] * b[:, 0] + H[2, 1] * b[:, 1] + H[2, 2]
    a = np.stack([(H[0, 0] * b[:, 0] + H[0, 1] * b[:, 1] + H[0, 2]) / z,
                  (H[1, 0] * b[:, 0] + H[1, 1] * b[:, 1] + H[1, 2]) / z], 1)
    a += rng.normal(0, 1.0, a.shape)
    bad = rng.random(n) < outlier_frac
    a[bad] = rng.uniform([0, 0], [w - 1, h - 1], (bad.sum(), 2))
    a = np.rint(a).astype(np.float32)   # keypoints sit on pixel centres
    b = np.rint(b).astype(np.float32)
    perm = rng.permutation(n)
    return a, b, np.arange(n), perm, b[perm]


@pytest.mark.parametrize("seed,n,frac,R,refine", [(1, 300, 0.3, 2000, 1), (2, 1000, 0.5, 2000, 1),
                                                   (3, 120, 0.7, 500, 3), (4, 5000, 0.4, 800, 1),
                                                   (5, 4, 0.0, 64, 1), (6, 60, 0.2, 8000, 0)])
def test_bitwise_vs_oracle(ours, seed, n, frac, R, refine):
    a, b_orig, ia, perm, b = synthetic_matches(seed, n, frac)
    # match i pairs a[i] with b_orig[i] = b[inverse(perm)[i]]
    inv = np.argsort(perm)
    f = G.S5Fixture(ours, n)
    f.set_points(a, b, ia, inv)
    f.config.hypotheses, f.config.threshold, f.config.seed, f.config.refinement_steps = R, 3.0, seed * 977, refine
    got = f.run()
    want, wmask, _ = oracle_s5(f, a, b, ia, inv, R, 3.0, seed * 977, refine)
    assert got["status"] == want["status"]
    assert got["num_inliers"] == want["num_inliers"]
    assert np.array_equal(f.mask_host(), wmask[:n])
    if want["status"] == 0:
        assert np.array_equal(got["H_s"], want["H_s"].reshape(9))
        assert np.array_equal(got["H"], want["H"].reshape(9))
        assert got["reproj_residual"] == want["reproj_residual"]
        assert got["inlier_coverage"] == want["inlier_coverage"]


def test_split_search_vs_oracle(ours):
    a, b_orig, ia, perm, b = synthetic_matches(9, 700, 0.45)
    inv = np.argsort(perm)
    f = G.S5Fixture(ours, 700)
    f.set_points(a, b, ia, inv)
    f.config.hypotheses, f.config.threshold, f.config.seed = 300, 3.0, 5
    f.run()
    f.config.previous_hypotheses, f.config.hypotheses = 300, 1900
    got = f.run()
    want, wmask, _ = oracle_s5(f, a, b, ia, inv, 1900, 3.0, 5, f.config.refinement_steps)
    assert np.array_equal(got["H"], want["H"].reshape(9)) and np.array_equal(f.mask_host(), wmask[:700])


def test_vs_reference_kernels(ours):
    """The reference's kernels (default nvcc contraction) pick the same
    inlier set; the homographies agree to well under 1e-3 px at the corners."""
    if not G.ref_available():
        pytest.skip("reference stage build not present")
    theirs = G.Lib("ref")
    for seed, n, frac in ((11, 400, 0.3), (12, 900, 0.5), (13, 150, 0.6)):
        a, b_orig, ia, perm, b = synthetic_matches(seed, n, frac)
        inv = np.argsort(perm)
        out = []
        for lib in (ours, theirs):
            f = G.S5Fixture(lib, n)
            f.set_points(a, b, ia, inv)
            # batch_size stays at the fixture's 32: the reference sizes its
            # workspace by it (src/s5/s5_config.cpp:14-17)
            f.config.hypotheses, f.config.threshold, f.config.seed = 2000, 3.0, seed
            out.append((f.run(), f.mask_host()))
        (r1, m1), (r2, m2) = out
        assert r1["status"] == r2["status"] == 0
        assert np.array_equal(m1, m2)
        assert synth.max_corner_error(r1["H"].reshape(3, 3), r2["H"].reshape(3, 3), 640, 480) < 1e-3

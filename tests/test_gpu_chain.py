"""The plain per-pair chain (S2, S2, S3, S3, S4, S5 on one stream, as the
reference harness runs it) against the CPU oracle chain on synthetic pairs of
the registration workload: keypoints, descriptors and matches bit for bit,
identical inlier masks, homography corners within 1e-3 px of the FP64
oracle."""
import numpy as np
import pytest

from crossstage_stitch_b200 import stages, synth
from oracle import chain

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def runner(cuda):
    return stages.PairRunner(640, 512, 2000, max_r=2000)


@pytest.mark.parametrize("index", range(4))
@pytest.mark.parametrize("k", [1000, 2000])
def test_chain_vs_oracle(runner, index, k):
    p = synth.config0_pair(index)
    knobs = stages.Knobs(max_keypoints=k, hypotheses=2000, seed=synth.BASE_SEED + index)
    res = runner.run(p.gray_a, p.gray_b, knobs)
    got = runner.download()
    want = chain.run_pair(p.gray_a, p.gray_b, knobs)
    for tag in "ab":
        assert np.array_equal(got[f"kp_{tag}"], want[f"kp_{tag}"])
        assert np.array_equal(got[f"desc_{tag}"], want[f"desc_{tag}"])
    assert np.array_equal(got["idx_a"], want["idx_a"]) and np.array_equal(got["idx_b"], want["idx_b"])
    assert np.array_equal(got["distance"], want["distance"])
    assert int(res["status"]) == want["status"]
    assert np.array_equal(got["mask"], want["mask"])
    if want["status"] == 0:
        assert synth.max_corner_error(res["H"], want["H"], 512, 512) < 1e-3
        assert res["num_inliers"] == want["num_inliers"]


def test_mixed_resolution_pair_vs_oracle(cuda):
    p, kn = synth.mixed_pair(1)
    h, w = p.gray_a.shape
    r = stages.PairRunner(w, h, kn["max_keypoints"], max_r=kn["hypotheses"])
    knobs = stages.Knobs(max_keypoints=kn["max_keypoints"], fast_threshold=kn["fast_threshold"],
                         hypotheses=kn["hypotheses"], seed=17)
    res = r.run(p.gray_a, p.gray_b, knobs)
    got = r.download()
    want = chain.run_pair(p.gray_a, p.gray_b, knobs)
    for tag in "ab":
        assert np.array_equal(got[f"kp_{tag}"], want[f"kp_{tag}"])
        assert np.array_equal(got[f"desc_{tag}"], want[f"desc_{tag}"])
    assert np.array_equal(got["idx_a"], want["idx_a"])
    assert np.array_equal(got["mask"], want["mask"])
    assert int(res["status"]) == want["status"]

"""The mixed-resolution workload at its full sizes: a batch holding a
3840x2160 and a 1920x1080 pair at 8 levels (K = 8000, FAST 10, R = 8000)
and a 640x480 pair (K = 500), run by the batched form (captured graph,
replayed twice over a poisoned workspace) against the per-pair drop-in
stages: every keypoint, descriptor, match, mask and homography result bit
for bit. The 1920x1080 pair is also checked against the CPU oracle chain:
keypoints, descriptors and matches bit for bit, the inlier mask identical
and the homography corners within 1e-3 px of the FP64 oracle."""
import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import batch, stages, synth
from oracle import chain

from .test_gpu_batch import compare

pytestmark = pytest.mark.gpu

SEED = synth.BASE_SEED + 300000


def cases():
    big = dict(max_keypoints=8000, fast_threshold=10, hypotheses=8000, levels=8, scale_factor=1.2)
    out = []
    p = synth.make_pair(SEED, 3840, 2160, overlap=(0.15, 0.7), corrupt=(0.2, 0.7))
    out.append((p.gray_a, p.gray_b, stages.Knobs(seed=SEED, **big)))
    p = synth.make_pair(SEED + 1, 1920, 1080, overlap=(0.15, 0.7), corrupt=(0.2, 0.7))
    out.append((p.gray_a, p.gray_b, stages.Knobs(seed=SEED + 1, **big)))
    p = synth.make_pair(SEED + 2, 640, 480, overlap=(0.15, 0.7), corrupt=(0.2, 0.7))
    out.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=500, fast_threshold=20, hypotheses=2000,
                                                  levels=8, scale_factor=1.2, seed=SEED + 2)))
    return out


@pytest.fixture(scope="module")
def full(cuda):
    cs = cases()
    W = max(max(a.shape[1], b.shape[1]) for a, b, _ in cs)
    H = max(max(a.shape[0], b.shape[0]) for a, b, _ in cs)
    runner = stages.PairRunner(W, H, 8000, max_r=8000)
    per_pair = []
    for a, b, k in cs:
        res = runner.run(a, b, k)
        per_pair.append((res, runner.download()))
    del runner
    torch.cuda.empty_cache()
    return cs, per_pair


def test_full_size_batch_equals_per_pair(full):
    cs, per_pair = full
    imgs = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b, _ in cs]
    b = batch.Batch([batch.pair_desc(ia, ib, k) for (ia, ib), (_, _, k) in zip(imgs, cs)])
    b.capture()
    b.ws.fill_(0xcd)  # replays must not depend on anything the capture run left
    for _ in range(2):
        b.launch()
        torch.cuda.synchronize()
        for i, (res, dl) in enumerate(per_pair):
            compare(b, i, res, dl)
    # the large pairs really are large: thousands of keypoints and a model
    for i in range(2):
        assert len(per_pair[i][1]["kp_a"]) > 4000 and per_pair[i][0]["status"] == 0


def test_full_size_1080p_pair_vs_oracle(full):
    cs, per_pair = full
    a, bb, k = cs[1]
    res, got = per_pair[1]
    want = chain.run_pair(a, bb, k)
    for tag in "ab":
        assert np.array_equal(got[f"kp_{tag}"], want[f"kp_{tag}"])
        assert np.array_equal(got[f"desc_{tag}"], want[f"desc_{tag}"])
    assert np.array_equal(got["idx_a"], want["idx_a"]) and np.array_equal(got["idx_b"], want["idx_b"])
    assert int(res["status"]) == want["status"] == 0
    assert np.array_equal(got["mask"], want["mask"])
    assert res["num_inliers"] == want["num_inliers"]
    assert synth.max_corner_error(res["H"], want["H"], 1920, 1080) < 1e-3

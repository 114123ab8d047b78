"""The batched form (one launch per stage kernel for all pairs, plain
enqueue and captured CUDA graph) against the per-pair drop-in path: every
keypoint, descriptor, match, mask and homography result bit for bit, for a
batch of uneven pairs (sizes, K, R, FAST threshold, mutual check, K = 0 and
an image too small to have an interior)."""
import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import batch, stages, synth

pytestmark = pytest.mark.gpu


def make_cases():
    cases = []
    for i in range(3):
        p = synth.config0_pair(i)
        cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=2000, hypotheses=2000, seed=100 + i)))
    p = synth.make_pair(7, 640, 480, overlap=(0.15, 0.7), corrupt=(0.2, 0.7))
    cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=500, fast_threshold=10, hypotheses=500,
                                                    cross_check=True, seed=5)))
    p = synth.make_pair(8, 1280, 720, overlap=(0.15, 0.7), corrupt=(0.2, 0.7))
    cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=8000, fast_threshold=20, hypotheses=8000,
                                                    seed=6)))
    p = synth.config0_pair(9)
    cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=0, hypotheses=64, seed=1)))
    rng = np.random.default_rng(4)
    tiny = rng.integers(0, 256, (60, 200), dtype=np.uint8)
    cases.append((tiny, tiny.copy(), stages.Knobs(max_keypoints=100, hypotheses=64, seed=2)))
    p = synth.config0_pair(10)
    cases.append((p.gray_a, p.gray_b[:400, :480].copy(), stages.Knobs(max_keypoints=1000, fast_threshold=40,
                                                                      hypotheses=3000, refinement_steps=3,
                                                                      seed=11)))
    return cases


@pytest.fixture(scope="module")
def cases(cuda):
    return make_cases()


@pytest.fixture(scope="module")
def per_pair(cases):
    W = max(max(a.shape[1], b.shape[1]) for a, b, _ in cases)
    H = max(max(a.shape[0], b.shape[0]) for a, b, _ in cases)
    K = max(k.max_keypoints for _, _, k in cases)
    runner = stages.PairRunner(W, H, max(K, 1), max_r=8000, cross_check=True)
    out = []
    for a, b, k in cases:
        res = runner.run(a, b, k)
        out.append((res, runner.download()))
    return out


def device_images(cases):
    return [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b, _ in cases]


def compare(b, i, want_res, want):
    got = b.outputs(i)
    for key in ("kp_a", "kp_b", "desc_a", "desc_b", "idx_a", "idx_b", "distance", "mask"):
        assert np.array_equal(got[key], want[key]), (i, key)
    r = b.result(i)
    assert r["status"] == want_res["status"], i
    assert r["num_matches"] == want_res["num_matches"] and r["num_inliers"] == want_res["num_inliers"]
    for key in ("H", "H_s"):
        np.testing.assert_array_equal(r[key], want_res[key])
    for key in ("inlier_ratio", "inlier_coverage", "reproj_residual"):
        assert (r[key] == want_res[key]) or (np.isnan(r[key]) and np.isnan(want_res[key])), (i, key)


def test_batch_enqueue_equals_per_pair(cases, per_pair):
    imgs = device_images(cases)
    descs = [batch.pair_desc(ia, ib, k) for (ia, ib), (_, _, k) in zip(imgs, cases)]
    b = batch.Batch(descs)
    b.enqueue()
    torch.cuda.synchronize()
    for i, (res, dl) in enumerate(per_pair):
        compare(b, i, res, dl)
    b.enqueue()   # a second run over the same workspace gives the same results
    torch.cuda.synchronize()
    for i, (res, dl) in enumerate(per_pair):
        compare(b, i, res, dl)


def test_batch_graph_equals_per_pair(cases, per_pair):
    imgs = device_images(cases)
    descs = [batch.pair_desc(ia, ib, k) for (ia, ib), (_, _, k) in zip(imgs, cases)]
    b = batch.Batch(descs)
    b.capture()
    b.ws.fill_(0xcd)  # replays must not depend on leftovers of the capture run
    for _ in range(2):
        b.launch()
        torch.cuda.synchronize()
        for i, (res, dl) in enumerate(per_pair):
            compare(b, i, res, dl)


def test_batch_rejects_invalid_pair(cuda):
    img = torch.zeros((100, 100), dtype=torch.uint8, device="cuda")
    good = batch.pair_desc(img, img, stages.Knobs(max_keypoints=10, hypotheses=16))
    bad = batch.pair_desc(img, img, stages.Knobs(max_keypoints=10, hypotheses=16, ratio=1.5))
    with pytest.raises(Exception) as e:
        batch.Batch([good, bad])
    assert "pair 1" in str(e.value)


def test_streaming_batches_equal_a_plain_batch(cuda):
    """Two alternating slots fed from pinned host buffers (copy overlapped
    with the previous step) give each step's pairs the results of a plain
    batch over the same images, bit for bit."""
    import torch

    from crossstage_stitch_b200.batch import Batch, StreamingBatches, pair_desc

    pairs = [synth.config0_pair(90 + i) for i in range(6)]
    knobs = [stages.Knobs(max_keypoints=1000, seed=900 + i, levels=8) for i in range(6)]
    sizes = [(p.gray_a.shape[1], p.gray_a.shape[0], p.gray_b.shape[1], p.gray_b.shape[0]) for p in pairs]
    sb = StreamingBatches(sizes, knobs)
    hosts = [sb.host_buffer(), sb.host_buffer()]
    order = [pairs, pairs[::-1]]  # step 1 feeds the pairs in reverse order under the same knobs
    for h, ps in zip(hosts, order):
        for i, p in enumerate(ps):
            sb.fill(h, i, p.gray_a, p.gray_b)
    got = []
    prev = None
    for step in range(4):
        s = sb.step(hosts[step % 2])
        if prev is not None:
            sb.wait(prev)
            got.append([sb.result(prev, i) for i in range(6)])
        prev = s
    sb.wait(prev)
    got.append([sb.result(prev, i) for i in range(6)])
    for step, res in enumerate(got):
        ps = order[step % 2]
        imgs = [(torch.from_numpy(p.gray_a).cuda(), torch.from_numpy(p.gray_b).cuda()) for p in ps]
        ref = Batch([pair_desc(a, b, k) for (a, b), k in zip(imgs, knobs)])
        ref.enqueue()
        torch.cuda.synchronize()
        for i in range(6):
            np.testing.assert_array_equal(res[i]["H"], ref.result(i)["H"])
            assert res[i]["num_inliers"] == ref.result(i)["num_inliers"]

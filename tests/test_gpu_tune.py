"""The autotuned, bucketed batched form: pairs of several resolution buckets
and K classes split into one tuned plan (own launch shapes and graph) per
bucket, replayed on several streams, give every pair the result of one
untuned plan over all pairs, bit for bit; the tuner's choices land in its
JSON cache and are reused."""
import json

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import batch, stages, synth, tune

pytestmark = pytest.mark.gpu


def test_bucketed_tuned_equals_single_plan(cuda, tmp_path):
    spec = [(640, 480, 500), (640, 480, 2000), (1280, 720, 2000), (512, 512, 1000), (1280, 720, 500)]
    pairs = []
    for i, (w, h, k) in enumerate(spec):
        p = synth.make_pair(synth.BASE_SEED + 700 + i, w, h, overlap=(0.15, 0.7), corrupt=(0.2, 0.7))
        kn = stages.Knobs(max_keypoints=k, fast_threshold=(10, 20, 40)[i % 3], hypotheses=(500, 2000)[i % 2],
                          seed=70 + i, levels=8)
        pairs.append((torch.from_numpy(p.gray_a).cuda(), torch.from_numpy(p.gray_b).cuda(), kn))
    single = batch.Batch([batch.pair_desc(a, b, k) for a, b, k in pairs])
    single.enqueue()
    torch.cuda.synchronize()
    cache = tmp_path / "tuning.json"
    tuner = tune.Tuner(cache, reps=1)
    bb = tune.BucketedBatch(pairs, tuner=tuner, streams=3)
    assert len(bb.batches) == 4   # (vga, k500) (vga, k2000) (720p, k2000) (720p, k500); 512x512 K=1000 -> (vga, k500)
    for _ in range(2):
        bb.launch()
        torch.cuda.synchronize()
        for i in range(len(pairs)):
            got, want = bb.result(i), single.result(i)
            assert got["status"] == want["status"] and got["num_inliers"] == want["num_inliers"]
            np.testing.assert_array_equal(got["H"], want["H"])
    table = json.loads(cache.read_text())
    assert len(table) == 4 and all(set(v["tuning"]) == set(tune.SPACE) for v in table.values())
    again = tune.Tuner(cache, reps=1)
    assert again.tune(("vga", "k500"), pairs[:1]) == table[again.key(("vga", "k500"))]["tuning"]

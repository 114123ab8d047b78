"""The reference's own stage sources built for sm_100a, driven pair by pair
the way harness/pipeline_runner.cu:366-416 drives them (S2 A, S2 B, S3 A,
S3 B, S4, S5 on one stream, one synchronisation per pair), next to this
library's plain per-pair form, on the same GPU and pairs: single level
(the reference has no pyramid), K = 1000 and 2000, R = 2000.

Checked: with the checker build of the reference (S2/S3 at -Xptxas -O0,
oracle/Makefile) the keypoints, descriptors and matches equal ours bit for
bit and the inlier masks are identical. Timed (printed as one JSON line per
K with -s): this library, the checker build and the reference's stock build
(its own flags throughout; CUDA 12.9 ptxas miscompiles its FAST score at
-O1 and above, so that build is a timing baseline only)."""
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi, stages, synth

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"
STAGES = ("s2_workspace_bytes", "s2_detect", "s3_workspace_bytes", "s3_describe", "s4_workspace_bytes",
          "s4_match", "s5_workspace_bytes", "s5_estimate")
N_TIMED = 16


class RefStages:
    """The stitch_* stage entry points served by a reference build."""

    def __init__(self, path: Path):
        if not path.exists():
            pytest.skip(f"reference stage build not present ({path.name})")
        self.L = C.CDLL(str(path))
        for name in STAGES:
            fn = getattr(self.L, "ref_" + name)
            fn.restype = C.c_int
            fn.argtypes = _abi.PROTOTYPES["stitch_" + name][1]
            setattr(self, "stitch_" + name, fn)


def timed(runner, pairs, knobs):
    """Per-pair device time (events around the six stage calls) and wall
    time (upload excluded, synchronisation included)."""
    stream = torch.cuda.current_stream()
    dev_ms, wall = [], 0.0
    for i, p in enumerate(pairs):
        runner.upload(p.gray_a, p.gray_b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t = time.perf_counter()
        e0.record(stream)
        (ha, wa), (hb, wb) = p.gray_a.shape, p.gray_b.shape
        runner.enqueue(wa, ha, wb, hb, knobs[i])
        e1.record(stream)
        stream.synchronize()
        wall += time.perf_counter() - t
        dev_ms.append(e0.elapsed_time(e1))
    dev_ms.sort()
    return {"pairs_per_s": len(pairs) / wall, "device_ms_p50": dev_ms[len(dev_ms) // 2],
            "device_ms_max": dev_ms[-1]}


@pytest.mark.parametrize("k", [1000, 2000])
def test_reference_chain_parity_and_timing(cuda, k):
    pairs = [synth.config0_pair(i) for i in range(N_TIMED)]
    knobs = [stages.Knobs(max_keypoints=k, hypotheses=2000, seed=synth.BASE_SEED + i) for i in range(N_TIMED)]
    ours = stages.PairRunner(512, 512, k, max_r=2000)
    checker = stages.PairRunner(512, 512, k, max_r=2000, stage_lib=RefStages(REF / "libref_stages.so"))
    stock = stages.PairRunner(512, 512, k, max_r=2000, stage_lib=RefStages(REF / "libref_stages_stock.so"))
    for i in range(4):
        p = pairs[i]
        r_ours = ours.run(p.gray_a, p.gray_b, knobs[i])
        r_ref = checker.run(p.gray_a, p.gray_b, knobs[i])
        a, b = ours.download(), checker.download()
        for key in ("kp_a", "kp_b", "desc_a", "desc_b", "idx_a", "idx_b", "distance", "mask"):
            assert np.array_equal(a[key], b[key]), (i, key)
        assert int(r_ours["status"]) == int(r_ref["status"])
        assert r_ours["num_inliers"] == r_ref["num_inliers"]
        if int(r_ours["status"]) == 0:
            assert synth.max_corner_error(r_ours["H"], r_ref["H"], 512, 512) < 1e-3
    out = {"workload": f"{N_TIMED} synthetic 512x512 pairs, single level, K={k}, FAST 20, R=2000, tau 3 px, "
                       f"one synchronisation per pair",
           "ours": None, "reference_checker": None, "reference_stock": None}
    for name, runner in (("ours", ours), ("reference_checker", checker), ("reference_stock", stock)):
        timed(runner, pairs[:3], knobs[:3])  # warm-up
        out[name] = timed(runner, pairs, knobs)
    out["ours_over_stock"] = out["ours"]["pairs_per_s"] / out["reference_stock"]["pairs_per_s"]
    print("\nREFERENCE_CHAIN " + json.dumps(out))


def test_reference_chain_mixed_resolution(cuda):
    """Mixed resolution (640x480 .. 3840x2160, per-pair K, FAST and R), single
    level: the reference's stock kernels pair by pair, this library's plain
    per-pair form, and its batched form (one graph for all pairs) on the
    same pairs; the checker build equals ours bit for bit on two pairs."""
    from crossstage_stitch_b200 import batch

    items = [synth.mixed_pair(i) for i in range(16)]
    pairs = [p for p, _ in items]
    knobs = [stages.Knobs(max_keypoints=kn["max_keypoints"], fast_threshold=kn["fast_threshold"],
                          hypotheses=kn["hypotheses"], seed=synth.BASE_SEED + i) for i, (_, kn) in enumerate(items)]
    W = max(max(p.gray_a.shape[1], p.gray_b.shape[1]) for p in pairs)
    H = max(max(p.gray_a.shape[0], p.gray_b.shape[0]) for p in pairs)
    K = max(k.max_keypoints for k in knobs)
    R = max(k.hypotheses for k in knobs)
    ours = stages.PairRunner(W, H, K, max_r=R)
    checker = stages.PairRunner(W, H, K, max_r=R, stage_lib=RefStages(REF / "libref_stages.so"))
    stock = stages.PairRunner(W, H, K, max_r=R, stage_lib=RefStages(REF / "libref_stages_stock.so"))
    small = sorted(range(16), key=lambda i: pairs[i].gray_a.size)[:2]
    for i in small:
        p = pairs[i]
        r_ours = ours.run(p.gray_a, p.gray_b, knobs[i])
        r_ref = checker.run(p.gray_a, p.gray_b, knobs[i])
        a, b = ours.download(), checker.download()
        for key in ("kp_a", "kp_b", "desc_a", "desc_b", "idx_a", "idx_b", "distance", "mask"):
            assert np.array_equal(a[key], b[key]), (i, key)
        assert int(r_ours["status"]) == int(r_ref["status"]) and r_ours["num_inliers"] == r_ref["num_inliers"]
    out = {"workload": "16 mixed-resolution pairs (640x480 .. 3840x2160), single level, K in {500, 2000, 8000}, "
                       "FAST in {10, 20, 40}, R in {500, 2000, 8000}; plain forms synchronise per pair",
           "mean_mpx_per_pair": sum(p.gray_a.size + p.gray_b.size for p in pairs) / 16 / 1e6}
    for name, runner in (("ours_plain", ours), ("reference_stock", stock)):
        timed(runner, pairs[:2], knobs[:2])  # warm-up
        out[name] = timed(runner, pairs, knobs)
    imgs = [(torch.from_numpy(p.gray_a).cuda(), torch.from_numpy(p.gray_b).cuda()) for p in pairs]
    bt = batch.Batch([batch.pair_desc(a, b, k) for (a, b), k in zip(imgs, knobs)])
    bt.capture()
    stream = torch.cuda.current_stream()
    for _ in range(3):
        bt.launch(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(5):
        bt.launch(stream)
    e1.record(stream)
    e1.synchronize()
    out["ours_batched"] = {"pairs_per_s": 16 * 5 / (e0.elapsed_time(e1) / 1e3)}
    for i in small:
        np.testing.assert_array_equal(bt.result(i)["H"], ours.run(pairs[i].gray_a, pairs[i].gray_b, knobs[i])["H"])
    out["batched_over_reference"] = out["ours_batched"]["pairs_per_s"] / out["reference_stock"]["pairs_per_s"]
    out["plain_over_reference"] = out["ours_plain"]["pairs_per_s"] / out["reference_stock"]["pairs_per_s"]
    print("\nREFERENCE_MIXED " + json.dumps(out))

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

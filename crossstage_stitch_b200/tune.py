"""Autotuner of the batched form's launch shapes, per resolution bucket.

A batch of uneven pairs is split into sub-batches by (resolution bucket, K
class) of its pairs: buckets VGA, 720p, 1080p and 4K by the larger image's
pixel count, K classes by the keypoint budget. Each sub-batch is a plan of
its own with its own launch shapes (stitch_batch_tuning: the persistent FAST
and blur grids, the S4 matcher, MSAC hypotheses per warp and the resize tile
height), captured as its own CUDA graph; BucketedBatch replays the graphs on
a few streams so that the buckets' kernels overlap. Results never depend on
the shapes: every plan equals the per-pair stages bit for bit.

Tuner picks a bucket's shapes by coordinate descent from the defaults, one
field at a time over its candidate values, timing the sub-batch's graph with
CUDA events on the device (median of a few replays), and caches the choice
in a JSON file keyed by (GPU name, bucket, K class): the STITCH_TUNE_CACHE
path, else ~/.cache/crossstage_stitch_b200/tuning.json.
"""
from __future__ import annotations

import json
import os
import statistics
from pathlib import Path

import torch

from . import batch
from .stages import Knobs

BUCKETS = (("vga", 640 * 480), ("720p", 1280 * 720), ("1080p", 1920 * 1080), ("4k", 3840 * 2160))
K_CLASSES = (("k500", 1000), ("k2000", 4000), ("k8000", 1 << 30))
# candidate values of each tuning field, the default first
SPACE = {
    "fast_ctas_per_sm": (7, 6, 4),
    "resize_tile_h": (64, 32, 16),
    "blur_ctas_per_sm": (6, 4),
    "matcher": (2, 5),          # 1 + matcher kind: tensor cores, pipelined tensor cores
    "search_hpw": (0, 8, 32),   # 0: chosen from the batch size
}


def bucket_of(w_a: int, h_a: int, w_b: int, h_b: int) -> str:
    """The bucket whose reference size is nearest (in log area) to the larger image."""
    import math
    area = max(w_a * h_a, w_b * h_b)
    return min(BUCKETS, key=lambda b: abs(math.log(area / b[1])))[0]


def k_class(k: int) -> str:
    return next(name for name, top in K_CLASSES if k <= top)


def group_key(img_a: torch.Tensor, img_b: torch.Tensor, knobs: Knobs) -> tuple[str, str]:
    return bucket_of(img_a.shape[1], img_a.shape[0], img_b.shape[1], img_b.shape[0]), k_class(knobs.max_keypoints)


def default_cache() -> Path:
    env = os.environ.get("STITCH_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "crossstage_stitch_b200" / "tuning.json"


class Tuner:
    """Launch shapes per (GPU, bucket, K class), measured and cached."""

    def __init__(self, cache: Path | str | None = None, device=None, reps: int = 3):
        self.path = Path(cache) if cache else default_cache()
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.gpu = torch.cuda.get_device_name(self.device)
        self.reps = reps
        self.table = json.loads(self.path.read_text()) if self.path.exists() else {}
        self.log: dict[str, dict] = {}   # key -> {"default_ms", "tuned_ms", "tuning"} of this process's runs

    def key(self, group: tuple[str, str]) -> str:
        return f"{self.gpu}|{group[0]}|{group[1]}"

    def time_plan(self, pairs, tuning: dict) -> float:
        """Median device ms of a replay of the sub-batch's graph."""
        b = batch.Batch([batch.pair_desc(a, bb, k) for a, bb, k in pairs], device=self.device, tuning=tuning)
        b.capture()
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        times = []
        for it in range(self.reps + 1):
            e0.record(stream)
            b.launch(stream)
            e1.record(stream)
            e1.synchronize()
            if it:
                times.append(e0.elapsed_time(e1))
        del b
        return statistics.median(times)

    def tune(self, group: tuple[str, str], pairs) -> dict:
        """The group's shapes: cached, else found by coordinate descent."""
        key = self.key(group)
        if key in self.table:
            return dict(self.table[key]["tuning"])
        best = {f: vals[0] for f, vals in SPACE.items()}
        default_ms = best_ms = self.time_plan(pairs, best)
        for field, vals in SPACE.items():
            for v in vals[1:]:
                trial = dict(best, **{field: v})
                ms = self.time_plan(pairs, trial)
                if ms < best_ms:
                    best, best_ms = trial, ms
        self.table[key] = {"tuning": best, "default_ms": default_ms, "tuned_ms": best_ms, "pairs": len(pairs)}
        self.log[key] = self.table[key]
        self.path.parent.mkdir(parents=True, exist_ok=True)
        self.path.write_text(json.dumps(self.table, indent=1, sort_keys=True))
        return dict(best)


class BucketedBatch:
    """One tuned plan and graph per (bucket, K class) of the pairs; launch()
    replays them on `streams` streams forked from and joined to the caller's
    stream. result(i) is pair i's result in the caller's order."""

    def __init__(self, pairs, tuner: Tuner | None = None, device=None, streams: int = 4):
        """pairs: (device image a, device image b, Knobs) in the caller's order."""
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        groups: dict[tuple[str, str], list[int]] = {}
        for i, (a, b, k) in enumerate(pairs):
            groups.setdefault(group_key(a, b, k), []).append(i)
        # largest groups first: they start first on the streams
        self.groups = sorted(groups.items(), key=lambda g: -sum(pairs[i][0].numel() for i in g[1]))
        self.where = {}
        self.batches, self.tunings = [], {}
        for gi, (g, idx) in enumerate(self.groups):
            sub = [pairs[i] for i in idx]
            tuning = tuner.tune(g, sub) if tuner else None
            self.tunings[f"{g[0]}|{g[1]}"] = tuning
            b = batch.Batch([batch.pair_desc(a, bb, k) for a, bb, k in sub], device=self.device, tuning=tuning)
            b.capture()
            self.batches.append(b)
            for li, i in enumerate(idx):
                self.where[i] = (gi, li)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, min(streams, len(self.batches))))]
        self.done = [torch.cuda.Event() for _ in self.streams]

    def launch(self, stream=None) -> None:
        s = stream if stream is not None else torch.cuda.current_stream()
        start = torch.cuda.Event()
        start.record(s)
        for st in self.streams:
            st.wait_event(start)
        for gi, b in enumerate(self.batches):
            b.launch(self.streams[gi % len(self.streams)])
        for st, d in zip(self.streams, self.done):
            d.record(st)
            s.wait_event(d)

    def result(self, i: int) -> dict:
        gi, li = self.where[i]
        return self.batches[gi].result(li)

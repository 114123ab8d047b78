"""Registration throughput benchmark: pairs/s and per-pair latency, batched
form vs the plain per-pair form, on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 64 synthetic 512x512 pairs, the batched-registration
configuration. Each pair is built from blobs, rectangles and band-limited
noise, then warped by a random homography. Knobs: K = 2000 keypoints per
image, FAST 20, ratio 0.8, R = 2000, tau = 3 px, 1 refinement, ORB on an
8-level pyramid at scale 1.2. One step registers all 64 pairs. The inputs
fit in L2, so a 512 MB buffer is written between timed steps to flush it
(outside the timed span).

- value: the batched form. One captured CUDA graph runs every stage for
  all 64 pairs, with the images resident in HBM. It is device-timed with
  CUDA events, and the max over ranks is taken.
- e2e: the same graph through the public API. Every step copies the 128
  images from pinned host memory and reads the 64 results back.
- plain_per_pair: the drop-in stages called pair by pair on one stream,
  with a sync per pair, as the reference harness does.
- roofline: the dominant kernel, timed from event marks recorded between
  the batched kernels inside the timed region.
- cpu_baseline: the CPU oracle chain (NumPy S2/S3 + C S4/S5) on the host
  cores.

With N GPUs each rank registers its own 64 pairs. Pairs are independent,
so this is replicas with weak scaling and no collective on the data path.

--impl reference times the reference's CPU path, restated as that oracle
chain, on the host cores, over a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_PAIRS = 64
SIZE = 512
K = 2000
R = 2000
LEVELS = 8
SCALE = 1.2
WORKLOAD = ("batched registration, 64 pairs 512x512 u8, K=2000, FAST 20, 8-level pyramid at 1.2, ratio 0.8, "
            "R=2000, tau 3 px")
PEAKS = ROOT / "MEASURED_PEAKS.json"


def knobs_for(i):
    from crossstage_stitch_b200 import stages, synth
    return stages.Knobs(max_keypoints=K, hypotheses=R, seed=synth.BASE_SEED + i, threshold=3.0, levels=LEVELS,
                        scale_factor=SCALE)


def layer_pixels(w, h):
    """Pixels of each pyramid layer (sizes cvRound(W / s_l) in float32)."""
    import numpy as np
    sf = float(np.float32(SCALE))
    out = []
    for l in range(LEVELS):
        inv = np.float32(1.0) / np.float32(sf ** l)
        lw, lh = int(np.rint(np.float32(w) * inv)), int(np.rint(np.float32(h) * inv))
        if lw <= 62 or lh <= 62:
            break
        out.append(lw * lh)
    return out


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.path = Path(f"/tmp/stitch_clocks_{os.getpid()}.csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "10"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        # the timed region starts only once the sampler is producing rows
        t0 = time.time()
        while self.proc is not None and self.proc.poll() is None and time.time() - t0 < 5.0:
            if self.path.exists() and self.path.stat().st_size > 0:
                break
            time.sleep(0.01)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = [r.split(",") for r in self.path.read_text().splitlines() if r.strip()]
        rows = [r for r in rows if len(r) > 8]
        sm = [float(r[1]) for r in rows]
        mx = [float(r[2]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def cpu_pair(args):
    """One pair through the CPU oracle chain (runs in a spawned worker)."""
    i, rank = args
    sys.path.insert(0, str(ROOT))
    from crossstage_stitch_b200 import synth
    from oracle import chain
    p = synth.config0_pair(rank * N_PAIRS + i)
    t = time.perf_counter()
    chain.run_pair(p.gray_a, p.gray_b, knobs_for(rank * N_PAIRS + i))
    return time.perf_counter() - t


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline(sample_pairs: int, workers: int, one_core_pairs: int = 4) -> dict:
    """The oracle chain on `workers` processes (all cores) and on one."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        pool.map(cpu_pair, [(0, 0)] * workers)  # warm the workers (imports)
        t = time.perf_counter()
        lat = pool.map(cpu_pair, [(i % N_PAIRS, 0) for i in range(sample_pairs)])
        wall = time.perf_counter() - t
    with ctx.Pool(1) as pool:
        pool.map(cpu_pair, [(0, 0)])
        t = time.perf_counter()
        lat1 = pool.map(cpu_pair, [(i % N_PAIRS, 0) for i in range(one_core_pairs)])
        wall1 = time.perf_counter() - t
    lat, lat1 = sorted(lat), sorted(lat1)
    return {"value": sample_pairs / wall, "unit": "pairs/s", "cores": workers, "kind": "port",
            "cpu_model": cpu_model(), "nproc": os.cpu_count(),
            "sample": f"{sample_pairs} pairs of the workload on {workers} processes "
                      f"(NumPy S2/S3 + C S4/S5 restatement of the reference)",
            "p50_ms": 1e3 * lat[len(lat) // 2], "p99_ms": 1e3 * lat[int(0.99 * (len(lat) - 1))],
            "one_core": {"value": one_core_pairs / wall1, "unit": "pairs/s", "cores": 1,
                         "sample": f"{one_core_pairs} pairs of the workload on one process",
                         "p50_ms": 1e3 * lat1[len(lat1) // 2], "p99_ms": 1e3 * lat1[-1]}}


def opencv_pair(i):
    """One pair through OpenCV on one thread: ORB (K features, 8 levels at
    1.2, FAST 20, Harris score, 31 px patches), brute-force Hamming kNN-2
    with ratio 0.8, RANSAC findHomography (3 px, 2000 iterations, confidence
    0.995). This is the product-like CPU chain of the reference's mock stages
    (tools/mock/stages.py:58-114) at this workload's knobs; its results are
    not the reference's."""
    import cv2
    import numpy as np
    from crossstage_stitch_b200 import synth
    cv2.setNumThreads(1)
    p = synth.config0_pair(i)
    t = time.perf_counter()
    orb = cv2.ORB_create(nfeatures=K, scaleFactor=SCALE, nlevels=LEVELS, edgeThreshold=31, fastThreshold=20,
                         scoreType=cv2.ORB_HARRIS_SCORE, patchSize=31)
    ka, da = orb.detectAndCompute(p.gray_a, None)
    kb, db = orb.detectAndCompute(p.gray_b, None)
    if da is not None and db is not None and len(ka) >= 2 and len(kb) >= 2:
        good = [m for m in cv2.BFMatcher(cv2.NORM_HAMMING).knnMatch(da, db, k=2)
                if len(m) == 2 and m[0].distance < 0.8 * m[1].distance]
        if len(good) >= 4:
            src = np.float64([kb[m[0].trainIdx].pt for m in good])
            dst = np.float64([ka[m[0].queryIdx].pt for m in good])
            cv2.setRNGSeed(i)
            cv2.findHomography(src, dst, cv2.RANSAC, 3.0, maxIters=2000, confidence=0.995)
    return time.perf_counter() - t


def opencv_baseline(n_pairs: int, workers: int) -> dict:
    """The OpenCV chain on 1 core and on `workers` processes (spawned pool)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = {"workload": f"{n_pairs} pairs of the workload, OpenCV ORB + BFMatcher + RANSAC findHomography",
           "unit": "pairs/s", "cores": workers}
    for n in (1, workers):
        with ctx.Pool(n) as pool:
            pool.map(opencv_pair, range(n))  # imports
            t = time.perf_counter()
            lat = sorted(pool.map(opencv_pair, range(n_pairs)))
            wall = time.perf_counter() - t
        key = "one_core" if n == 1 else "all_cores"
        out[key] = n_pairs / wall
        out[key + "_p50_ms"] = 1e3 * lat[len(lat) // 2]
        out[key + "_p99_ms"] = 1e3 * lat[int(0.99 * (len(lat) - 1))]
    return out


REF_STAGES = ("s2_workspace_bytes", "s2_detect", "s3_workspace_bytes", "s3_describe", "s4_workspace_bytes",
              "s4_match", "s5_workspace_bytes", "s5_estimate")


def reference_gpu_per_pair(pairs: int = N_PAIRS, reps: int = 3) -> dict:
    """The reference's own S2-S5 stage sources, built for sm_100a with the
    reference's flags (oracle/_ref/libref_stages_stock.so), driven pair by
    pair as its harness does (S2 A, S2 B, S3 A, S3 B, S4, S5 on one stream,
    one synchronisation per pair; harness/pipeline_runner.cu:335-416) on the
    workload's pairs and knobs, single level (the reference has no
    pyramid). Wall time per pair, uploads excluded."""
    import ctypes as C
    import torch
    from crossstage_stitch_b200 import _abi, stages, synth
    path = ROOT / "oracle" / "_ref" / "libref_stages_stock.so"
    if not path.exists():
        return {"unavailable": "the reference's stage build (oracle/_ref/libref_stages_stock.so) is not present"}
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}

    class RefStages:
        def __init__(self):
            self.L = C.CDLL(str(path))
            for name in REF_STAGES:
                fn = getattr(self.L, "ref_" + name)
                fn.restype = C.c_int
                fn.argtypes = _abi.PROTOTYPES["stitch_" + name][1]
                setattr(self, "stitch_" + name, fn)

    torch.cuda.set_device(0)
    knobs = [stages.Knobs(max_keypoints=K, hypotheses=R, seed=synth.BASE_SEED + i, threshold=3.0)
             for i in range(pairs)]
    ps = [synth.config0_pair(i) for i in range(pairs)]
    runner = stages.PairRunner(SIZE, SIZE, K, max_r=R, stage_lib=RefStages())
    stream = torch.cuda.current_stream()
    lat = []
    for rep in range(reps + 1):
        for i, p in enumerate(ps):
            runner.upload(p.gray_a, p.gray_b)
            torch.cuda.synchronize()
            t = time.perf_counter()
            runner.enqueue(SIZE, SIZE, SIZE, SIZE, knobs[i])
            stream.synchronize()
            if rep:
                lat.append(time.perf_counter() - t)
    lat.sort()
    return {"value": len(lat) / sum(lat), "unit": "pairs/s", "build": "reference sources, reference flags, sm_100a",
            "workload": f"{pairs} pairs of the workload, single level, K={K}, FAST 20, R={R}, one "
                        f"synchronisation per pair, {reps} passes",
            "p50_ms": 1e3 * lat[len(lat) // 2], "p99_ms": 1e3 * lat[int(0.99 * (len(lat) - 1))]}


def run_reference(args):
    """The reference arm: the oracle chain on every host core, one pool for
    the whole run; a step registers the workload's 64 pairs, spread over the
    worker processes. The line also carries the reference's own GPU kernels
    per pair (reference_gpu_per_pair), measured after the timed CPU steps."""
    import multiprocessing as mp
    workers = min(os.cpu_count() or 1, 32)
    ctx = mp.get_context("spawn")
    times, lat = [], []
    with ctx.Pool(workers) as pool:
        pool.map(cpu_pair, [(0, 0)] * workers)  # warm the workers (imports)
        t = time.perf_counter()
        pool.map(cpu_pair, [(i, 0) for i in range(workers)], chunksize=1)
        rate = workers / (time.perf_counter() - t)
        # a step is the workload's 64 pairs, or its first `per_step` pairs
        # when 64 would take the whole run past REFERENCE_SECONDS
        per_step = min(N_PAIRS, max(workers, int(rate * REFERENCE_SECONDS / max(1, args.steps + args.warmup))))
        for _ in range(args.warmup):
            pool.map(cpu_pair, [(i, 0) for i in range(per_step)], chunksize=1)
        for _ in range(args.steps):
            t = time.perf_counter()
            lat += pool.map(cpu_pair, [(i, 0) for i in range(per_step)], chunksize=1)
            times.append(time.perf_counter() - t)
    v = per_step * args.steps / sum(times)
    lat.sort()
    sample = (f"{args.steps} steps of {per_step} of the workload's {N_PAIRS} pairs on {workers} processes "
              f"(NumPy S2/S3 + C S4/S5 restatement of the reference)")
    try:
        gpu = reference_gpu_per_pair()
    except Exception as e:  # the reference's GPU build is reported, never required
        gpu = {"unavailable": f"{type(e).__name__}: {e}"}
    line = {"impl": "reference", "metric": "pairs/s", "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/i32/f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "pairs_per_step": per_step},
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": workers, "kind": "port", "sample": sample,
                             "cpu_model": cpu_model(), "nproc": os.cpu_count(),
                             "p50_ms": 1e3 * lat[len(lat) // 2], "p99_ms": 1e3 * lat[int(0.99 * (len(lat) - 1))]},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_gpu_per_pair": gpu}
    print(json.dumps(line), flush=True)


# DRAM bytes (read + write) per launch of a kernel of the batched step, from
# one ncu capture of this workload (dram__bytes_read.sum + dram__bytes_write.sum).
NCU_TRAFFIC = {
    "fast_nms": (110.70e6, "ncu capture of this workload (fast_kernel, one launch)"),
    "blur": (192.09e6, "ncu capture of this workload (blur_tiles_kernel, one launch)"),
    "describe": (171.16e6, "ncu capture of this workload (describe_kernel, one launch)"),
    "search": (13.09e6, "ncu capture of this workload (scoring kernel)"),
}

N_MIXED = 256
REFERENCE_SECONDS = 150.0   # bound on the reference arm's CPU steps (warm-up and timed)
SERVED_RATES = (200, 500, 1000, 2000)
SERVED_SECONDS = 60.0       # per rate, served form
PLAIN_SERVED_SECONDS = 10.0  # per rate, the plain per-pair comparison on the start of the same trace
DEADLINE_MS = 25.0           # the latency target at 1000 pairs/s


def mixed_pair_job(i):
    """One pair of the mixed-resolution workload (runs in a spawned worker)."""
    sys.path.insert(0, str(ROOT))
    from crossstage_stitch_b200 import synth
    p, kn = synth.mixed_pair(i)
    return p.gray_a, p.gray_b, kn


def make_mixed(n: int, workers: int):
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(mixed_pair_job, range(n), chunksize=1)


def mixed_knobs(kn, seed):
    from crossstage_stitch_b200 import stages
    return stages.Knobs(max_keypoints=kn["max_keypoints"], fast_threshold=kn["fast_threshold"],
                        hypotheses=kn["hypotheses"], seed=seed, levels=LEVELS, scale_factor=SCALE)


def run_mixed(mixed, steps, warmup, dev, flush):
    """Mixed-resolution workload: the batched graph over all pairs vs the plain
    per-pair stages, same pairs and knobs, images resident on the device."""
    import torch
    from crossstage_stitch_b200 import batch, stages, synth
    knobs = [mixed_knobs(kn, synth.BASE_SEED + 100000 + i) for i, (_, _, kn) in enumerate(mixed)]
    imgs = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _ in mixed]
    b = batch.Batch([batch.pair_desc(ia, ib, k) for (ia, ib), k in zip(imgs, knobs)], device=dev)
    b.capture()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for it in range(warmup + steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0.record(stream)
        b.launch(stream)
        e1.record(stream)
        e1.synchronize()
        if it >= warmup:
            times.append(e0.elapsed_time(e1))
    t_batch = sum(times) / len(times)
    # per-kernel split from a copy of the graph with event marks (own workspace)
    from crossstage_stitch_b200 import _abi
    bm = batch.Batch([batch.pair_desc(ia, ib, k) for (ia, ib), k in zip(imgs, knobs)], device=dev)
    marks = [torch.cuda.Event(enable_timing=True) for _ in _abi.BATCH_MARKS]
    bm.set_marks(marks)
    bm.capture()
    split = [0.0] * len(marks)
    for it in range(warmup + steps):
        flush.zero_()
        torch.cuda.synchronize()
        bm.launch(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            for i in range(1, len(marks)):
                split[i] += marks[i - 1].elapsed_time(marks[i]) / steps
    del bm
    kernel_ms = {_abi.BATCH_MARKS[i]: round(split[i], 4) for i in range(1, len(marks))}
    # the autotuned form: one tuned plan and graph per (resolution bucket, K
    # class), replayed on four streams; the tuner's cache is fresh per run
    import tempfile
    from crossstage_stitch_b200 import tune
    tuner = tune.Tuner(Path(tempfile.gettempdir()) / f"stitch_tuning_{os.getpid()}.json", device=dev)
    t_tune = time.perf_counter()
    bb = tune.BucketedBatch([(ia, ib, k) for (ia, ib), k in zip(imgs, knobs)], tuner=tuner, device=dev)
    tune_s = time.perf_counter() - t_tune
    times_b = []
    for it in range(warmup + steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0.record(stream)
        bb.launch(stream)
        e1.record(stream)
        e1.synchronize()
        if it >= warmup:
            times_b.append(e0.elapsed_time(e1))
    t_bucketed = sum(times_b) / len(times_b)
    parity_bucketed = all(same_result(bb.result(i), b.result(i)) for i in range(len(mixed)))
    buckets = {k.split("|", 1)[1]: {"pairs": v["pairs"], "tuning": v["tuning"], "default_ms": round(v["default_ms"], 3),
                                    "tuned_ms": round(v["tuned_ms"], 3)} for k, v in tuner.log.items()}
    del bb
    W = max(max(a.shape[1], bb.shape[1]) for a, bb, _ in mixed)
    H = max(max(a.shape[0], bb.shape[0]) for a, bb, _ in mixed)
    runner = stages.PairRunner(W, H, max(k.max_keypoints for k in knobs), max_r=max(k.hypotheses for k in knobs),
                               device=dev)
    lat, plain_results = [], []

    def plain(record):
        for (ia, ib), k in zip(imgs, knobs):
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            runner.enqueue(ia.shape[1], ia.shape[0], ib.shape[1], ib.shape[0], k, stream, images=(ia, ib))
            f1.record(stream)
            stream.synchronize()
            if record:
                lat.append(f0.elapsed_time(f1))
                plain_results.append(stages.result_dict(runner.result))

    plain(False)
    torch.cuda.synchronize()
    e0.record(stream)
    plain(True)
    e1.record(stream)
    e1.synchronize()
    t_plain = e0.elapsed_time(e1)
    lat.sort()
    n = len(mixed)
    mpx = sum(a.size + bb.size for a, bb, _ in mixed) / n / 1e6
    parity = all(same_result(b.result(i), plain_results[i]) for i in range(n)) and parity_bucketed
    del b
    return {"workload": f"{n} mixed pairs from {{640x480, 1280x720, 1920x1080, 3840x2160}}, K in {{500, 2000, 8000}}, "
                        f"FAST in {{10, 20, 40}}, R in {{500, 2000, 8000}}, 8 levels at 1.2, repeated-texture outliers",
            "pairs": n, "mean_mpx_per_pair": round(mpx, 3),
            "batched": {"value": n / (t_batch / 1e3), "unit": "pairs/s", "ms_per_step": t_batch,
                        "kernel_ms": kernel_ms},
            "plain_per_pair": {"value": n / (t_plain / 1e3), "unit": "pairs/s", "p50_ms": lat[len(lat) // 2],
                               "p99_ms": lat[int(0.99 * (len(lat) - 1))]},
            "batched_over_plain": (n / (t_batch / 1e3)) / (n / (t_plain / 1e3)),
            "bucketed": {"value": n / (t_bucketed / 1e3), "unit": "pairs/s", "ms_per_step": t_bucketed,
                         "form": "one autotuned plan and CUDA graph per (resolution bucket, K class), 4 streams",
                         "tuning_seconds": round(tune_s, 2), "buckets": buckets},
            "bucketed_over_plain": (n / (t_bucketed / 1e3)) / (n / (t_plain / 1e3)), "parity": parity}


def percentile(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(q * (len(v) - 1) + 0.5))] if v else None


def same_result(got: dict, want: dict) -> bool:
    """A batched pair's result equals the plain per-pair result: status,
    match and inlier counts, and every bit of H."""
    import numpy as np
    return (int(got["status"]) == int(want["status"]) and got["num_matches"] == want["num_matches"]
            and got["num_inliers"] == want["num_inliers"]
            and np.array_equal(np.asarray(got["H"]).view(np.uint64), np.asarray(want["H"]).view(np.uint64)))


def run_served(mixed, dev, seconds: float, plain_seconds: float):
    """Open-loop Poisson arrivals of the mixed pairs (per-request seeds) at each
    rate for `seconds`: the served form (8 GB arena) against the plain
    per-pair stages serving the same trace one request at a time for
    `plain_seconds`. Latency runs from the arrival (submit, before the
    host-to-device copies) to the result on the host. A request is dropped
    when its result is not on the host within DEADLINE_MS of its arrival
    (late, or refused at submit); drop_rate = dropped / arrivals."""
    import numpy as np
    import torch
    from crossstage_stitch_b200 import stages, synth
    from crossstage_stitch_b200.server import Server, pinned_image
    pool = [(pinned_image(a), pinned_image(b), kn) for a, b, kn in mixed]
    W = max(max(a.shape[1], b.shape[1]) for a, b, _ in pool)
    H = max(max(a.shape[0], b.shape[0]) for a, b, _ in pool)
    runner = stages.PairRunner(W, H, 8000, max_r=8000, device=dev)
    dev_a = torch.empty((H, W), dtype=torch.uint8, device=dev)
    dev_b = torch.empty((H, W), dtype=torch.uint8, device=dev)
    out = []
    for rate in SERVED_RATES:
        rng = np.random.default_rng(synth.BASE_SEED + rate)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, int(rate * seconds * 1.2) + 16))
        arrivals = arrivals[arrivals < seconds]
        picks = rng.integers(0, len(pool), len(arrivals))
        # served form
        srv = Server(arena_bytes=8 << 30, max_batch=64, streams=2, device=dev.index)
        for i in range(min(8, len(pool))):          # warm-up requests, not timed
            srv.submit(pool[i][0], pool[i][1], mixed_knobs(pool[i][2], 1), tag=1 << 40 | i)
        srv.drain()
        res, refused, t0 = [], 0, time.perf_counter()
        for n, (t, p) in enumerate(zip(arrivals, picks)):
            while True:
                rem = t - (time.perf_counter() - t0)
                if rem <= 0:
                    break
                res += srv.poll()
                if rem > 5e-4:
                    time.sleep(2e-4)
            a, b, kn = pool[p]
            refused += srv.submit(a, b, mixed_knobs(kn, synth.BASE_SEED + 500000 + n), tag=n) != 0
        res += srv.drain(timeout_s=max(120.0, seconds))
        span = max(r["done_ms"] for r in res) - min(r["submit_ms"] for r in res)
        srv.close()
        lat = [r["latency_ms"] for r in res]
        late = sum(v > DEADLINE_MS for v in lat)
        # plain per-pair on the same trace (its first plain_seconds), first come first served
        plain_n = int(np.searchsorted(arrivals, plain_seconds))
        plat, t0 = [], time.perf_counter()
        for n in range(plain_n):
            t, p = arrivals[n], picks[n]
            while time.perf_counter() - t0 < t:
                pass
            a, b, kn = pool[p]
            h, w = a.shape
            hb, wb = b.shape
            dev_a[:h, :w].copy_(a, non_blocking=True)
            dev_b[:hb, :wb].copy_(b, non_blocking=True)
            runner.enqueue(w, h, wb, hb, mixed_knobs(kn, synth.BASE_SEED + 500000 + n), images=(dev_a, dev_b))
            torch.cuda.current_stream().synchronize()
            plat.append(1e3 * (time.perf_counter() - t0 - t))
        plain_span = time.perf_counter() - t0
        out.append({"offered_pairs_s": rate, "seconds": seconds, "requests": len(arrivals),
                    "completed": len(res), "refused": refused,
                    "throughput_pairs_s": len(res) / (span / 1e3), "p50_ms": percentile(lat, 0.5),
                    "p99_ms": percentile(lat, 0.99), "late": late,
                    "drop_rate": (late + refused) / max(len(arrivals), 1),
                    "mean_batch_pairs": sum(r["batch_pairs"] for r in res) / max(len(res), 1),
                    "plain_per_pair": {"seconds": plain_seconds, "requests": plain_n,
                                       "p50_ms": percentile(plat, 0.5), "p99_ms": percentile(plat, 0.99),
                                       "throughput_pairs_s": plain_n / max(plain_span, 1e-9),
                                       "drop_rate": sum(v > DEADLINE_MS for v in plat) / max(plain_n, 1)}})
    return {"arrivals": "open-loop Poisson", "hbm_budget_bytes": 8 << 30, "deadline_ms": DEADLINE_MS,
            "drop_rule": f"a request whose result is not on the host within {DEADLINE_MS} ms of its arrival "
                         f"(late, or refused at submit) is dropped",
            "request_pool": f"{len(pool)} mixed-resolution pairs, per-request S5 seeds", "rates": out}


def planted_descriptors(nq, nt, seed):
    """Uniform 256-bit rows; 30 % of queries get a planted partner at
    Binomial(256, 0.05) distance, 5 % a second one at the same distance."""
    import numpy as np
    rng = np.random.default_rng(seed)
    q = rng.integers(0, 256, (nq, 32), dtype=np.uint8)
    t = rng.integers(0, 256, (nt, 32), dtype=np.uint8)
    for qi in rng.choice(nq, size=int(0.3 * nq), replace=False):
        d = rng.binomial(256, 0.05)
        for _ in range(2 if rng.random() < 0.05 / 0.3 else 1):
            row = np.unpackbits(q[qi]).copy()
            row[rng.choice(256, size=d, replace=False)] ^= 1
            t[rng.integers(0, nt)] = np.packbits(row)
    return q, t


def run_matching(dev, reps=20):
    """Matching microbenchmark: 8192 x 8192 planted 256-bit descriptors,
    kNN-2 with ratio 0.8 (s4_match, one direction) with the __popc kernel
    and with the tcgen05 kind::i8 kernel; the forward neighbours and the
    matches of both must agree bit for bit."""
    import ctypes as C
    import torch
    from crossstage_stitch_b200 import _abi, synth
    from crossstage_stitch_b200._abi import Descriptors, Keypoints, Matches, S4Config
    L = _abi.load()
    n = 8192
    q, t = planted_descriptors(n, n, synth.BASE_SEED)
    dq, dt = torch.from_numpy(q).to(dev), torch.from_numpy(t).to(dev)
    cnt = torch.tensor([n], dtype=torch.int32, device=dev)
    kq = Keypoints(0, 0, 0, n, cnt.data_ptr())
    kt = Keypoints(0, 0, 0, n, cnt.data_ptr())
    Dq, Dt = Descriptors(0, 32, 32, dq.data_ptr()), Descriptors(0, 32, 32, dt.data_ptr())
    cfg = S4Config()
    cfg.ratio_threshold = 0.8
    nb = C.c_size_t()
    assert L.stitch_s4_workspace_bytes(n, n, C.byref(cfg), C.byref(nb)) == 0
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    ia = torch.empty(n, dtype=torch.int32, device=dev)
    ib = torch.empty(n, dtype=torch.int32, device=dev)
    dist = torch.empty(n, dtype=torch.float32, device=dev)
    mc = torch.zeros(1, dtype=torch.int32, device=dev)
    m = Matches(ia.data_ptr(), ib.data_ptr(), dist.data_ptr(), n, mc.data_ptr())
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out, got = {}, {}
    before = L.stitch_s4_matcher()
    for name, kind in (("popc", 0), ("tensor", 1), ("tensor128", 2), ("tensor64", 3), ("tensor_pipe", 4)):
        assert L.stitch_s4_set_matcher(kind) == 0
        call = lambda: L.stitch_s4_match(C.byref(kq), C.byref(Dq), C.byref(kt), C.byref(Dt), C.byref(cfg),
                                         C.byref(m), C.c_void_p(ws.data_ptr()), nb.value,
                                         C.c_void_p(stream.cuda_stream))
        for _ in range(3):
            assert call() == 0
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            call()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        k = int(mc.item())
        got[name] = (ws[:n * 24].cpu(), ia[:k].cpu(), ib[:k].cpu(), dist[:k].cpu())
        out[name] = {"ms": ms, "pairs_per_s": n * n / (ms / 1e3), "matches": k}
    L.stitch_s4_set_matcher(before)
    errors = L.stitch_s4_tc_errors()
    peaks = json.loads(PEAKS.read_text()) if PEAKS.exists() else {}
    int_peak = 148 * 64 * 1.965e9 * 3 / 1e12
    out["popc"].update(achieved=24.0 * n * n / (out["popc"]["ms"] / 1e3) / 1e12, unit="Tops/s", peak=int_peak,
                       peak_source="nominal INT32 issue rate (64 lanes x 3 ops/clk/SM)")
    t_peak = 2 * peaks.get("bf16_tflops", 1590.0)
    for name in ("tensor", "tensor128", "tensor64", "tensor_pipe"):
        out[name].update(achieved=512.0 * n * n / (out[name]["ms"] / 1e3) / 1e12, unit="Tops/s", peak=t_peak,
                         peak_source="dense int8 = 2 x measured bf16 burst")
    for v in out.values():
        v["frac"] = v["achieved"] / v["peak"]
    exact = all(torch.equal(a, b) for name in ("tensor", "tensor128", "tensor64", "tensor_pipe")
                for a, b in zip(got["popc"], got[name]))
    return {"workload": "8192 x 8192 planted 256-bit descriptors, kNN-2 + ratio 0.8 (s4_match, one direction)",
            "bit_exact": bool(exact), "tc_errors": errors,
            "chosen": min(out, key=lambda k: out[k]["ms"]), **out}


def run_render(dev, flush, reps=20):
    """S6 feather render microbenchmark: a 1920x1080 RGB pair (uniform noise)
    under a near-identity homography with a 310 px shift and mild
    perspective, onto its 2220x1145 canvas. L2 is flushed before every
    launch; each launch is timed alone with CUDA events on its stream.
    Algorithmic bytes per render: both RGB images read once (3 B/px) and the
    canvas written once (3 B RGB + 1 B mask per pixel)."""
    import numpy as np
    import torch
    from crossstage_stitch_b200 import render
    rng = np.random.default_rng(6)
    a = torch.from_numpy(rng.integers(0, 256, (1080, 1920, 3), dtype=np.uint8)).to(dev)
    b = torch.from_numpy(rng.integers(0, 256, (1080, 1920, 3), dtype=np.uint8)).to(dev)
    H = [[0.98, 0.02, 310.5], [-0.015, 1.01, 22.25], [1e-5, -2e-5, 1.0]]
    g = render.prepare_geometry(1920, 1080, 1920, 1080, H)
    out = torch.empty((g.height, g.width, 3), dtype=torch.uint8, device=dev)
    mask = torch.empty((g.height, g.width), dtype=torch.uint8, device=dev)
    stats = torch.zeros(2, dtype=torch.int64, device=dev)
    for _ in range(3):
        render.render(a, b, g, out, mask, stats)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        render.render(a, b, g, out, mask, stats)
        e1.record(stream)
    torch.cuda.synchronize()
    ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
    px = g.width * g.height
    nbytes = 2 * 3 * 1920 * 1080 + 4 * px
    peaks = json.loads(PEAKS.read_text()) if PEAKS.exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = nbytes / (ms / 1e3) / 1e9
    union, overlap = (int(v) for v in stats.cpu())
    return {"workload": "feather render, 1920x1080 RGB pair onto a 2220x1145 canvas (L2 flushed per launch)",
            "canvas": [g.width, g.height], "union_pixels": union, "overlap_pixels": overlap,
            "ms_per_render": ms, "canvas_mpix_per_s": px / (ms / 1e3) / 1e6, "panoramas_per_s": 1e3 / ms,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "bytes_per_render": nbytes,
                         "peak_source": "measured hbm_gbs" if "hbm_gbs" in peaks else "fallback"}}


def algorithmic_work(batch, n_pairs, counts):
    """Per-kernel algorithmic work of one step (bytes for pixel kernels,
    ops for matching and estimation), from the actual keypoint and match
    counts (counts: list of (n_a, n_b, n_matches))."""
    layers = layer_pixels(SIZE, SIZE)
    px = 2 * n_pairs * sum(layers)                      # every layer of both images
    resized = 2 * n_pairs * sum(layers[l - 1] + layers[l] for l in range(1, len(layers)))
    knn_pairs = sum(a * b for a, b, _ in counts)
    resid = sum(R * m for _, _, m in counts)
    return {
        "pyramid": ("hbm", 1.0 * resized, "GB/s"),       # previous layer read + layer write
        # FAST reads every layer pixel once; its sparse maxima list (8 B per
        # maximum, at most about 1 % of pixels) is left out
        "fast_nms": ("hbm", 1.0 * px, "GB/s"),
        "blur": ("hbm", 2.0 * px, "GB/s"),               # upper bound: every tile blurred (read + write)
        # descriptor pairs x 256 int8 MACs (2 ops each) on the tensor cores
        "knn": ("tensor", 512.0 * knn_pairs, "Tops/s"),
        "search": ("fp64", 25.0 * resid + 2000.0 * R * n_pairs, "TFLOP/s"),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-resolution and served sections")
    ap.add_argument("--served-seconds", type=float, default=SERVED_SECONDS,
                    help="seconds of arrivals per rate in the served section")
    ap.add_argument("--only", choices=["matching", "render", "batched"], default=None,
                    help="run only the matching microbenchmark (popc vs tensor cores), the S6 feather "
                         "render microbenchmark, or the batched step with its kernel marks, and print its JSON")
    ap.add_argument("--runs-csv", default=None,
                    help="write the timed plain per-pair runs as rows of the reference harness's runs.csv")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    if args.only == "matching":
        import torch
        torch.cuda.set_device(local)
        print(json.dumps(run_matching(torch.device("cuda", local), reps=args.steps)), flush=True)
        return
    if args.only == "render":
        import torch
        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
        print(json.dumps(run_render(dev, torch.empty(128 << 20, dtype=torch.int32, device=dev),
                                    reps=args.steps)), flush=True)
        return

    cpu = None
    if args.only == "batched":
        args.no_cpu_baseline = args.no_mixed = True
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(32, min(os.cpu_count() or 1, 32))   # spawned pool, before any CUDA work
        try:
            cpu["opencv_chain"] = opencv_baseline(N_PAIRS, min(os.cpu_count() or 1, 32))
        except ImportError as e:  # OpenCV is not part of the product
            cpu["opencv_chain"] = {"unavailable": str(e)}
    mixed = None
    if rank == 0 and world == 1 and not args.no_mixed:
        mixed = make_mixed(N_MIXED, min(os.cpu_count() or 1, 32))   # spawned pool, before any CUDA work

    import torch
    import torch.distributed as dist
    from crossstage_stitch_b200 import _abi, batch, replicas, stages, synth

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    L = _abi.load()
    mine = replicas.pair_indices(N_PAIRS, rank)  # each rank registers its own pairs (weak scaling)
    pairs = [synth.config0_pair(g) for g in mine]
    knobs = [knobs_for(g) for g in mine]
    host = [(torch.from_numpy(p.gray_a).pin_memory(), torch.from_numpy(p.gray_b).pin_memory()) for p in pairs]
    imgs = [(a.to(dev), b.to(dev)) for a, b in host]
    flush = torch.empty(128 << 20, dtype=torch.int32, device=dev)  # 512 MB, written by a vectorised fill

    # ---- batched form: one graph for all pairs
    # The timed graph carries no event marks (an event-record node between two
    # kernels costs about 5 us of graph time); a marked copy of it, on its own workspace, gives
    # the per-kernel split.
    descs = [batch.pair_desc(ia, ib, k) for (ia, ib), k in zip(imgs, knobs)]
    b = batch.Batch(descs, device=dev)
    b.capture()
    bm = batch.Batch(descs, device=dev)
    marks = [torch.cuda.Event(enable_timing=True) for _ in _abi.BATCH_MARKS]
    bm.set_marks(marks)
    bm.capture()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)

    def timed_graph(steps):
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            start.record(stream)
            b.launch(stream)
            stop.record(stream)
            stop.synchronize()
            total += start.elapsed_time(stop)
        return total

    def kernel_split(steps):
        per_kernel = [0.0] * len(marks)
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            bm.launch(stream)
            torch.cuda.synchronize()
            for i in range(1, len(marks)):
                per_kernel[i] += marks[i - 1].elapsed_time(marks[i])
        return per_kernel

    if args.only == "batched":
        for _ in range(args.warmup):
            timed_graph(1)
            kernel_split(1)
        t_b = timed_graph(args.steps)
        per_k = kernel_split(args.steps)
        (t_b,) = replicas.max_over_ranks([t_b], device=dev)
        names = list(_abi.BATCH_MARKS)
        if rank == 0:
            print(json.dumps({"workload": WORKLOAD, "pairs_per_s": N_PAIRS * args.steps * world / (t_b / 1e3),
                              "ms_per_step": t_b / args.steps,
                              "kernel_ms": {names[i]: per_k[i] / args.steps for i in range(1, len(names))}}),
                  flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- end to end through the public streaming API: every step copies its
    # 128 images from a pinned host buffer (one copy, overlapped with the
    # previous step's registration) and the host reads the step's results;
    # L2 is flushed on the compute stream before every step's registration.
    sb = batch.StreamingBatches([(SIZE, SIZE, SIZE, SIZE)] * N_PAIRS, knobs, device=dev)
    hosts = [sb.host_buffer(), sb.host_buffer()]
    for h in hosts:
        for i, p in enumerate(pairs):
            sb.fill(h, i, p.gray_a, p.gray_b)

    step_latency_ms = []   # per step: submit of its image copy -> its results on the host

    def timed_e2e(steps, record=False):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(sb.copy_stream)
        prev = None
        t_submit = {}
        for step in range(steps):
            with torch.cuda.stream(sb.streams[sb.next]):   # the stream of the slot this step takes
                flush.zero_()
            t0 = time.perf_counter()
            slot = sb.step(hosts[step % 2])
            t_submit[slot] = t0
            if prev is not None:
                sb.wait(prev)
                _ = sb.result(prev, N_PAIRS - 1)["status"]   # the step's results on the host
                if record:
                    step_latency_ms.append(1e3 * (time.perf_counter() - t_submit[prev]))
            prev = slot
        sb.wait(prev)
        _ = sb.result(prev, N_PAIRS - 1)["status"]
        if record:
            step_latency_ms.append(1e3 * (time.perf_counter() - t_submit[prev]))
        for d in sb.done:
            sb.copy_stream.wait_event(d)
        e1.record(sb.copy_stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        timed_graph(1)
        kernel_split(1)
        timed_e2e(2)
    clocks = Clocks(local)
    l0 = L.stitch_launch_count()
    t_batch = timed_graph(args.steps)
    launches = L.stitch_launch_count() - l0
    t_e2e = timed_e2e(args.steps, record=True)
    clk = clocks.stop()
    per_kernel = kernel_split(args.steps)
    e2e_equal = all(bool((sb.result(sb.next ^ 1, i)["H"] == b.result(i)["H"]).all()) for i in range(N_PAIRS))

    # ---- plain per-pair form (drop-in stages, one pair at a time)
    runner = stages.PairRunner(SIZE, SIZE, K, max_r=R, device=dev)
    lat, plain_results = [], []

    def plain_step(record):
        for i in range(N_PAIRS):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            runner.enqueue(SIZE, SIZE, SIZE, SIZE, knobs[i], stream, images=imgs[i])
            e1.record(stream)
            stream.synchronize()
            if record:
                lat.append(e0.elapsed_time(e1))
                plain_results.append(stages.result_dict(runner.result))

    plain_step(False)
    torch.cuda.synchronize()
    start.record(stream)
    plain_step(True)
    stop.record(stream)
    stop.synchronize()
    t_plain = start.elapsed_time(stop)
    if args.runs_csv and rank == 0:
        from crossstage_stitch_b200 import runs
        with open(args.runs_csv, "w") as f:
            f.write(runs.header())
            for i, (res, ms) in enumerate(zip(plain_results, lat)):
                f.write(runs.row(runs.record_from_result(res, f"synthetic_{rank * N_PAIRS + i}", knobs[i], S=1.0,
                                                         run_id="bench", dataset="synthetic", t_e2e=ms)))
    lat.sort()
    # the timed batched step against the plain per-pair stages, every pair
    parity_config1 = all(same_result(b.result(i), plain_results[i]) for i in range(N_PAIRS))

    matching = run_matching(dev) if rank == 0 else None
    render_res = run_render(dev, flush) if rank == 0 else None
    mixed_res = served_res = None
    if mixed is not None:
        mixed_res = run_mixed(mixed, max(3, args.steps // 2), args.warmup, dev, flush)
        served_res = run_served(mixed, dev, args.served_seconds, min(PLAIN_SERVED_SECONDS, args.served_seconds))

    counts = []
    for i in range(N_PAIRS):
        o = b.outputs(i)
        counts.append((len(o["kp_a"]), len(o["kp_b"]), len(o["idx_a"])))

    t_batch, t_e2e, t_plain = replicas.max_over_ranks([t_batch, t_e2e, t_plain], device=dev)
    pairs_total = N_PAIRS * args.steps * world
    if rank == 0:
        names = _abi.BATCH_MARKS
        kern = {names[i]: per_kernel[i] / args.steps for i in range(1, len(names))}
        ksum = sum(kern.values())
        work = algorithmic_work(b, N_PAIRS, counts)
        # the roofline object is the largest HBM- or tensor-bound kernel; the
        # FP64-bound MSAC scoring kernel is reported beside it (roofline_fp64)
        dominant = max((k for k in kern if k in work and work[k][0] in ("hbm", "tensor")), key=kern.get)
        peaks = json.loads(PEAKS.read_text()) if PEAKS.exists() else {}
        roof = None
        if dominant in work:
            bound, amount, unit = work[dominant]
            achieved = amount / (kern[dominant] / 1e3) / (1e9 if unit == "GB/s" else 1e12)
            if bound == "hbm":
                peak, src = peaks.get("hbm_gbs", 6650.0), ("measured" if "hbm_gbs" in peaks else "fallback")
            elif bound == "tensor":
                peak, src = 2 * peaks.get("bf16_tflops", 1590.0), "dense int8 = 2 x measured bf16 burst"
            elif bound == "fp64":
                peak, src = 37.0, "nominal B200 FP64 (no measured FP64 peak on this pool)"
            else:
                peak, src = 148 * 64 * 1.965e9 * 3 / 1e12, "nominal INT32 issue rate (64 lanes x 3 ops/clk/SM)"
            roof = {"kernel": dominant, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                    "frac": achieved / peak, "peak_source": src,
                    "traffic": NCU_TRAFFIC.get(dominant, (None, None))[0],
                    "traffic_source": NCU_TRAFFIC.get(dominant, (None, None))[1],
                    "ms_per_launch": kern[dominant]}
            if dominant == "fast_nms":
                roof["note"] = ("ALU-issue bound: about 68 thread-instructions per layer pixel (ncu), so its HBM "
                                "fraction is set by the instruction count, not by wasted traffic")
        roof_fp64 = None
        if "search" in kern and "search" in work:
            amount = work["search"][1]
            ach = amount / (kern["search"] / 1e3) / 1e12
            roof_fp64 = {"kernel": "search", "bound": "fp64", "achieved": ach, "peak": 37.0, "unit": "TFLOP/s",
                         "frac": ach / 37.0, "ms_per_launch": kern["search"],
                         "peak_source": "nominal B200 FP64 (no measured FP64 peak on this pool)"}
        line = {"metric": "pairs/s", "value": pairs_total / (t_batch / 1e3), "unit": "pairs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_batch / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/i32/f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "form": "batched (CUDA graph, 1 launch per stage kernel)",
                           "pairs_per_step": N_PAIRS, "pyramid_levels": LEVELS, "scale_factor": SCALE,
                           "l2": "512 MB flush between steps (inputs 33.5 MB < L2)",
                           "parallelism": f"replicas x{world}"},
                "latency": {"unit": "ms", "p50": percentile(step_latency_ms, 0.5),
                            "p99": percentile(step_latency_ms, 0.99), "steps": len(step_latency_ms),
                            "what": "per step of 64 pairs through the streaming API: host submit of the "
                                    "step's image copy to its results on the host (every pair of a step "
                                    "completes with it)"},
                "parity": {"config1": parity_config1,
                           "mixed": None if mixed_res is None else mixed_res.pop("parity"),
                           "what": "batched results equal the plain per-pair stages for every pair of the "
                                   "timed workloads (status, match and inlier counts, H bit for bit)"},
                "e2e": {"value": pairs_total / (t_e2e / 1e3), "unit": "pairs/s",
                        "h2d_bytes_per_step": N_PAIRS * 2 * SIZE * SIZE,
                        "d2h_bytes_per_step": N_PAIRS * 184,
                        "api": "batch.StreamingBatches (one pinned-host copy per step, overlapped with the "
                               "previous step; results read on the host every step)",
                        "results_equal_batched": e2e_equal},
                "plain_per_pair": {"value": N_PAIRS / (t_plain / 1e3), "unit": "pairs/s",
                                   "p50_ms": lat[len(lat) // 2], "p99_ms": lat[int(0.99 * (len(lat) - 1))]},
                "batched_over_plain": (pairs_total / (t_batch / 1e3)) / (N_PAIRS / (t_plain / 1e3)),
                "kernel_ms": {k: round(v, 5) for k, v in kern.items()}, "kernel_ms_sum": ksum,
                "kernel_ms_source": "a copy of the graph with an event mark after every kernel group",
                "keypoints_mean": statistics.mean(a + b_ for a, b_, _ in counts) / 2,
                "matches_mean": statistics.mean(m for _, _, m in counts),
                "gpu_launches": launches, "clocks": clk, "roofline": roof, "roofline_fp64": roof_fp64,
                "cpu_baseline": cpu,
                "matching": matching, "render": render_res, "mixed": mixed_res, "served": served_res}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

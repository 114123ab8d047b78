"""Registration throughput benchmark: pairs/s and per-pair latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form plain|batched]

Workload: 64 synthetic 512x512 pairs (the batched-registration configuration:
blobs + rectangles + band-limited noise, warped by a random homography,
K = 2000 keypoints per image, FAST 20, ratio 0.8, R = 2000, tau = 3 px,
1 refinement). One step registers all 64 pairs. Inputs are smaller than L2,
so a 512 MB buffer is written between timed steps to flush it.

`value` is device time with the images already in HBM (CUDA events on the
launching stream, max over ranks); `e2e` is the same work through the public
API with the images copied from pinned host memory and every pair's result
read back inside the timed region. With N GPUs each rank registers its own
64 pairs (pairs are independent: replicas, weak scaling).

--impl reference times the reference's CPU path (the CPU oracle of the
chain: NumPy S2/S3 + C S4/S5) on the host cores, on a bounded sample.
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
WORKLOAD = "batched registration, 64 pairs 512x512 u8, K=2000, FAST 20, ratio 0.8, R=2000, tau 3 px"


def knobs_for(i):
    from crossstage_stitch_b200 import stages, synth
    return stages.Knobs(max_keypoints=K, hypotheses=R, seed=synth.BASE_SEED + i, threshold=3.0)


def make_pairs(rank: int):
    from crossstage_stitch_b200 import synth
    return [synth.config0_pair(rank * N_PAIRS + i) for i in range(N_PAIRS)]


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.path = Path(f"/tmp/stitch_clocks_{os.getpid()}.csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = [r.split(",") for r in self.path.read_text().splitlines() if r.strip()]
        sm = [float(r[1]) for r in rows if len(r) > 8]
        mx = [float(r[2]) for r in rows if len(r) > 8]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) > 8 for i in range(4)
                          if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def cpu_pair(args):
    """One pair through the CPU oracle chain (runs in a worker process)."""
    i, rank = args
    sys.path.insert(0, str(ROOT))
    from crossstage_stitch_b200 import synth
    from oracle import chain
    p = synth.config0_pair(rank * N_PAIRS + i)
    t = time.perf_counter()
    chain.run_pair(p.gray_a, p.gray_b, knobs_for(rank * N_PAIRS + i))
    return time.perf_counter() - t


def cpu_baseline(sample_pairs: int, workers: int) -> dict:
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        pool.map(cpu_pair, [(0, 0)] * workers)  # warm the workers (imports, oracle build)
        t = time.perf_counter()
        lat = pool.map(cpu_pair, [(i % N_PAIRS, 0) for i in range(sample_pairs)])
        wall = time.perf_counter() - t
    return {"value": sample_pairs / wall, "unit": "pairs/s", "cores": workers, "kind": "port",
            "sample": f"{sample_pairs} pairs of the workload on {workers} processes (NumPy S2/S3 + C S4/S5 oracle)",
            "p50_ms": 1e3 * statistics.median(lat), "p99_ms": 1e3 * sorted(lat)[int(0.99 * (len(lat) - 1))]}


def run_reference(args, rank, world):
    if rank != 0:
        return
    workers = min(os.cpu_count() or 1, 32)
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(workers, workers)
    for _ in range(args.steps):
        vals.append(cpu_baseline(workers, workers))
    v = statistics.median(x["value"] for x in vals)
    line = {"impl": "reference", "metric": "pairs/s", "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8/i32/f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "pyramid_levels": 1},
            "cpu_baseline": {**vals[-1], "value": v},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(32, min(os.cpu_count() or 1, 32))   # before any CUDA work (spawned pool)

    import torch
    import torch.distributed as dist
    from crossstage_stitch_b200 import _abi, stages

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    pairs = make_pairs(rank)
    runner = stages.PairRunner(SIZE, SIZE, K, max_r=R, device=dev)
    imgs = [(torch.from_numpy(p.gray_a).to(dev), torch.from_numpy(p.gray_b).to(dev)) for p in pairs]
    host = [(torch.from_numpy(p.gray_a).pin_memory(), torch.from_numpy(p.gray_b).pin_memory()) for p in pairs]
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    L = _abi.load()

    def step_resident(lat=None):
        for i in range(N_PAIRS):
            if lat is not None:
                e0 = torch.cuda.Event(enable_timing=True); e0.record(stream)
            runner.enqueue(SIZE, SIZE, SIZE, SIZE, knobs_for(rank * N_PAIRS + i), stream, images=imgs[i])
            if lat is not None:
                e1 = torch.cuda.Event(enable_timing=True); e1.record(stream)
                lat.append((e0, e1))
            stream.synchronize()  # the plain form reads every pair's result before the next

    def step_e2e():
        out = []
        for i in range(N_PAIRS):
            runner.img[0].copy_(host[i][0], non_blocking=True)
            runner.img[1].copy_(host[i][1], non_blocking=True)
            runner.enqueue(SIZE, SIZE, SIZE, SIZE, knobs_for(rank * N_PAIRS + i), stream)
            stream.synchronize()
            out.append(runner.result.num_inliers)
        return out

    def timed(fn, steps):
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        return total

    for _ in range(args.warmup):
        step_resident()
        step_e2e()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    launches0 = L.stitch_launch_count()
    t_res = timed(step_resident, args.steps)
    launches = L.stitch_launch_count() - launches0
    t_e2e = timed(step_e2e, args.steps)
    clk = clocks.stop()
    lat = []
    step_resident(lat)
    torch.cuda.synchronize()
    lat_ms = sorted(a.elapsed_time(b) for a, b in lat)
    tt = torch.tensor([t_res, t_e2e], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    t_res, t_e2e = tt.tolist()
    pairs_total = N_PAIRS * args.steps * world
    if rank == 0:
        line = {"metric": "pairs/s", "value": pairs_total / (t_res / 1e3), "unit": "pairs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_res / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/i32/f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "form": "plain per-pair", "pairs_per_step": N_PAIRS,
                           "pyramid_levels": 1, "l2": "512 MB flush between steps",
                           "parallelism": f"replicas x{world}"},
                "p50_pair_ms": lat_ms[len(lat_ms) // 2], "p99_pair_ms": lat_ms[int(0.99 * (len(lat_ms) - 1))],
                "e2e": {"value": pairs_total / (t_e2e / 1e3), "unit": "pairs/s",
                        "h2d_bytes_per_step": N_PAIRS * 2 * SIZE * SIZE,
                        "d2h_bytes_per_step": N_PAIRS * C_RESULT_BYTES},
                "gpu_launches": launches, "clocks": clk, "roofline": None, "cpu_baseline": cpu}
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


C_RESULT_BYTES = 184

if __name__ == "__main__":
    main()

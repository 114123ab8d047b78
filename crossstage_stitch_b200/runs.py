"""runs.csv rows in the reference harness's format, so the reference's
analysis tooling reads this library's per-pair results unchanged.

Columns and number formatting follow harness/main.cpp:33-77 (write_csv_header,
write_csv_row) over the fields of harness/harness_types.hpp:40-110; the
column groups are documented in docs/conventions.md:96-123. Fixed-config rows
(empty policy_id) print S with 4 decimals, times with 3, ratios with 6, H
with 17 significant digits and leave the four policy columns empty;
adaptive rows print S with 17 significant digits, times with 6, and H only
when the status is OK.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

COLUMNS = (
    "run_id,git_rev,dataset,split,pair_id,config_id,repeat_idx,is_warmup,seed,"
    "S,K,R,blend_mode,"
    "t_h2d,t_s1,t_s2,t_s3,t_s4,t_s5,t_s6,t_controller,t_d2h,t_e2e,"
    "num_kp_a,num_kp_b,num_matches,num_inliers,inlier_ratio,inlier_coverage,reproj_residual,"
    "h0,h1,h2,h3,h4,h5,h6,h7,h8,"
    "canvas_pixels,overlap_pixels,blend_mode_effective,num_levels,peak_workspace_bytes,cache_hit,"
    "status,fail_stage,policy_id,attempt_count,t_probe_gpu,t_stream_wait,probe_gradient_a,probe_gradient_b,"
    "t_probe_s1,t_probe_grad,t_probe"
).split(",")


@dataclass
class RunRecord:
    run_id: str = ""
    git_rev: str = "HEAD"
    dataset: str = "udis_d"
    split: str = "dev"
    pair_id: str = ""
    config_id: str = ""
    repeat_idx: int = 0
    is_warmup: int = 0
    seed: int = 0
    S: float = 0.5
    K: int = 1000
    R: int = 256
    blend_mode: str = "feather"
    t_h2d: float = 0.0
    t_s1: float = 0.0
    t_s2: float = 0.0
    t_s3: float = 0.0
    t_s4: float = 0.0
    t_s5: float = 0.0
    t_s6: float = 0.0
    t_controller: float = 0.0
    t_d2h: float = 0.0
    t_e2e: float = 0.0
    num_kp_a: int = 0
    num_kp_b: int = 0
    num_matches: int = 0
    num_inliers: int = 0
    inlier_ratio: float = 0.0
    inlier_coverage: float = 0.0
    reproj_residual: float = 0.0
    H: list = field(default_factory=lambda: [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0])
    canvas_pixels: int = 0
    overlap_pixels: int = 0
    blend_mode_effective: str = "feather"
    num_levels: int = 0
    peak_workspace_bytes: int = 0
    cache_hit: int = 0
    status: str = "OK"
    fail_stage: str = ""
    policy_id: str = ""
    attempt_count: int = 0
    t_probe_gpu: float = 0.0
    t_stream_wait: float = 0.0
    probe_gradient_a: float = 0.0
    probe_gradient_b: float = 0.0
    t_probe_s1: float = 0.0
    t_probe_grad: float = 0.0
    t_probe: float = 0.0


def _fixed(x: float, digits: int) -> str:
    if math.isnan(x):
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    return f"{x:.{digits}f}"


def _general(x: float, digits: int) -> str:
    if math.isnan(x):
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    return "%.*g" % (digits, x)


def header() -> str:
    return ",".join(COLUMNS) + "\n"


def row(r: RunRecord) -> str:
    fixed_cfg = r.policy_id == ""
    out = [r.run_id, r.git_rev, r.dataset, r.split, r.pair_id, r.config_id, str(r.repeat_idx),
           str(r.is_warmup), str(r.seed)]
    out.append(_fixed(r.S, 4) if fixed_cfg else _general(r.S, 17))
    out += [str(r.K), str(r.R), r.blend_mode]
    td = 3 if fixed_cfg else 6
    out += [_fixed(t, td) for t in (r.t_h2d, r.t_s1, r.t_s2, r.t_s3, r.t_s4, r.t_s5, r.t_s6, r.t_controller,
                                     r.t_d2h, r.t_e2e)]
    out += [str(r.num_kp_a), str(r.num_kp_b), str(r.num_matches), str(r.num_inliers)]
    out += [_fixed(v, 6) for v in (r.inlier_ratio, r.inlier_coverage, r.reproj_residual)]
    show_h = r.status == "OK" or fixed_cfg
    out += [_general(float(h), 17) if show_h else "" for h in r.H]
    out += [str(r.canvas_pixels), str(r.overlap_pixels), r.blend_mode_effective, str(r.num_levels),
            str(r.peak_workspace_bytes), str(int(r.cache_hit)), r.status, r.fail_stage]
    if fixed_cfg:
        out += ["", "", "", ""]
    else:
        out += [r.policy_id, str(r.attempt_count), _fixed(r.t_probe_gpu, 6), _fixed(r.t_stream_wait, 6)]
    out += [_general(r.probe_gradient_a, 17), _general(r.probe_gradient_b, 17)]
    out += [_general(t, 4) for t in (r.t_probe_s1, r.t_probe_grad, r.t_probe)]
    return ",".join(out) + "\n"


def config_id(S: float, K: int, R: int, blend: str = "feather") -> str:
    """The fixed-config id, e.g. S0.50_K1000_R256_Bfeather (docs/conventions.md:118)."""
    return f"S{S:.2f}_K{K}_R{R}_B{blend}"


STATUS_NAMES = ("OK", "INVALID_ARGUMENT", "INSUFFICIENT_WORKSPACE", "CUDA_ERROR", "NOT_ENOUGH_POINTS", "DEGENERATE")


def record_from_result(res: dict, pair_id: str, knobs, S: float = 1.0, **fields) -> RunRecord:
    """A fixed-config record from a result dict of stages.result_dict (or
    the served form's poll()) and the pair's knobs."""
    st = int(res["status"])
    r = RunRecord(pair_id=pair_id, S=S, K=knobs.max_keypoints, R=knobs.hypotheses, seed=knobs.seed,
                  config_id=config_id(S, knobs.max_keypoints, knobs.hypotheses),
                  num_matches=res.get("num_matches", 0), num_inliers=res.get("num_inliers", 0),
                  inlier_ratio=res.get("inlier_ratio", 0.0), inlier_coverage=res.get("inlier_coverage", 0.0),
                  reproj_residual=res.get("reproj_residual", 0.0),
                  status=STATUS_NAMES[st] if 0 <= st < len(STATUS_NAMES) else str(st),
                  fail_stage="" if st == 0 else "S5")
    if "H" in res:
        r.H = [float(v) for v in res["H"].ravel()]
    for k, v in fields.items():
        setattr(r, k, v)
    return r

"""runs.csv rows in the reference harness's layout (harness/main.cpp:33-77):
the header, the fixed-config row format and the adaptive row format."""
import math

import numpy as np

from crossstage_stitch_b200 import runs, stages

REFERENCE_HEADER = (
    "run_id,git_rev,dataset,split,pair_id,config_id,repeat_idx,is_warmup,seed,S,K,R,blend_mode,t_h2d,t_s1,t_s2,"
    "t_s3,t_s4,t_s5,t_s6,t_controller,t_d2h,t_e2e,num_kp_a,num_kp_b,num_matches,num_inliers,inlier_ratio,"
    "inlier_coverage,reproj_residual,h0,h1,h2,h3,h4,h5,h6,h7,h8,canvas_pixels,overlap_pixels,"
    "blend_mode_effective,num_levels,peak_workspace_bytes,cache_hit,status,fail_stage,policy_id,attempt_count,"
    "t_probe_gpu,t_stream_wait,probe_gradient_a,probe_gradient_b,t_probe_s1,t_probe_grad,t_probe\n")


def test_header():
    assert runs.header() == REFERENCE_HEADER
    assert len(runs.COLUMNS) == 56


def test_fixed_row():
    r = runs.RunRecord(run_id="r1", pair_id="p7", config_id="S0.50_K1000_R256_Bfeather", seed=42, S=0.5,
                       t_s2=1.23456, t_e2e=10.0, num_kp_a=900, num_kp_b=880, num_matches=300, num_inliers=200,
                       inlier_ratio=2 / 3, inlier_coverage=0.5, reproj_residual=float("nan"),
                       H=[1.0, 0.1, 3.0, 0.0, 1.0, 0.0, 1e-5, 0.0, 1.0], probe_gradient_a=0.25, t_probe=1.5)
    line = runs.row(r)
    f = line.rstrip("\n").split(",")
    assert len(f) == 56
    assert f[:13] == ["r1", "HEAD", "udis_d", "dev", "p7", "S0.50_K1000_R256_Bfeather", "0", "0", "42", "0.5000",
                      "1000", "256", "feather"]
    assert f[13:23] == ["0.000", "0.000", "1.235", "0.000", "0.000", "0.000", "0.000", "0.000", "0.000", "10.000"]
    assert f[23:30] == ["900", "880", "300", "200", "0.666667", "0.500000", "nan"]
    assert f[30:39] == ["1", "0.10000000000000001", "3", "0", "1", "0", "1.0000000000000001e-05", "0", "1"]
    assert f[39:47] == ["0", "0", "feather", "0", "0", "0", "OK", ""]
    assert f[47:51] == ["", "", "", ""]
    assert f[51:] == ["0.25", "0", "0", "0", "1.5"]


def test_adaptive_row_hides_h_unless_ok():
    r = runs.RunRecord(policy_id="gate", attempt_count=2, S=0.75, t_s4=0.5, t_probe_gpu=0.125,
                       status="DEGENERATE", fail_stage="S5")
    f = runs.row(r).rstrip("\n").split(",")
    assert f[9] == "0.75" and f[17] == "0.500000"
    assert f[30:39] == [""] * 9
    assert f[45:51] == ["DEGENERATE", "S5", "gate", "2", "0.125000", "0.000000"]


def test_record_from_result():
    res = {"status": stages.Status(0), "H": np.eye(3), "num_matches": 10, "num_inliers": 8, "inlier_ratio": 0.8,
           "inlier_coverage": 0.5, "reproj_residual": 0.3}
    r = runs.record_from_result(res, "p1", stages.Knobs(max_keypoints=2000, hypotheses=2000, seed=5), S=1.0,
                                t_e2e=2.5)
    assert r.config_id == "S1.00_K2000_R2000_Bfeather" and r.status == "OK" and r.t_e2e == 2.5
    assert runs.row(r).count(",") == 55
    assert math.isclose(r.inlier_ratio, 0.8)

"""The whole per-pair chain on the CPU: S2/S3 (s2s3.py, or pyramid.py when
the knobs ask for more than one level), S4 and S5 (liboracle.so). Test
infrastructure only."""
from __future__ import annotations

import numpy as np

from . import c_oracle, pyramid


def match(desc_a: np.ndarray, desc_b: np.ndarray, ratio: float, cross_check: bool):
    fwd = c_oracle.top2(desc_a, desc_b)
    rev = c_oracle.top2(desc_b, desc_a) if cross_check and desc_b.shape[0] else None
    return c_oracle.accept(fwd, rev, ratio)


def run_pair(gray_a: np.ndarray, gray_b: np.ndarray, knobs, scale=1.0) -> dict:
    """knobs: any object with the fields of stages.Knobs."""
    k = knobs.max_keypoints
    levels, factor = getattr(knobs, "levels", 1), getattr(knobs, "scale_factor", 1.2)
    ka, da = pyramid.detect_and_describe(gray_a, knobs.fast_threshold, k, levels, factor, knobs.harris_k)
    kb, db = pyramid.detect_and_describe(gray_b, knobs.fast_threshold, k, levels, factor, knobs.harris_k)
    ia, ib, dist = match(da, db, knobs.ratio, knobs.cross_check)
    nm = ia.shape[0]
    pts = np.stack([ka[ia, 0], ka[ia, 1], kb[ib, 0], kb[ib, 1]], 1).astype(np.float64) if nm else \
        np.zeros((0, 4))
    sa = c_oracle.make_scale_info(gray_a.shape[1], gray_a.shape[0], scale)
    sb = c_oracle.make_scale_info(gray_b.shape[1], gray_b.shape[0], scale)
    status_in = 0 if nm >= 4 else 4
    res, mask, _ = c_oracle.s5(pts, k, knobs.hypotheses, knobs.threshold, knobs.seed,
                               knobs.refinement_steps, sa, sb, status_in)
    res.update({"kp_a": ka, "kp_b": kb, "desc_a": da, "desc_b": db, "idx_a": ia, "idx_b": ib,
                "distance": dist, "mask": mask[:nm]})
    return res

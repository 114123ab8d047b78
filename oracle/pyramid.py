"""CPU oracle of the scale-pyramid S2/S3 (levels > 1). TEST INFRASTRUCTURE ONLY.

The reference is single-level (docs/decisions/s2-s3-orb.md:84; no pyramid in
src/s2_s3/s2.cu:1-4 or tools/s2_s3/reference.py:1-12), so this module has no
reference implementation to be pinned against: parity for levels > 1 is
unpinned. It extends the single-level oracle (s2s3.py) with OpenCV ORB's
level semantics (modules/features2d/src/orb.cpp, OpenCV 4.x):

  - layer scale   s_l = float((double) sf ** l), where sf is the scale factor
                  rounded to float32 (cv::ORB::create takes it as a float);
    layer size    (cvRound(W * (1.f / s_l)), cvRound(H * (1.f / s_l))), the
                  product and the reciprocal rounded to float32;
  - layer image   level l resized from level l-1 with INTER_LINEAR_EXACT
                  (fixed-point bilinear, restated below);
  - budgets       n_l = cvRound(d * factor**l) with factor = float(1 / sf)
                  and d = float(K (1 - factor) / (1 - float(factor**L))),
                  the last level takes K minus the rest. When the rounded
                  shares of the first L-1 levels would exceed K (only for K
                  below about 2 L), each share is clamped to what is left, so
                  the total never exceeds K (OpenCV would return more);
  - per level     the single-level S2 on the layer image with budget n_l,
                  angles on the layer image, rBRIEF on its blurred copy;
  - output        levels concatenated in order, (x, y) multiplied by s_l in
                  float32, responses unchanged, descriptors in the same order.

Layers whose width or height is at most 2 * EDGE hold no keypoint; they and
all smaller layers are not built.
"""
from __future__ import annotations

import math

import numpy as np

from . import s2s3

F32 = np.float32


def _sf(scale_factor: float) -> float:
    return float(F32(scale_factor))


def layer_scales(levels: int, scale_factor: float) -> np.ndarray:
    sf = _sf(scale_factor)
    return np.array([F32(math.pow(sf, l)) for l in range(levels)], F32)


def layer_sizes(width: int, height: int, levels: int, scale_factor: float) -> list[tuple[int, int]]:
    out = []
    for s in layer_scales(levels, scale_factor):
        inv = F32(1.0) / s
        out.append((int(np.rint(F32(width) * inv)), int(np.rint(F32(height) * inv))))
    return out


def level_budgets(k: int, levels: int, scale_factor: float) -> list[int]:
    if levels == 1:
        return [k]
    factor = F32(1.0 / _sf(scale_factor))
    d = F32(F32(k) * (F32(1.0) - factor)) / (F32(1.0) - F32(math.pow(float(factor), levels)))
    d = F32(d)
    out, used = [], 0
    for _ in range(levels - 1):
        n = min(int(np.rint(d)), k - used)
        out.append(n)
        used += n
        d = F32(d * factor)
    out.append(max(k - used, 0))
    return out


def _linear_exact_taps(src: int, dst: int) -> tuple[np.ndarray, np.ndarray]:
    """Per destination index: left source index and the 8-bit weight of the
    right neighbour. Indices left of the source (or any index when src == 1)
    take pixel 0 with weight 0; those past the last interval take pixel src-1
    with weight 0."""
    scale = 1.0 / (float(dst) / float(src))
    f = scale * (np.arange(dst, dtype=np.float64) + 0.5) - 0.5
    iv = np.floor(f)
    c1 = np.rint((f - iv) * 256.0).astype(np.int64)
    iv = iv.astype(np.int64)
    ofs = np.where(iv < 0, 0, np.where(iv >= src - 1, src - 1, iv))
    c1 = np.where((iv < 0) | (iv >= src - 1), 0, c1)
    if src == 1:
        ofs[:] = 0
        c1[:] = 0
    return ofs, c1


def resize_linear_exact(img: np.ndarray, width: int, height: int) -> np.ndarray:
    """INTER_LINEAR_EXACT for uint8: horizontal taps give values with 8
    fractional bits, vertical taps 16, rounded once: (v + 2^15) >> 16."""
    sh, sw = img.shape
    xo, xc = _linear_exact_taps(sw, width)
    yo, yc = _linear_exact_taps(sh, height)
    src = img.astype(np.int64)
    xo1 = np.minimum(xo + 1, sw - 1)
    hor = src[:, xo] * (256 - xc) + src[:, xo1] * xc          # (sh, width)
    yo1 = np.minimum(yo + 1, sh - 1)
    v = hor[yo] * (256 - yc)[:, None] + hor[yo1] * yc[:, None]  # (height, width)
    return ((v + (1 << 15)) >> 16).astype(np.uint8)


def build_layers(gray: np.ndarray, levels: int, scale_factor: float) -> list[np.ndarray]:
    """Layer images that can hold keypoints (each dimension > 2 * EDGE)."""
    h, w = gray.shape
    layers = []
    prev = gray
    for l, (lw, lh) in enumerate(layer_sizes(w, h, levels, scale_factor)):
        if lw <= 2 * s2s3.EDGE or lh <= 2 * s2s3.EDGE:
            break
        prev = prev if l == 0 else resize_linear_exact(prev, lw, lh)
        layers.append(prev)
    return layers


def detect_and_describe(gray: np.ndarray, fast_threshold: int, max_keypoints: int, levels: int,
                        scale_factor: float, harris_k: float = 0.04) -> tuple[np.ndarray, np.ndarray]:
    """(N, 3) float32 rows (x, y, response) in level-0 coordinates and (N, 32)
    uint8 descriptors, levels concatenated in order."""
    if levels <= 1:
        return s2s3.detect_and_describe(gray, fast_threshold, max_keypoints, harris_k)
    budgets = level_budgets(max_keypoints, levels, scale_factor)
    scales = layer_scales(levels, scale_factor)
    kps, descs = [], []
    for l, layer in enumerate(build_layers(gray, levels, scale_factor)):
        kp = s2s3.detect(layer, fast_threshold, budgets[l], harris_k)
        desc = s2s3.describe(layer, kp)
        kp = kp.copy()
        kp[:, 0] = kp[:, 0] * scales[l]
        kp[:, 1] = kp[:, 1] * scales[l]
        kps.append(kp)
        descs.append(desc)
    if not kps:
        return np.zeros((0, 3), F32), np.zeros((0, s2s3.DESCRIPTOR_BYTES), np.uint8)
    return np.concatenate(kps).astype(F32), np.concatenate(descs)

"""CPU oracle for S2 (FAST-9 + NMS + Harris top-K) and S3 (IC angle + rBRIEF).

TEST INFRASTRUCTURE ONLY. This module is the checker that the CUDA stages are
compared against; the product never imports it.

It restates, in NumPy, the reference's single-level ORB path:
  - FAST-9 score map ........ tools/s2_s3/reference.py:50-77, src/s2_s3/s2.cu:39-79
  - strict 3x3 NMS, 31-px edge  reference.py:80-94, s2.cu:82-106
  - 2K pre-selection by score, ties to the smaller raster index
                               reference.py:97-100,143, s2.cu:111-235
  - Harris (integer sums, float32 formula, no FMA)
                               reference.py:103-128, s2.cu:248-285
  - top-K by response, ties to the smaller raster index
                               reference.py:146, s2.cu:289-310
  - 7x7 sigma-2 float32 Gaussian, reflect-101, rows then columns
                               reference.py:152-188, src/s2_s3/s3.cu:47-73
  - intensity-centroid angle with cv::fastAtan2 in float32
                               reference.py:191-247, s3.cu:76-145
  - rBRIEF-256, byte l = pairs 8l..8l+7, bit j = pair 8l+j
                               reference.py:250-284, s3.cu:98-156

Every float32 operation is a separate NumPy float32 op, so each product and
sum is rounded on its own, which is what the CUDA code does with
__fmul_rn/__fadd_rn. Parity of this module is pinned by golden files made with
the reference's own reference.py (tests/golden/make_golden.py).
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

EDGE = 31
HALF_PATCH = 15
FAST_RADIUS = 3
HARRIS_BLOCK = 7
CANDIDATE_FACTOR = 2
DESCRIPTOR_BYTES = 32

# Bresenham circle of radius 3, clockwise from straight below: (dx, dy).
CIRCLE = np.array([(0, 3), (1, 3), (2, 2), (3, 1), (3, 0), (3, -1), (2, -2), (1, -3),
                   (0, -3), (-1, -3), (-2, -2), (-3, -1), (-3, 0), (-3, 1), (-2, 2), (-1, 3)],
                  dtype=np.int64)

_PATTERN_FILE = (Path(__file__).resolve().parents[1] / "crossstage_stitch_b200" / "csrc"
                 / "orb_pattern_31.inc")

F32 = np.float32


def pattern() -> np.ndarray:
    """(256, 4) int32 point pairs (x0, y0, x1, y1), parsed from the shared data table."""
    text = _PATTERN_FILE.read_text(encoding="utf-8")
    body = text[text.index("*/") + 2:]
    vals = [int(v) for v in body.replace("\n", " ").replace(",", " ").split()]
    arr = np.array(vals, dtype=np.int32)
    if arr.size != 1024:
        raise ValueError("pattern table must hold 1024 values")
    return arr.reshape(256, 4)


# ------------------------------------------------------------------ S2 detect

def fast_score_map(gray: np.ndarray, threshold: int) -> np.ndarray:
    """uint8 FAST-9 score: max over 16 circular 9-arcs of the arc's minimum
    contrast (centre brighter or darker), minus one; 0 when that maximum does
    not exceed the threshold or within 3 px of the border."""
    if not 1 <= threshold <= 254:
        raise ValueError("threshold must be in [1, 254]")
    h, w = gray.shape
    out = np.zeros((h, w), np.uint8)
    r = FAST_RADIUS
    if h <= 2 * r or w <= 2 * r:
        return out
    g = gray.astype(np.int32)
    centre = g[r:h - r, r:w - r]
    diff = np.stack([centre - g[r + dy:h - r + dy, r + dx:w - r + dx] for dx, dy in CIRCLE])
    ring = np.concatenate([diff, diff[:8]], axis=0)          # 24 entries: circular windows
    lo = np.minimum.reduce([ring[j:j + 16] for j in range(9)])  # min over window starting k
    hi = np.maximum.reduce([ring[j:j + 16] for j in range(9)])
    best = np.maximum(lo, -hi).max(axis=0)
    out[r:h - r, r:w - r] = np.where(best > threshold, best - 1, 0).astype(np.uint8)
    return out


def nms_maxima(scores: np.ndarray) -> np.ndarray:
    """Scores that are strictly greater than all 8 neighbours, inside [EDGE, dim-EDGE)."""
    h, w = scores.shape
    out = np.zeros_like(scores)
    if h <= 2 * EDGE or w <= 2 * EDGE:
        return out
    s = scores.astype(np.int32)
    c = s[EDGE:h - EDGE, EDGE:w - EDGE]
    keep = c > 0
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dx or dy:
                keep &= c > s[EDGE + dy:h - EDGE + dy, EDGE + dx:w - EDGE + dx]
    out[EDGE:h - EDGE, EDGE:w - EDGE] = np.where(keep, c, 0).astype(np.uint8)
    return out


def preselect(maxima: np.ndarray, count: int) -> np.ndarray:
    """Raster indices of the `count` best maxima by (score desc, index asc)."""
    flat = maxima.ravel()
    idx = np.flatnonzero(flat)
    order = np.lexsort((idx, -flat[idx].astype(np.int64)))
    return idx[order[:count]]


def harris(gray: np.ndarray, xs: np.ndarray, ys: np.ndarray, k: float) -> np.ndarray:
    """float32 Harris response over a 7x7 window of 3x3 Sobel gradients."""
    g = gray.astype(np.int64)
    a = np.zeros(xs.shape, np.int64)
    b = np.zeros_like(a)
    c = np.zeros_like(a)
    half = HARRIS_BLOCK // 2
    for i in range(HARRIS_BLOCK):
        for j in range(HARRIS_BLOCK):
            y = ys - half + i
            x = xs - half + j
            gx = 2 * (g[y, x + 1] - g[y, x - 1]) + (g[y - 1, x + 1] - g[y - 1, x - 1]) \
                + (g[y + 1, x + 1] - g[y + 1, x - 1])
            gy = 2 * (g[y + 1, x] - g[y - 1, x]) + (g[y + 1, x - 1] - g[y - 1, x - 1]) \
                + (g[y + 1, x + 1] - g[y - 1, x + 1])
            a += gx * gx
            b += gy * gy
            c += gx * gy
    unit = F32(1) / (F32(4 * HARRIS_BLOCK) * F32(255))
    scale4 = unit * unit * unit * unit
    fa, fb, fc = a.astype(F32), b.astype(F32), c.astype(F32)
    kk = F32(k)
    trace = fa + fb
    det = fa * fb - fc * fc
    penalty = (kk * trace) * trace
    return ((det - penalty) * scale4).astype(F32)


def detect(gray: np.ndarray, fast_threshold: int, max_keypoints: int,
           harris_k: float = 0.04) -> np.ndarray:
    """S2 result: float32 (N, 3) rows (x, y, response), response descending,
    ties by raster index ascending; N = min(K, number of pre-selected maxima)."""
    if gray.dtype != np.uint8 or gray.ndim != 2:
        raise ValueError("gray must be uint8 (H, W)")
    if max_keypoints < 0:
        raise ValueError("max_keypoints must be >= 0")
    w = gray.shape[1]
    maxima = nms_maxima(fast_score_map(gray, fast_threshold))
    if max_keypoints == 0 or not maxima.any():
        return np.zeros((0, 3), np.float32)
    cand = preselect(maxima, CANDIDATE_FACTOR * max_keypoints)
    xs, ys = cand % w, cand // w
    resp = harris(gray, xs, ys, harris_k)
    # Descending response; NumPy float64 view of float32 values is exact.
    order = np.lexsort((cand, -resp.astype(np.float64)))[:max_keypoints]
    return np.stack([xs[order], ys[order], resp[order]], axis=1).astype(np.float32)


# ---------------------------------------------------------------- S3 describe

def gaussian_taps(ksize: int = 7, sigma: float = 2.0) -> np.ndarray:
    """float32 taps: exp(-x^2 / (2 sigma^2)) in float64, normalised, rounded to float32."""
    half = [math.exp(-(x * x) / (2.0 * sigma * sigma)) for x in range(-(ksize // 2), 0)]
    norm = 1.0 / (2.0 * sum(half) + 1.0)
    side = [v * norm for v in half]
    return np.array(side + [norm] + side[::-1], np.float32)


TAPS = gaussian_taps()


def blur(gray: np.ndarray) -> np.ndarray:
    """uint8 7x7 Gaussian: row pass then column pass, taps accumulated from the
    leftmost (topmost) tap with separately rounded products and sums, borders
    reflected without repeating the edge pixel, round half to even, clamp."""
    h, w = gray.shape
    r = 3

    def reflect(i: np.ndarray, n: int) -> np.ndarray:
        if n == 1:
            return np.zeros_like(i)
        i = i.copy()
        while True:
            bad = (i < 0) | (i >= n)
            if not bad.any():
                return i
            i = np.where(i < 0, -i, np.where(i >= n, 2 * n - 2 - i, i))

    cols = reflect(np.arange(-r, w + r), w)
    rows_idx = reflect(np.arange(-r, h + r), h)
    src = gray.astype(np.float32)
    padded = src[:, cols]
    row = np.zeros((h, w), np.float32)
    for i in range(7):
        row = row + TAPS[i] * padded[:, i:i + w]
    rowp = row[rows_idx, :]
    col = np.zeros((h, w), np.float32)
    for i in range(7):
        col = col + TAPS[i] * rowp[i:i + h, :]
    return np.clip(np.rint(col), 0, 255).astype(np.uint8)


def patch_half_widths(half: int = HALF_PATCH) -> np.ndarray:
    """Half-width of each row of the circular orientation patch (ORB umax)."""
    u = [0] * (half + 2)
    vmax = int(math.floor(half * math.sqrt(2.0) / 2 + 1))
    vmin = int(math.ceil(half * math.sqrt(2.0) / 2))
    for v in range(vmax + 1):
        u[v] = int(np.rint(math.sqrt(float(half * half - v * v))))
    v0 = 0
    for v in range(half, vmin - 1, -1):
        while u[v0] == u[v0 + 1]:
            v0 += 1
        u[v] = v0
        v0 += 1
    return np.array(u[:half + 1], np.int32)


_DEG = F32(180.0 / math.pi)
_C1 = F32(0.9997878412794807) * _DEG
_C3 = F32(-0.3258083974640975) * _DEG
_C5 = F32(0.1555786518463281) * _DEG
_C7 = F32(-0.04432655554792128) * _DEG
_TINY = F32(np.finfo(np.float64).eps)


def fast_atan2_deg(y: np.ndarray, x: np.ndarray) -> np.ndarray:
    """cv::fastAtan2 (odd polynomial in the ratio of the smaller to the larger
    magnitude), degrees in [0, 360), every step in float32."""
    y = y.astype(F32)
    x = x.astype(F32)
    ax, ay = np.abs(x), np.abs(y)
    wide = ax >= ay
    t = np.where(wide, ay / (ax + _TINY), ax / (ay + _TINY)).astype(F32)
    t2 = t * t
    p = ((((_C7 * t2 + _C5) * t2 + _C3) * t2 + _C1) * t).astype(F32)
    a = np.where(wide, p, F32(90) - p).astype(F32)
    a = np.where(x < 0, F32(180) - a, a).astype(F32)
    a = np.where(y < 0, F32(360) - a, a).astype(F32)
    return a


def orientation(gray: np.ndarray, xs: np.ndarray, ys: np.ndarray) -> np.ndarray:
    """Intensity-centroid angle in degrees (float32), unblurred image."""
    g = gray.astype(np.int64)
    umax = patch_half_widths()
    m10 = np.zeros(xs.shape, np.int64)
    m01 = np.zeros_like(m10)
    for u in range(-HALF_PATCH, HALF_PATCH + 1):
        m10 += u * g[ys, xs + u]
    for v in range(1, HALF_PATCH + 1):
        d = int(umax[v])
        for u in range(-d, d + 1):
            up, down = g[ys + v, xs + u], g[ys - v, xs + u]
            m10 += u * (up + down)
            m01 += v * (up - down)
    return fast_atan2_deg(m01.astype(F32), m10.astype(F32))


def describe(gray: np.ndarray, keypoints: np.ndarray) -> np.ndarray:
    """S3 result: (N, 32) uint8 rBRIEF rows; all-zero rows for keypoints that
    lie closer than EDGE to a border."""
    n = keypoints.shape[0]
    out = np.zeros((n, DESCRIPTOR_BYTES), np.uint8)
    if n == 0:
        return out
    h, w = gray.shape
    xs = np.rint(keypoints[:, 0]).astype(np.int64)
    ys = np.rint(keypoints[:, 1]).astype(np.int64)
    inside = (xs >= EDGE) & (xs < w - EDGE) & (ys >= EDGE) & (ys < h - EDGE)
    if not inside.any():
        return out
    xs, ys = xs[inside], ys[inside]
    rad = orientation(gray, xs, ys) * F32(math.pi / 180.0)
    ca = np.cos(rad.astype(np.float64)).astype(F32)
    sa = np.sin(rad.astype(np.float64)).astype(F32)
    smooth = blur(gray).astype(np.int32)
    pat = pattern()

    def at(px: int, py: int) -> np.ndarray:
        fx, fy = F32(px), F32(py)
        rx = np.rint(fx * ca - fy * sa).astype(np.int64)
        ry = np.rint(fx * sa + fy * ca).astype(np.int64)
        return smooth[ys + ry, xs + rx]

    bits = np.stack([at(p[0], p[1]) < at(p[2], p[3]) for p in pat], axis=1)  # (n, 256)
    packed = np.zeros((xs.size, DESCRIPTOR_BYTES), np.uint8)
    for j in range(8):
        packed |= bits[:, j::8].astype(np.uint8) << j
    out[inside] = packed
    return out


def detect_and_describe(gray: np.ndarray, fast_threshold: int, max_keypoints: int,
                        harris_k: float = 0.04) -> tuple[np.ndarray, np.ndarray]:
    kp = detect(gray, fast_threshold, max_keypoints, harris_k)
    return kp, describe(gray, kp)

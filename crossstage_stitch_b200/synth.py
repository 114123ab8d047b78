"""Seeded synthetic image pairs with a known homography.

The recipe is the registration benchmark's own description of its inputs:
view A is a procedural grey scene (Gaussian blobs with sigma U[3, 30] px and
amplitude U[-80, 80], axis-aligned rectangles with intensity U[0, 255], and
band-limited noise of sigma 10 low-passed at 0.1 cycles/px, clipped to
[0, 255]); view B is A warped bilinearly by a random homography (rotation
U[-10, 10] degrees, scale U[0.9, 1.1], a translation that leaves 40-70 % of
the frame overlapping, perspective terms U[-1e-4, 1e-4]) plus N(0, 2) noise.
Blob and rectangle counts scale with the image area (40 and 60 at 512x512).
The mixed-resolution variant draws sizes from {640x480, 1280x720,
1920x1080, 3840x2160}, overlap U[15, 70] % and corrupts 20-70 % of the
overlap with repeated texture tiles, so many putative matches are wrong.

H maps B pixel coordinates to A pixel coordinates (the stages' convention).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

BASE_SEED = 20261203
RESOLUTIONS = ((640, 480), (1280, 720), (1920, 1080), (3840, 2160))


@dataclass
class Pair:
    gray_a: np.ndarray
    gray_b: np.ndarray
    H: np.ndarray  # B -> A
    seed: int


def _band_limited_noise(rng: np.random.Generator, h: int, w: int, sigma: float, cutoff: float) -> np.ndarray:
    white = rng.standard_normal((h, w))
    f = np.fft.rfft2(white)
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    f[(fx * fx + fy * fy) > cutoff * cutoff] = 0
    n = np.fft.irfft2(f, s=(h, w))
    sd = n.std()
    return n * (sigma / sd) if sd > 0 else n


def scene(rng: np.random.Generator, w: int, h: int) -> np.ndarray:
    area = (w * h) / (512.0 * 512.0)
    n_rect = max(1, int(round(60 * area)))
    n_blob = max(1, int(round(40 * area)))
    img = np.full((h, w), 128.0)
    for _ in range(n_rect):
        rw = int(rng.integers(8, max(9, w // 6)))
        rh = int(rng.integers(8, max(9, h // 6)))
        x0 = int(rng.integers(0, max(1, w - rw)))
        y0 = int(rng.integers(0, max(1, h - rh)))
        img[y0:y0 + rh, x0:x0 + rw] = rng.uniform(0, 255)
    yy = np.arange(h, dtype=np.float64)[:, None]
    xx = np.arange(w, dtype=np.float64)[None, :]
    for _ in range(n_blob):
        s = rng.uniform(3, 30)
        amp = rng.uniform(-80, 80)
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        r = int(4 * s)
        x0, x1 = max(0, int(cx) - r), min(w, int(cx) + r + 1)
        y0, y1 = max(0, int(cy) - r), min(h, int(cy) + r + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        g = np.exp(-((xx[:, x0:x1] - cx) ** 2 + (yy[y0:y1] - cy) ** 2) / (2 * s * s))
        img[y0:y1, x0:x1] += amp * g
    img += _band_limited_noise(rng, h, w, 10.0, 0.1)
    return np.clip(img, 0, 255)


def _translation_for_overlap(frac: float, phi: float, w: int, h: int) -> tuple[float, float]:
    c, s = abs(math.cos(phi)), abs(math.sin(phi))
    lo, hi = 0.0, float(w + h)
    for _ in range(60):
        t = 0.5 * (lo + hi)
        ov = max(0.0, 1 - t * c / w) * max(0.0, 1 - t * s / h)
        lo, hi = (t, hi) if ov > frac else (lo, t)
    t = 0.5 * (lo + hi)
    return t * math.cos(phi), t * math.sin(phi)


def random_homography(rng: np.random.Generator, w: int, h: int, overlap: tuple[float, float]) -> np.ndarray:
    theta = math.radians(rng.uniform(-10, 10))
    s = rng.uniform(0.9, 1.1)
    frac = rng.uniform(*overlap)
    tx, ty = _translation_for_overlap(frac, rng.uniform(0, 2 * math.pi), w, h)
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    rs = np.array([[s * math.cos(theta), -s * math.sin(theta), 0],
                   [s * math.sin(theta), s * math.cos(theta), 0], [0, 0, 1]])
    to_c = np.array([[1, 0, -cx], [0, 1, -cy], [0, 0, 1.0]])
    back = np.array([[1, 0, cx + tx], [0, 1, cy + ty], [0, 0, 1.0]])
    H = back @ rs @ to_c
    H[2, 0] = rng.uniform(-1e-4, 1e-4)
    H[2, 1] = rng.uniform(-1e-4, 1e-4)
    return H / H[2, 2]


def warp_bilinear(src: np.ndarray, H: np.ndarray, w: int, h: int) -> np.ndarray:
    """B(x, y) = A(H [x, y, 1]) with bilinear interpolation, 0 outside A."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    z = H[2, 0] * xx + H[2, 1] * yy + H[2, 2]
    u = (H[0, 0] * xx + H[0, 1] * yy + H[0, 2]) / z
    v = (H[1, 0] * xx + H[1, 1] * yy + H[1, 2]) / z
    sh, sw = src.shape
    inside = (u >= 0) & (v >= 0) & (u <= sw - 1) & (v <= sh - 1) & (z > 0)
    u = np.where(inside, u, 0)
    v = np.where(inside, v, 0)
    x0 = np.clip(np.floor(u).astype(np.int64), 0, sw - 1)
    y0 = np.clip(np.floor(v).astype(np.int64), 0, sh - 1)
    x1 = np.clip(x0 + 1, 0, sw - 1)
    y1 = np.clip(y0 + 1, 0, sh - 1)
    fx, fy = u - x0, v - y0
    out = (src[y0, x0] * (1 - fx) * (1 - fy) + src[y0, x1] * fx * (1 - fy) +
           src[y1, x0] * (1 - fx) * fy + src[y1, x1] * fx * fy)
    return np.where(inside, out, 0.0)


def make_pair(seed: int, w: int = 512, h: int = 512, overlap: tuple[float, float] = (0.4, 0.7),
              corrupt: tuple[float, float] | None = None) -> Pair:
    rng = np.random.default_rng(seed)
    a = scene(rng, w, h)
    H = random_homography(rng, w, h, overlap)
    b = warp_bilinear(a, H, w, h) + rng.normal(0, 2.0, (h, w))
    if corrupt is not None:
        _repeat_tiles(rng, b, rng.uniform(*corrupt))
    return Pair(np.clip(np.rint(a), 0, 255).astype(np.uint8),
                np.clip(np.rint(b), 0, 255).astype(np.uint8), H, seed)


def _repeat_tiles(rng: np.random.Generator, img: np.ndarray, frac: float) -> None:
    """Overwrites about `frac` of the image with copies of one texture tile, so
    features there match many places (repeated-structure outliers)."""
    h, w = img.shape
    t = max(16, min(h, w) // 12)
    ty, tx = int(rng.integers(0, h - t)), int(rng.integers(0, w - t))
    tile = img[ty:ty + t, tx:tx + t].copy()
    n = int(frac * (h * w) / (t * t))
    for _ in range(n):
        y, x = int(rng.integers(0, h - t)), int(rng.integers(0, w - t))
        img[y:y + t, x:x + t] = tile


def config0_pair(index: int = 0) -> Pair:
    """One 512x512 pair of the per-pair / batched registration workload."""
    return make_pair(BASE_SEED + index)


def mixed_pair(index: int) -> tuple[Pair, dict]:
    """One pair of the mixed-resolution workload and its per-pair knobs."""
    rng = np.random.default_rng(BASE_SEED + 100000 + index)
    w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
    knobs = {"max_keypoints": int(rng.choice([500, 2000, 8000])),
             "fast_threshold": int(rng.choice([10, 20, 40])),
             "hypotheses": int(rng.choice([500, 2000, 8000]))}
    return make_pair(BASE_SEED + 200000 + index, w, h, overlap=(0.15, 0.7), corrupt=(0.2, 0.7)), knobs


def corner_error(h_est: np.ndarray, h_true: np.ndarray, w: int, h: int) -> float:
    """Mean distance (px) between the four frame corners mapped by two
    homographies (the reference's corner_error, tools/mock/stages.py:167-171)."""
    c = np.array([[0, 0, 1], [w - 1, 0, 1], [0, h - 1, 1], [w - 1, h - 1, 1]], np.float64).T
    a, b = h_est @ c, h_true @ c
    return float(np.mean(np.linalg.norm(a[:2] / a[2] - b[:2] / b[2], axis=0)))


def max_corner_error(h_est: np.ndarray, h_true: np.ndarray, w: int, h: int) -> float:
    c = np.array([[0, 0, 1], [w - 1, 0, 1], [0, h - 1, 1], [w - 1, h - 1, 1]], np.float64).T
    a, b = h_est @ c, h_true @ c
    return float(np.max(np.linalg.norm(a[:2] / a[2] - b[:2] / b[2], axis=0)))

"""Generates the S6 feather golden fixtures from the reference's FP64 NumPy path.

Run here, where the reference tree is mounted:
    python tests/golden/make_s6_golden.py --reference <reference tree>

It imports tools/s6_reference/reference.py from the reference tree and renders,
in feather mode, the eight cases of the reference's own golden exporter
(tools/s6_reference/generate_fixtures.py:49-60: odd identity, negative and
fractional translations, a projective map, separated footprints, one pixel,
one column, one row, on the exporter's XOR/modular test pattern) plus five
larger cases of this file (rotation with scale, a wide projective map, B
inside A at a fractional offset, a mirrored axis swap, a 120x160 shifted
copy). Everything lands in one compressed s6_feather.npz (per case: a, b, H,
panorama, mask and the canvas width/height/origin) and s6_manifest.json with
the versions and the file's SHA-256. The GPU box never runs this script; it
only reads the committed files.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import math
import platform
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def pattern(width: int, height: int, phase: int) -> np.ndarray:
    """The reference exporter's RGB test pattern (modular ramps and an XOR)."""
    yy, xx = np.indices((height, width), dtype=np.int32)
    return np.stack([(13 * xx + 7 * yy + phase) % 256, (3 * xx + 17 * yy + 2 * phase) % 256,
                     ((9 * xx) ^ (5 * yy) ^ phase) % 256], axis=-1).astype(np.uint8)


def smooth(width: int, height: int, seed: int) -> np.ndarray:
    """A smooth deterministic RGB texture (sums of sinusoids), compresses well."""
    yy, xx = np.indices((height, width), dtype=np.float64)
    rng = np.random.default_rng(seed)
    chans = []
    for _ in range(3):
        f = rng.uniform(0.02, 0.2, 4)
        p = rng.uniform(0, 2 * math.pi, 2)
        v = np.sin(f[0] * xx + f[1] * yy + p[0]) + np.cos(f[2] * xx - f[3] * yy + p[1])
        chans.append(np.clip(np.round(127.5 + 63 * v), 0, 255))
    return np.stack(chans, axis=-1).astype(np.uint8)


def similarity(deg: float, s: float, tx: float, ty: float) -> np.ndarray:
    c, n = s * math.cos(math.radians(deg)), s * math.sin(math.radians(deg))
    return np.array([[c, -n, tx], [n, c, ty], [0, 0, 1.0]])


def cases():
    eye = np.eye(3)
    ref = [
        ("identity_odd", 13, 9, 13, 9, eye),
        ("negative_translation", 13, 9, 11, 7, np.array([[1, 0, -3], [0, 1, -2], [0, 0, 1.]])),
        ("fractional_translation", 13, 9, 11, 7, np.array([[1, 0, 0.375], [0, 1, -0.25], [0, 0, 1.]])),
        ("projective", 17, 13, 15, 11, np.array([[1.02, 0.03, -2], [-0.02, 0.98, 1], [0.001, -0.001, 1.]])),
        ("separated", 13, 9, 11, 7, np.array([[1, 0, 17], [0, 1, 2], [0, 0, 1.]])),
        ("single_pixel", 1, 1, 1, 1, eye),
        ("one_column", 1, 9, 1, 9, eye),
        ("one_row", 9, 1, 9, 1, eye),
    ]
    out = [(name, pattern(wa, ha, 11), pattern(wb, hb, 37), h) for name, wa, ha, wb, hb, h in ref]
    out.append(("rotate_scale", smooth(96, 64, 1), smooth(80, 60, 2), similarity(7.0, 0.9, 30.0, -12.0)))
    out.append(("projective_wide", smooth(128, 96, 3), smooth(120, 90, 4),
                np.array([[0.97, 0.04, 41.5], [-0.03, 1.01, 6.25], [2.0e-4, -1.5e-4, 1.0]])))
    out.append(("b_inside_a", smooth(96, 64, 5), smooth(40, 30, 6),
                np.array([[1, 0, 20.5], [0, 1, 10.25], [0, 0, 1.]])))
    out.append(("axis_swap_mirror", smooth(48, 40, 7), smooth(40, 48, 8),
                np.array([[0, -1, 60], [1, 0, -5], [0, 0, 1.]])))
    a = smooth(160, 120, 9)
    b = np.zeros_like(a)
    b[4:, 8:] = a[:-4, :-8]  # B(x, y) = A(x - 8, y - 4); H maps B to A
    out.append(("shifted_copy", a, b, np.array([[1, 0, -8], [0, 1, -4], [0, 0, 1.]])))
    return out


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", type=Path, required=True, help="the reference source tree")
    ap.add_argument("--out", type=Path, default=HERE)
    args = ap.parse_args()
    sys.path.insert(0, str(args.reference))
    from tools.s6_reference.reference import render  # noqa: E402  (reference tree)

    arrays, manifest = {}, {"numpy": np.__version__, "python": platform.python_version(),
                            "source": "tools/s6_reference/reference.py (reference tree), mode feather",
                            "cases": {}}
    for name, a, b, h in cases():
        res = render(a, b, h, "feather")
        g = res.geometry
        arrays[f"{name}.a"] = a
        arrays[f"{name}.b"] = b
        arrays[f"{name}.H"] = np.asarray(h, np.float64)
        arrays[f"{name}.panorama"] = res.panorama
        arrays[f"{name}.mask"] = res.mask
        arrays[f"{name}.canvas"] = np.array([g.width, g.height, g.origin_x, g.origin_y], np.int64)
        manifest["cases"][name] = {"a": list(a.shape), "b": list(b.shape), "canvas": [g.width, g.height],
                                   "origin": [g.origin_x, g.origin_y], "union": int(res.mask.sum())}
        print(f"{name}: canvas {g.width}x{g.height} origin ({g.origin_x}, {g.origin_y})")
    path = args.out / "s6_feather.npz"
    np.savez_compressed(path, **arrays)
    manifest["sha256"] = hashlib.sha256(path.read_bytes()).hexdigest()
    (args.out / "s6_manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()

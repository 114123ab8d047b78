"""Generates the S2/S3 golden fixtures from the reference's own NumPy path.

Run here, where the reference tree is mounted:
    python tests/golden/make_golden.py --reference <reference tree>

It imports tools/s2_s3/reference.py and tools/s2_s3/fixtures.py from the
reference tree and evaluates the nine cases that the reference's golden
exporter defines (tools/s2_s3/export_golden.py:34-47): the textured scene at
K 500/2000, an odd 333x257 scene at K 1000/20000/1 (threshold 40), noise at
K 300 with threshold 10 and harris_k 0.04/0, a flat image and a thin image.
Each case is written as one compressed .npz holding the inputs (gray, knobs)
and the reference outputs (blurred image, keypoints x/y/response,
descriptors), plus manifest.json with the versions and a SHA-256 per file.
The GPU box never runs this script; it only reads the committed .npz files.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import platform
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def cases(fixtures):
    scene = fixtures.textured_scene()
    odd = fixtures.textured_scene(seed=3, height=257, width=333)
    return [
        ("scene_k500", scene, 20, 500, 0.04),
        ("scene_k2000", scene, 20, 2000, 0.04),
        ("odd_k1000", odd, 20, 1000, 0.04),
        ("odd_k20000_all", odd, 20, 20000, 0.04),
        ("odd_k1_t40", odd, 40, 1, 0.04),
        ("noise_k300_t10", fixtures.noise(5, 192, 256), 10, 300, 0.04),
        ("noise_k300_t10_harris0", fixtures.noise(5, 192, 256), 10, 300, 0.0),
        ("flat_k100", np.full((128, 128), 77, np.uint8), 20, 100, 0.04),
        ("tiny_k100", fixtures.noise(9, 62, 200), 10, 100, 0.04),
    ]


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", type=Path, required=True, help="the reference source tree")
    ap.add_argument("--out", type=Path, default=HERE)
    args = ap.parse_args()
    sys.path.insert(0, str(args.reference))
    from tools.s2_s3 import fixtures, reference  # noqa: E402  (reference tree)
    import cv2  # noqa: E402

    manifest = {"numpy": np.__version__, "opencv": cv2.__version__,
                "python": platform.python_version(),
                "source": "tools/s2_s3/reference.py (reference tree)", "cases": {}}
    for name, gray, thr, k, hk in cases(fixtures):
        kp, desc = reference.detect_and_describe(gray, thr, k, hk)
        path = args.out / f"s2s3_{name}.npz"
        np.savez_compressed(path, gray=gray, blurred=reference.blur(gray),
                            keypoints=np.ascontiguousarray(kp, np.float32),
                            descriptors=np.ascontiguousarray(desc, np.uint8),
                            knobs=np.array([thr, k], np.int64),
                            harris_k=np.array([hk], np.float32))
        manifest["cases"][name] = {"file": path.name, "width": int(gray.shape[1]),
                                   "height": int(gray.shape[0]), "fast_threshold": thr,
                                   "max_keypoints": k, "harris_k": hk,
                                   "count": int(kp.shape[0]),
                                   "sha256": hashlib.sha256(path.read_bytes()).hexdigest()}
        print(f"{name}: {kp.shape[0]} keypoints")
    taps = reference.BLUR_TAPS.astype(np.float32)
    manifest["blur_taps_hex"] = [float(t).hex() for t in taps]
    manifest["umax"] = [int(v) for v in reference.umax()]
    pat = reference.load_pattern()
    manifest["pattern_sha256"] = hashlib.sha256(
        np.ascontiguousarray(pat, np.int32).tobytes()).hexdigest()
    (args.out / "s2s3_manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()

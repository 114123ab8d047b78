"""The S2/S3 oracle against golden fixtures made by the reference's own
tools/s2_s3/reference.py (tests/golden/make_golden.py): keypoints,
responses, blur and descriptors bit for bit on all nine reference cases."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import s2s3

GOLDEN = Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((GOLDEN / "s2s3_manifest.json").read_text())
CASES = sorted(MANIFEST["cases"])


def load(name):
    z = np.load(GOLDEN / MANIFEST["cases"][name]["file"])
    thr, k = (int(v) for v in z["knobs"])
    return z, thr, k, float(z["harris_k"][0])


@pytest.mark.parametrize("name", CASES)
def test_fixture_integrity(name):
    c = MANIFEST["cases"][name]
    assert hashlib.sha256((GOLDEN / c["file"]).read_bytes()).hexdigest() == c["sha256"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_golden(name):
    z, thr, k, hk = load(name)
    kp, desc = s2s3.detect_and_describe(z["gray"], thr, k, hk)
    assert kp.shape == z["keypoints"].shape
    assert np.array_equal(kp, z["keypoints"])
    assert np.array_equal(desc, z["descriptors"])
    assert np.array_equal(s2s3.blur(z["gray"]), z["blurred"])


def test_tables_match_reference():
    assert [float(t).hex() for t in s2s3.TAPS] == MANIFEST["blur_taps_hex"]
    assert [int(v) for v in s2s3.patch_half_widths()] == MANIFEST["umax"]
    pat = np.ascontiguousarray(s2s3.pattern(), np.int32)
    assert hashlib.sha256(pat.tobytes()).hexdigest() == MANIFEST["pattern_sha256"]


def test_edge_cases():
    flat = np.full((100, 100), 9, np.uint8)
    assert s2s3.detect(flat, 20, 50).shape == (0, 3)
    rng = np.random.default_rng(1)
    noise = rng.integers(0, 256, (64, 64), dtype=np.uint8)   # 64 > 2*31: one interior row/col pair
    kp = s2s3.detect(noise, 10, 5)
    assert kp.shape[0] <= 5
    assert s2s3.detect(noise, 10, 0).shape == (0, 3)
    with pytest.raises(ValueError):
        s2s3.fast_score_map(noise, 0)

"""The scale-pyramid oracle (levels > 1) against OpenCV's ORB.

The reference is single-level, so the pyramid has no reference vectors. The
oracle is checked instead against cv2.ORB_create(nlevels=8, scaleFactor=1.2,
edgeThreshold=31, patchSize=31, WTA_K=2, HARRIS_SCORE) with the acceptance
bar the reference uses for its single-level check against OpenCV
(tests/python/test_s2_s3_reference.py:75-87): keypoint sets overlap >= 95 %,
Harris responses exact on shared keypoints, >= 99 % of their descriptors
bit-exact and the rest within 2 bits. The layer images themselves are checked
bit for bit against cv2.resize(INTER_LINEAR_EXACT).
"""
import numpy as np
import pytest

from crossstage_stitch_b200 import synth
from oracle import pyramid, s2s3

cv2 = pytest.importorskip("cv2")


def cv_orb(k, levels=8, scale=1.2, threshold=20):
    return cv2.ORB_create(nfeatures=k, scaleFactor=scale, nlevels=levels, edgeThreshold=31, firstLevel=0,
                          WTA_K=2, scoreType=cv2.ORB_HARRIS_SCORE, patchSize=31, fastThreshold=threshold)


@pytest.mark.parametrize("size", [(512, 512), (333, 257), (640, 480), (100, 37), (1, 5), (7, 1)])
@pytest.mark.parametrize("factor", [1.2, 1.44, 2.0, 3.7])
def test_resize_matches_opencv_linear_exact(size, factor):
    w, h = size
    img = np.random.default_rng(w * 7 + h).integers(0, 256, (h, w), dtype=np.uint8)
    dw, dh = max(1, round(w / factor)), max(1, round(h / factor))
    want = cv2.resize(img, (dw, dh), interpolation=cv2.INTER_LINEAR_EXACT)
    assert np.array_equal(pyramid.resize_linear_exact(img, dw, dh), want)


def test_budgets_and_scales():
    assert pyramid.level_budgets(1000, 8, 1.2) == [217, 181, 151, 126, 105, 87, 73, 60]
    assert pyramid.level_budgets(2000, 8, 1.2) == [434, 362, 302, 251, 209, 175, 145, 122]
    assert pyramid.level_budgets(777, 1, 1.2) == [777]
    for k in (0, 1, 3, 7, 15, 999, 20000):
        for levels in (2, 5, 8, 16):
            b = pyramid.level_budgets(k, levels, 1.2)
            assert len(b) == levels and min(b) >= 0 and sum(b) == k
    assert [s for s in pyramid.layer_sizes(512, 512, 8, 1.2)] == [
        (512, 512), (427, 427), (356, 356), (296, 296), (247, 247), (206, 206), (171, 171), (143, 143)]
    # the scale factor is a float32, as in cv::ORB::create
    assert pyramid.layer_scales(8, 1.2)[7] == np.float32(np.float64(np.float32(1.2)) ** 7)


@pytest.fixture(scope="module")
def view_a():
    return synth.config0_pair(0).gray_a


@pytest.mark.parametrize("k", [500, 1000, 2000])
def test_pyramid_matches_opencv_orb(view_a, k):
    kp, desc = pyramid.detect_and_describe(view_a, 20, k, 8, 1.2)
    cv_kp, cv_desc = cv_orb(k).detectAndCompute(view_a, None)
    assert len(kp) == len(cv_kp) == len(desc)
    # per-level counts: OpenCV's octave field against the oracle's level spans
    layers = pyramid.build_layers(view_a, 8, 1.2)
    budgets = pyramid.level_budgets(k, 8, 1.2)
    counts = [len(s2s3.detect(layer, 20, budgets[l])) for l, layer in enumerate(layers)]
    assert counts == np.bincount([p.octave for p in cv_kp], minlength=8).tolist()
    theirs = {(float(p.pt[0]), float(p.pt[1])): (np.float32(p.response), d) for p, d in zip(cv_kp, cv_desc)}
    mine = {(float(x), float(y)): (r, d) for (x, y, r), d in zip(kp, desc)}
    shared = set(theirs) & set(mine)
    assert len(shared) >= 0.95 * len(cv_kp)
    assert all(theirs[p][0] == mine[p][0] for p in shared)
    bits = np.array([int(np.unpackbits(theirs[p][1] ^ mine[p][1]).sum()) for p in shared])
    assert np.count_nonzero(bits == 0) >= 0.99 * len(shared)
    assert bits.max() <= 2


def test_single_level_is_the_reference_path(view_a):
    kp1, d1 = pyramid.detect_and_describe(view_a, 20, 300, 1, 1.2)
    kp0, d0 = s2s3.detect_and_describe(view_a, 20, 300)
    assert np.array_equal(kp1, kp0) and np.array_equal(d1, d0)


def test_small_layers_hold_nothing():
    img = synth.make_pair(5, 130, 90).gray_a
    layers = pyramid.build_layers(img, 8, 1.2)
    # 130x90 -> 108x75 -> 90x62: the third layer is 62 rows high, not built
    assert [layer.shape for layer in layers] == [(90, 130), (75, 108)]
    kp, desc = pyramid.detect_and_describe(img, 10, 200, 8, 1.2)
    assert kp.shape[0] == desc.shape[0] and kp.shape[0] <= 200
    tiny = np.full((40, 40), 9, np.uint8)
    kp, desc = pyramid.detect_and_describe(tiny, 20, 100, 8, 1.2)
    assert kp.shape == (0, 3) and desc.shape == (0, 32)

"""S6 on the CPU: the canvas geometry of the oracle, of this library's host
code (stitch_s6_prepare_geometry; no device work) and, where it was built
from the reference tree, of the reference's own src/s6/geometry.cpp, all on
the known answers of the reference's tests/test_s6_geometry.cpp:40-193 and
bit for bit on each other; then the oracle's feather render against the
reference's FP64 NumPy render (tests/golden/s6_feather.npz; canvas and mask
exact, RGB within 2, the reference's own bar in tests/test_s6_cuda.cu:443-448)
and against the expectations of tests/test_s6_cuda.cu:105-276."""
import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

from crossstage_stitch_b200 import _abi
from oracle import c_oracle

ROOT = Path(__file__).resolve().parents[1]
REF_GEOM = ROOT / "oracle" / "_ref" / "libref_s6geom.so"
GOLDEN = ROOT / "tests" / "golden" / "s6_feather.npz"

OK, INVALID, INSUFFICIENT, DEGENERATE = 0, 1, 2, 5
IDENTITY = [1, 0, 0, 0, 1, 0, 0, 0, 1.0]
INT_MAX = 2**31 - 1
SIZE_MAX = 2**64 - 1


def policy(**kw):
    p = dict(denominator_tolerance=1e-12, inverse_tolerance=1e-12, snap_tolerance=1e-10,
             max_canvas_pixels=16777216)
    p.update(kw)
    return p


class Impl:
    """prepare_geometry of one implementation, as (status, geometry dict)."""

    def __init__(self, which):
        self.which = which
        if which == "library":
            self.fn = _abi.load().stitch_s6_prepare_geometry
        elif which == "reference":
            if not REF_GEOM.exists():
                pytest.skip("reference geometry build not present (oracle/_ref)")
            self.fn = C.CDLL(str(REF_GEOM)).ref_s6_prepare_geometry
            self.fn.restype = C.c_int
            self.fn.argtypes = _abi.PROTOTYPES["stitch_s6_prepare_geometry"][1]

    def __call__(self, wa, ha, wb, hb, h, p=None):
        p = p or policy()
        if self.which == "oracle":
            op = c_oracle.s6_policy(p["denominator_tolerance"], p["inverse_tolerance"], p["snap_tolerance"],
                                    p["max_canvas_pixels"])
            st, g = c_oracle.s6_geometry(wa, ha, wb, hb, h, op)
            return st, {"width": g.w, "height": g.h, "origin_x": g.ox, "origin_y": g.oy, "width_a": g.wa,
                        "height_a": g.ha, "width_b": g.wb, "height_b": g.hb, "denominator_tolerance": g.den_tol,
                        "snap_tolerance": g.snap_tol, "inverse": list(g.inv)}
        sp = _abi.S6Policy(**p)
        g = _abi.S6Geometry()
        hp = None if h is None else (C.c_double * 9)(*h)
        st = self.fn(wa, ha, wb, hb, hp, C.byref(sp), C.byref(g))
        return st, {k: (list(getattr(g, k)) if k == "inverse" else getattr(g, k)) for k, _ in g._fields_}


@pytest.fixture(params=["oracle", "library", "reference"])
def prep(request):
    return Impl(request.param)


def inverse_point(g, ax, ay, bx, by, tol=1e-10):
    m = g["inverse"]
    w = m[6] * ax + m[7] * ay + m[8]
    assert math.isfinite(w) and w != 0
    assert abs((m[0] * ax + m[1] * ay + m[2]) / w - bx) <= tol
    assert abs((m[3] * ax + m[4] * ay + m[5]) / w - by) <= tol


def expect_failure(prep, status, wa, ha, wb, hb, h, p=None):
    st, g = prep(wa, ha, wb, hb, h, p)
    assert st == status
    assert (g["width"], g["height"], g["origin_x"], g["origin_y"]) == (0, 0, 0, 0)
    assert (g["width_a"], g["height_a"], g["width_b"], g["height_b"]) == (0, 0, 0, 0)
    assert all(v == 0 for v in g["inverse"])


def test_identity_and_dimensions(prep):
    st, g = prep(4, 3, 4, 3, IDENTITY)
    assert st == OK and (g["width"], g["height"], g["origin_x"], g["origin_y"]) == (4, 3, 0, 0)
    assert (g["width_a"], g["height_a"], g["width_b"], g["height_b"]) == (4, 3, 4, 3)
    inverse_point(g, 3, 2, 3, 2)
    st, g = prep(4, 3, 6, 2, IDENTITY)
    assert st == OK and (g["width"], g["height"]) == (6, 3)
    st, g = prep(1, 1, 1, 1, IDENTITY)
    assert st == OK and (g["width"], g["height"]) == (1, 1)
    inverse_point(g, 0, 0, 0, 0)


def test_translation_and_scale_equivalence(prep):
    t = [1, 0, -2, 0, 1, 0, 0, 0, 1.0]
    st, g = prep(4, 3, 4, 3, t)
    assert st == OK and (g["width"], g["height"], g["origin_x"], g["origin_y"]) == (6, 3, -2, 0)
    inverse_point(g, -2, 0, 0, 0)
    inverse_point(g, 1, 2, 3, 2)
    for factor in (-1.0, 1e-320, 1e-250, -1e250):
        st, g = prep(4, 3, 4, 3, [v * factor for v in t])
        assert st == OK and (g["width"], g["height"], g["origin_x"]) == (6, 3, -2)
        inverse_point(g, -2, 2, 0, 2)
    st, g = prep(2, 3, 2, 3, [1, 0, 0, 0, 1, -3, 0, 0, 1.0])
    assert st == OK and (g["width"], g["height"], g["origin_y"]) == (2, 6, -3)
    st, g = prep(2, 2, 4, 3, [0, 1, 0, 1, 0, 0, 0, 0, 1.0])  # axis interchange: a row pivot
    assert st == OK and (g["width"], g["height"]) == (3, 4)
    inverse_point(g, 2, 3, 3, 2)


def test_projective_and_h33(prep):
    st, g = prep(2, 2, 4, 3, [1, 0, 0, 0, 1, 0, 0.25, 0, 1.0])
    assert st == OK and (g["width"], g["height"]) == (3, 3)
    inverse_point(g, 12.0 / 7, 8.0 / 7, 3, 2)
    expect_failure(prep, DEGENERATE, 2, 1, 2, 1, [1, 0, 1, 0, 1, 0, 1, 0, 0.0])
    st, g = prep(2, 1, 2, 1, [1, 0, 1, 0, 1, 0, 1, 0, 1e-5])
    assert st == OK and (g["width"], g["height"]) == (100001, 1)
    inverse_point(g, 100000, 0, 0, 0, 1e-9)


def test_horizon_singular_and_conditioning(prep):
    expect_failure(prep, DEGENERATE, 3, 3, 3, 3, [1, 0, 0, 0, 1, 0, 1, 0, -1.0])
    expect_failure(prep, DEGENERATE, 3, 3, 3, 3, [1, 0, 0, 0, 1, 0, -0.5, 0, 1.0])
    expect_failure(prep, DEGENERATE, 2, 2, 2, 2, [1, 2, 0, 2, 4, 0, 0, 0, 1.0])
    expect_failure(prep, DEGENERATE, 4, 3, 4, 3, [1e-15, 0, 0, 0, 1, 0, 0, 0, 1.0])
    for bad in (math.inf, math.nan):
        h = list(IDENTITY)
        h[2] = bad
        expect_failure(prep, DEGENERATE, 2, 2, 2, 2, h)
    expect_failure(prep, DEGENERATE, 2, 2, 2, 2, [0.0] * 9)
    st, g = prep(20001, 1, 10001, 1, [1, 0, 10000, 0, 1, 0, 0, 0, 1.0])
    assert st == OK and (g["width"], g["height"]) == (20001, 1)
    inverse_point(g, 10000, 0, 0, 0, 1e-8)


def test_snapping_budget_and_overflow(prep):
    t = [1, 0, -2 - 5e-11, 0, 1, 0, 0, 0, 1.0]
    st, g = prep(4, 3, 4, 3, t)
    assert st == OK and (g["width"], g["origin_x"]) == (6, -2)
    t[2] = -2 - 1e-6
    st, g = prep(4, 3, 4, 3, t)
    assert st == OK and (g["width"], g["origin_x"]) == (7, -3)
    t[2] = -2
    expect_failure(prep, INSUFFICIENT, 4, 3, 4, 3, t, policy(max_canvas_pixels=17))
    st, _ = prep(4, 3, 4, 3, t, policy(max_canvas_pixels=18))
    assert st == OK
    for far in (1e30, -1e30):
        t[2] = far
        expect_failure(prep, INSUFFICIENT, 4, 3, 4, 3, t, policy(max_canvas_pixels=SIZE_MAX))
    expect_failure(prep, INSUFFICIENT, INT_MAX, 2, 1, 1, IDENTITY)
    t[2] = 1000000 + 1e-10  # the scale-aware rounding floor snaps this
    st, g = prep(2, 1, 2, 1, t, policy(max_canvas_pixels=2000000, inverse_tolerance=1e-15))
    assert st == OK and (g["width"], g["height"]) == (1000002, 1)
    st, g = prep(INT_MAX, 1, INT_MAX, 1, IDENTITY, policy(max_canvas_pixels=INT_MAX))
    assert st == OK and (g["width"], g["height"]) == (INT_MAX, 1)


def test_invalid_arguments(prep):
    for dims in ((0, 2, 2, 2), (2, -1, 2, 2), (2, 2, 0, 2), (2, 2, 2, -1)):
        expect_failure(prep, INVALID, *dims, IDENTITY)
    expect_failure(prep, INVALID, 2, 2, 2, 2, None)
    for bad in (dict(denominator_tolerance=0), dict(inverse_tolerance=math.nan), dict(inverse_tolerance=1),
                dict(snap_tolerance=-1), dict(max_canvas_pixels=0)):
        expect_failure(prep, INVALID, 2, 2, 2, 2, IDENTITY, policy(**bad))


def test_policy_propagation(prep):
    st, g = prep(2, 2, 2, 2, IDENTITY, policy(denominator_tolerance=1e-9, snap_tolerance=1e-7))
    assert st == OK and g["denominator_tolerance"] == 1e-9 and g["snap_tolerance"] == 1e-7


def test_library_null_output_and_default_policy():
    L = _abi.load()
    assert L.stitch_s6_prepare_geometry(2, 2, 2, 2, (C.c_double * 9)(*IDENTITY), None, None) == INVALID
    p = _abi.S6Policy()
    L.stitch_s6_default_policy(C.byref(p))
    assert (p.denominator_tolerance, p.inverse_tolerance, p.snap_tolerance, p.max_canvas_pixels) == (
        1e-12, 1e-12, 1e-10, 16777216)
    g = _abi.S6Geometry()  # a NULL policy is the default policy
    assert L.stitch_s6_prepare_geometry(4, 3, 4, 3, (C.c_double * 9)(1, 0, -2, 0, 1, 0, 0, 0, 1), None,
                                        C.byref(g)) == OK
    assert (g.width, g.origin_x) == (6, -2)


def random_homographies(n, seed):
    rng = np.random.default_rng(seed)
    for _ in range(n):
        wa, ha, wb, hb = (int(v) for v in rng.integers(1, 2000, 4))
        ang = rng.uniform(-0.5, 0.5)
        s = rng.uniform(0.5, 2.0)
        h = np.array([[s * math.cos(ang), -s * math.sin(ang), rng.uniform(-500, 500)],
                      [s * math.sin(ang), s * math.cos(ang), rng.uniform(-500, 500)],
                      [rng.normal(0, 2e-4), rng.normal(0, 2e-4), 1.0]])
        h *= rng.choice([-1.0, 1.0]) * 10.0 ** rng.uniform(-3, 3)
        yield wa, ha, wb, hb, [float(v) for v in h.ravel()]


@pytest.mark.parametrize("other", ["library", "reference"])
def test_geometry_bit_exact_against_oracle(other):
    """Same 80-bit operations in the same order: identical status, canvas and inverse bits."""
    o, x = Impl("oracle"), Impl(other)
    n_ok = 0
    for wa, ha, wb, hb, h in random_homographies(400, 11):
        so, go = o(wa, ha, wb, hb, h)
        sx, gx = x(wa, ha, wb, hb, h)
        assert so == sx, (wa, ha, wb, hb, h)
        assert go == gx, (wa, ha, wb, hb, h)
        n_ok += so == OK
    assert n_ok > 200


def golden_cases():
    z = np.load(GOLDEN)
    names = sorted({k.split(".")[0] for k in z.files})
    return [(n, {k.split(".", 1)[1]: z[k] for k in z.files if k.split(".")[0] == n}) for n in names]


GOLDEN_CASES = golden_cases()


@pytest.mark.parametrize("name,case", GOLDEN_CASES, ids=[n for n, _ in GOLDEN_CASES])
def test_oracle_feather_vs_reference_fp64(name, case):
    a, b, h = case["a"], case["b"], case["H"]
    st, g = c_oracle.s6_geometry(a.shape[1], a.shape[0], b.shape[1], b.shape[0], h)
    assert st == OK
    assert [g.w, g.h, g.ox, g.oy] == case["canvas"].tolist()
    pano, mask, (n_union, n_overlap) = c_oracle.s6_feather(a, b, g)
    np.testing.assert_array_equal(mask, case["mask"])
    diff = np.abs(pano.astype(np.int32) - case["panorama"].astype(np.int32))
    assert diff.max() <= 2, (name, int(diff.max()))
    assert n_union == int(case["mask"].sum()) and n_overlap <= n_union


def oracle_render(a, b, h):
    st, g = c_oracle.s6_geometry(a.shape[1], a.shape[0], b.shape[1], b.shape[0], h)
    assert st == OK
    return g, *c_oracle.s6_feather(a, b, g)


def test_known_answers_from_reference_render_tests():
    # identity, black valid (tests/test_s6_cuda.cu:105-125)
    for w, hh in ((1, 1), (1, 9), (11, 1), (11, 7), (33, 17)):
        px = ((np.arange(w * hh * 3) * 37) % 256).astype(np.uint8).reshape(hh, w, 3)
        px[0, 0] = 0
        _, pano, mask, _ = oracle_render(px, px, IDENTITY)
        assert np.abs(pano.astype(int) - px.astype(int)).max() <= 1 and mask.all()
    # full overlap (:126-139): equal scores average 20 and 200
    _, pano, _, _ = oracle_render(np.full((7, 9, 3), 20, np.uint8), np.full((7, 9, 3), 200, np.uint8), IDENTITY)
    assert np.abs(pano.astype(int) - 110).max() <= 1
    # negative origin (:140-165)
    a, b = np.full((3, 5, 3), 20, np.uint8), np.full((3, 5, 3), 200, np.uint8)
    g, pano, mask, stats = oracle_render(a, b, [1, 0, -2, 0, 1, -1, 0, 0, 1.0])
    assert (g.w, g.h, g.ox, g.oy) == (7, 4, -2, -1) and stats == (24, 6)
    for y in range(g.h):
        for x in range(g.w):
            xa, ya = x + g.ox, y + g.oy
            ma = 0 <= xa < 5 and 0 <= ya < 3
            mb = -2 <= xa < 3 and -1 <= ya < 2
            assert mask[y, x] == (ma or mb)
            if not (ma and mb):
                assert (pano[y, x] == (20 if ma else 200 if mb else 0)).all()
    # gap (:166-191)
    g, pano, mask, stats = oracle_render(np.zeros((3, 4, 3), np.uint8), np.full((3, 4, 3), 255, np.uint8),
                                         [1, 0, 7, 0, 1, 0, 0, 0, 1.0])
    assert (g.w, g.h) == (11, 3) and stats == (24, 0)
    xs = np.arange(11)
    assert (mask == ((xs < 4) | (xs >= 7))[None, :]).all()
    assert (pano == np.where(xs >= 7, 255, 0)[None, :, None]).all()
    # statistics (:263-276)
    assert oracle_render(np.zeros((3, 5, 3), np.uint8), np.zeros((3, 5, 3), np.uint8), IDENTITY)[3] == (15, 15)
    assert oracle_render(np.zeros((3, 259, 3), np.uint8), np.zeros((3, 259, 3), np.uint8),
                         IDENTITY)[3] == (777, 777)

"""ctypes binding of liboracle.so (the C restatement of S4/S5).

Test infrastructure only."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class OTop2(C.Structure):
    _fields_ = [("first_distance", C.c_double), ("second_distance", C.c_double),
                ("first_index", C.c_int), ("second_index", C.c_int)]


class OModel(C.Structure):
    _fields_ = [("h", C.c_double * 9), ("loss", C.c_double), ("hypothesis", C.c_int), ("valid", C.c_int)]


class OResult(C.Structure):
    _fields_ = [("H", C.c_double * 9), ("H_s", C.c_double * 9), ("num_matches", C.c_int),
                ("num_inliers", C.c_int), ("inlier_ratio", C.c_double), ("inlier_coverage", C.c_double),
                ("reproj_residual", C.c_double), ("status", C.c_int)]


class OS6Policy(C.Structure):
    _fields_ = [("den_tol", C.c_double), ("inv_tol", C.c_double), ("snap_tol", C.c_double),
                ("max_pixels", C.c_size_t)]


class OS6Geom(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("ox", C.c_int), ("oy", C.c_int), ("wa", C.c_int),
                ("ha", C.c_int), ("wb", C.c_int), ("hb", C.c_int), ("den_tol", C.c_double),
                ("snap_tol", C.c_double), ("inv", C.c_double * 9)]


TOP2_DTYPE = np.dtype([("first_distance", "<f8"), ("second_distance", "<f8"),
                       ("first_index", "<i4"), ("second_index", "<i4")])

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
        L = C.CDLL(str(LIB))
        vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        L.oracle_s4_top2.argtypes = [ip, vp, ip, ip, ip, vp, ip, ip, ip, ip, vp]
        L.oracle_s4_accept.argtypes = [vp, ip, vp, C.c_double, ip, vp, vp, vp]
        L.oracle_s4_accept.restype = ip
        L.oracle_residual2.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double]
        L.oracle_residual2.restype = C.c_double
        L.oracle_s1.argtypes = [vp, ip, ip, ip, ip, ip, vp]
        L.oracle_s1_gradient.argtypes = [vp, ip, ip, ip]
        L.oracle_s1_gradient.restype = C.c_double
        L.oracle_splitmix64.argtypes = [C.c_uint64]
        L.oracle_splitmix64.restype = C.c_uint64
        L.oracle_sample_four.argtypes = [ip, C.c_uint64, ip, vp]
        L.oracle_fit.argtypes = [ip, vp, vp, vp]
        L.oracle_nondegenerate.argtypes = [vp]
        L.oracle_valid_domain.argtypes = [vp, ip, ip]
        L.oracle_mat3_inverse.argtypes = [vp, vp]
        L.oracle_s5_search.argtypes = [ip, vp, C.c_uint64, ip, ip, ip, ip, C.c_double, C.POINTER(OModel)]
        L.oracle_s5_finish.argtypes = [ip, vp, ip, C.POINTER(OModel), ip, ip, C.c_double, ip, ip, ip, ip,
                                       ip, ip, vp, vp, vp, C.POINTER(OResult)]
        L.oracle_make_scale_info.argtypes = [ip, ip, C.c_double, vp, vp, vp]
        L.oracle_s6_geometry.argtypes = [ip, ip, ip, ip, vp, C.POINTER(OS6Policy), C.POINTER(OS6Geom)]
        L.oracle_s6_feather.argtypes = [vp, ip, vp, ip, C.POINTER(OS6Geom), vp, ip, vp, ip, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray | None) -> C.c_void_p:
    return C.c_void_p(0 if a is None else a.ctypes.data)


def top2(desc_q: np.ndarray, desc_t: np.ndarray, count_q: int | None = None, count_t: int | None = None,
         l2: bool = False) -> np.ndarray:
    """Exact top-2 of every query row (structured TOP2_DTYPE array)."""
    q = np.ascontiguousarray(desc_q)
    t = np.ascontiguousarray(desc_t)
    cq, ct = q.shape[0], t.shape[0]
    nq = cq if count_q is None else count_q
    nt = ct if count_t is None else count_t
    dim = q.shape[1] if q.ndim == 2 else 1
    out = np.zeros(cq, TOP2_DTYPE)
    if cq == 0:
        return out
    lib().oracle_s4_top2(1 if l2 else 0, _p(q), cq, nq, q.strides[0] if q.ndim == 2 else q.itemsize,
                         _p(t) if ct else C.c_void_p(0), ct, nt,
                         (t.strides[0] if t.ndim == 2 else t.itemsize) if ct else 1, dim, _p(out))
    return out


def accept(forward: np.ndarray, reverse: np.ndarray | None, ratio: float, l2: bool = False):
    """Ratio test, optional mutual check, compaction in query order."""
    n = forward.shape[0]
    ia = np.zeros(max(n, 1), np.int32)
    ib = np.zeros(max(n, 1), np.int32)
    d = np.zeros(max(n, 1), np.float32)
    m = lib().oracle_s4_accept(_p(forward), n, _p(reverse), ratio, 1 if l2 else 0, _p(ia), _p(ib), _p(d))
    return ia[:m], ib[:m], d[:m]


def mat3_inverse(m: np.ndarray) -> np.ndarray | None:
    m = np.ascontiguousarray(m, np.float64).reshape(9)
    out = np.zeros(9)
    return out if lib().oracle_mat3_inverse(_p(m), _p(out)) else None


def make_scale_info(w: int, h: int, s: float = 1.0) -> dict:
    wh = np.zeros(2, np.int32)
    sxy = np.zeros(2)
    d = np.zeros(9)
    st = lib().oracle_make_scale_info(w, h, s, _p(wh), _p(sxy), _p(d))
    if st != 0:
        raise ValueError("invalid scale")
    return {"orig_w": w, "orig_h": h, "work_w": int(wh[0]), "work_h": int(wh[1]), "sx": sxy[0], "sy": sxy[1],
            "D": d}


def s5(points: np.ndarray, mask_capacity: int, hypotheses: int, threshold: float, seed: int,
       refinement_steps: int, scale_a: dict, scale_b: dict, status_in: int = 0,
       previous: OModel | None = None, first: int = 0):
    """Full S5 on (nm, 4) double points (ax, ay, bx, by). Returns (result dict,
    mask (mask_capacity,), raw best model)."""
    L = lib()
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 4)
    nm = pts.shape[0]
    best = OModel() if previous is None else previous
    if status_in == 0:
        L.oracle_s5_search(nm, _p(pts), seed, first, hypotheses, scale_b["work_w"], scale_b["work_h"],
                           threshold, C.byref(best))
    inv_a = mat3_inverse(scale_a["D"])
    d_b = np.ascontiguousarray(scale_b["D"], np.float64)
    mask = np.zeros(max(mask_capacity, 1), np.uint8)
    res = OResult()
    L.oracle_s5_finish(nm, _p(pts), mask_capacity, C.byref(best), status_in, refinement_steps, threshold,
                       scale_a["work_w"], scale_a["work_h"], scale_b["work_w"], scale_b["work_h"],
                       scale_b["orig_w"], scale_b["orig_h"], _p(inv_a), _p(d_b), _p(mask), C.byref(res))
    out = {"H": np.array(res.H[:]).reshape(3, 3), "H_s": np.array(res.H_s[:]).reshape(3, 3),
           "num_matches": res.num_matches, "num_inliers": res.num_inliers, "inlier_ratio": res.inlier_ratio,
           "inlier_coverage": res.inlier_coverage, "reproj_residual": res.reproj_residual,
           "status": res.status}
    return out, mask[:mask_capacity], best


def s1(rgb: np.ndarray, work_w: int, work_h: int) -> np.ndarray:
    """S1 of an (h, w, 3) uint8 RGB image to (work_h, work_w) GRAY8."""
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    h, w, _ = rgb.shape
    out = np.zeros((work_h, work_w), np.uint8)
    lib().oracle_s1(rgb.ctypes.data, w, h, 3 * w, work_w, work_h, out.ctypes.data)
    return out


def s1_gradient(gray: np.ndarray) -> float:
    gray = np.ascontiguousarray(gray, dtype=np.uint8)
    h, w = gray.shape
    return lib().oracle_s1_gradient(gray.ctypes.data, w, h, w)


def s6_policy(den_tol: float = 1e-12, inv_tol: float = 1e-12, snap_tol: float = 1e-10,
              max_pixels: int = 16777216) -> OS6Policy:
    return OS6Policy(den_tol, inv_tol, snap_tol, max_pixels)


def s6_geometry(wa: int, ha: int, wb: int, hb: int, h, policy: OS6Policy | None = None):
    """(status, OS6Geom) of the B -> A canvas geometry; h None passes NULL."""
    g = OS6Geom()
    hp = None if h is None else np.ascontiguousarray(h, np.float64).reshape(9)
    st = lib().oracle_s6_geometry(wa, ha, wb, hb, _p(hp), C.byref(policy or s6_policy()), C.byref(g))
    return st, g


def s6_feather(a: np.ndarray, b: np.ndarray, g: OS6Geom):
    """Feather render of RGB8 (h, w, 3) images a, b on geometry g:
    (panorama (g.h, g.w, 3) uint8, mask (g.h, g.w) uint8 0/1, (union, overlap))."""
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.uint8)
    assert a.shape == (g.ha, g.wa, 3) and b.shape == (g.hb, g.wb, 3)
    out = np.zeros((g.h, g.w, 3), np.uint8)
    mask = np.zeros((g.h, g.w), np.uint8)
    stats = np.zeros(2, np.uint64)
    lib().oracle_s6_feather(_p(a), a.strides[0], _p(b), b.strides[0], C.byref(g), _p(out), out.strides[0],
                            _p(mask), mask.strides[0], _p(stats))
    return out, mask, (int(stats[0]), int(stats[1]))

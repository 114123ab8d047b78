"""Helpers for the GPU tests: run one stage through the C ABI of this
library, or of the reference's own stage sources built for sm_100a
(oracle/_ref/libref_stages.so, a checker), on identical device buffers."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import torch

from crossstage_stitch_b200 import _abi
from crossstage_stitch_b200._abi import (BINARY_U8, FLOAT32, Descriptors, HomographyResult, ImageView, Keypoints,
                                         Matches, S2Config, S4Config, S5Config, ScaleInfo, Top2)

ROOT = Path(__file__).resolve().parents[1]
REF_STAGES = ROOT / "oracle" / "_ref" / "libref_stages.so"
PAD = 37  # pitch padding, exercises pitch_bytes != width
ref = C.byref


class Lib:
    """Uniform access to the stage entry points of one library."""

    def __init__(self, which: str = "ours"):
        self.which = which
        if which == "ours":
            self.L = _abi.load()
            self.pre = "stitch_"
        else:
            if not REF_STAGES.exists():
                raise FileNotFoundError(REF_STAGES)
            self.L = C.CDLL(str(REF_STAGES))
            self.pre = "ref_"
            for name in ("s2_workspace_bytes", "s2_detect", "s3_workspace_bytes", "s3_describe",
                         "s4_workspace_bytes", "s4_match", "s4_knn_top2", "s5_workspace_bytes", "s5_estimate"):
                fn = getattr(self.L, "ref_" + name)
                fn.restype = C.c_int
                fn.argtypes = _abi.PROTOTYPES["stitch_" + name][1]

    def __getattr__(self, name):
        return getattr(self.L, self.pre + name)


def stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def dev(a: np.ndarray, device="cuda") -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def pitched(gray: np.ndarray, pad: int = PAD) -> torch.Tensor:
    h, w = gray.shape
    t = torch.full((h, w + pad), 0xa5, dtype=torch.uint8, device="cuda")
    t[:, :w] = dev(gray)
    return t


def workspace(nbytes: int, guard: int = 64) -> torch.Tensor:
    return torch.full((nbytes + guard,), 0xa5, dtype=torch.uint8, device="cuda")


def detect_describe(lib: Lib, gray: np.ndarray, thr: int, k: int, harris_k: float = 0.04, capacity=None,
                    stride: int = 48):
    """S2 then S3 on one stream; returns (keypoints (n,3), descriptors (n,32),
    blurred image or None, status codes)."""
    h, w = gray.shape
    img = pitched(gray)
    iv = ImageView(img.data_ptr(), w, h, img.stride(0), 1)
    cap = k if capacity is None else capacity
    n = max(cap, 1)
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    y = torch.zeros_like(x)
    resp = torch.zeros_like(x)
    cnt = torch.full((1,), 0x7f7f7f7f, dtype=torch.int32, device="cuda")
    desc = torch.full((n, stride), 0xcd, dtype=torch.uint8, device="cuda")
    kp = Keypoints(x.data_ptr(), y.data_ptr(), resp.data_ptr(), cap, cnt.data_ptr())
    cfg = S2Config(thr, k, harris_k)
    b2, b3 = C.c_size_t(), C.c_size_t()
    assert lib.s2_workspace_bytes(w, h, ref(cfg), ref(b2)) == 0
    assert lib.s3_workspace_bytes(w, h, ref(b3)) == 0
    ws2, ws3 = workspace(b2.value), workspace(b3.value)
    s = stream()
    st2 = lib.s2_detect(ref(iv), ref(cfg), ref(kp), C.c_void_p(ws2.data_ptr()), b2.value, s)
    d = Descriptors(BINARY_U8, 32, stride, desc.data_ptr())
    st3 = lib.s3_describe(ref(iv), ref(kp), ref(d), C.c_void_p(ws3.data_ptr()), b3.value, s)
    torch.cuda.synchronize()
    cnum = int(cnt.item())
    blurred = None
    if cap > 0 and st3 == 0:
        blurred = ws3[:w * h].reshape(h, w).cpu().numpy() if lib.which == "ours" else None
    kps = torch.stack([x[:cnum], y[:cnum], resp[:cnum]], 1).cpu().numpy() if cnum > 0 else np.zeros((0, 3), np.float32)
    raw = desc[:max(cnum, 0)].cpu().numpy()
    assert (raw[:, 32:] == 0xcd).all(), "descriptor stride padding was written"
    assert (ws2[b2.value:] == 0xa5).all().item() and (ws3[b3.value:] == 0xa5).all().item(), "workspace overrun"
    return kps, raw[:, :32].copy(), blurred, (st2, st3, cnum)


def match(lib: Lib, da: np.ndarray, db: np.ndarray, ratio: float = 0.8, cross: bool = False,
          count_a=None, count_b=None, pad_a: int = 0, pad_b: int = 0, dtype: int = BINARY_U8):
    """S4 on host descriptor arrays; returns (Top2 array, idx_a, idx_b, dist, status)."""
    ca, cb = da.shape[0], db.shape[0]
    dim = da.shape[1] if da.ndim == 2 else 1
    elem = 4 if dtype == FLOAT32 else 1
    np_t = np.float32 if dtype == FLOAT32 else np.uint8

    def side(arr, cap, pad, count):
        rows = torch.zeros((max(cap, 1), dim + pad), dtype=torch.float32 if dtype == FLOAT32 else torch.uint8,
                           device="cuda")
        if cap:
            rows[:cap, :dim] = dev(arr.reshape(cap, dim).astype(np_t))
        cnt = torch.tensor([cap if count is None else count], dtype=torch.int32, device="cuda")
        kp = Keypoints(0, 0, 0, cap, cnt.data_ptr())
        d = Descriptors(dtype, dim, (dim + pad) * elem, rows.data_ptr())
        return rows, cnt, kp, d

    ra, na, ka, dA = side(da, ca, pad_a, count_a)
    rb, nb, kb, dB = side(db, cb, pad_b, count_b)
    cfg = S4Config()
    cfg.ratio_threshold = ratio
    cfg.cross_check = 1 if cross else 0
    b = C.c_size_t()
    assert lib.s4_workspace_bytes(ca, cb, ref(cfg), ref(b)) == 0
    ws = workspace(b.value)
    n = max(ca, 1)
    ia = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    ib = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    dist = torch.zeros(n, dtype=torch.float32, device="cuda")
    mc = torch.full((1,), 0x7f7f7f7f, dtype=torch.int32, device="cuda")
    m = Matches(ia.data_ptr(), ib.data_ptr(), dist.data_ptr(), ca, mc.data_ptr())
    top = torch.zeros((n, 24), dtype=torch.uint8, device="cuda")
    s = stream()
    st_top = lib.s4_knn_top2(ref(ka), ref(dA), ref(kb), ref(dB), C.c_void_p(top.data_ptr()), s)
    st = lib.s4_match(ref(ka), ref(dA), ref(kb), ref(dB), ref(cfg), ref(m), C.c_void_p(ws.data_ptr()), b.value, s)
    torch.cuda.synchronize()
    assert (ws[b.value:] == 0xa5).all().item(), "S4 workspace overrun"
    k = int(mc.item())
    t2 = np.frombuffer(top[:ca].cpu().numpy().tobytes(), dtype=np.dtype([("first_distance", "<f8"),
                                                                         ("second_distance", "<f8"),
                                                                         ("first_index", "<i4"),
                                                                         ("second_index", "<i4")]))
    return t2, ia[:k].cpu().numpy(), ib[:k].cpu().numpy(), dist[:k].cpu().numpy(), (st_top, st)


class S5Fixture:
    """Device buffers for S5 on host keypoints/matches (reference fixture
    tests/test_s5_cuda.cu:40-97)."""

    def __init__(self, lib: Lib, n: int, capacity: int | None = None):
        self.lib = lib
        self.n = n
        cap = n if capacity is None else capacity
        self.cap = cap
        z = lambda dt: torch.zeros(max(cap, 1), dtype=dt, device="cuda")
        self.ax, self.ay, self.bx, self.by = (z(torch.float32) for _ in range(4))
        self.ia, self.ib = z(torch.int32), z(torch.int32)
        self.mask = torch.full((max(cap, 1),), 0xee, dtype=torch.uint8, device="cuda")
        self.na = torch.tensor([n], dtype=torch.int32, device="cuda")
        self.nb = torch.tensor([n], dtype=torch.int32, device="cuda")
        self.nm = torch.tensor([n], dtype=torch.int32, device="cuda")
        self.config = S5Config(257, 0, 32, 2, 0.5, 20261022, 1)
        b = C.c_size_t()
        assert lib.s5_workspace_bytes(ref(self.config), ref(b)) == 0
        self.bytes = b.value
        self.ws = torch.zeros(self.bytes, dtype=torch.uint8, device="cuda")
        self.pinned = torch.zeros(C.sizeof(HomographyResult), dtype=torch.uint8, pin_memory=True)
        self.sa = ScaleInfo()
        self.sb = ScaleInfo()
        _abi.load().stitch_make_scale_info(640, 480, 1.0, ref(self.sa))
        _abi.load().stitch_make_scale_info(640, 480, 1.0, ref(self.sb))

    def set_points(self, a: np.ndarray, b: np.ndarray, ia=None, ib=None):
        """a, b: (n, 2) float32 keypoints; match i pairs a[ia[i]] with b[ib[i]]."""
        n = a.shape[0]
        self.ax[:n] = dev(a[:, 0].astype(np.float32)); self.ay[:n] = dev(a[:, 1].astype(np.float32))
        self.bx[:n] = dev(b[:, 0].astype(np.float32)); self.by[:n] = dev(b[:, 1].astype(np.float32))
        idx = np.arange(n, dtype=np.int32)
        self.ia[:n] = dev(idx if ia is None else np.asarray(ia, np.int32))
        self.ib[:n] = dev(idx if ib is None else np.asarray(ib, np.int32))

    def views(self):
        ka = Keypoints(self.ax.data_ptr(), self.ay.data_ptr(), 0, self.cap, self.na.data_ptr())
        kb = Keypoints(self.bx.data_ptr(), self.by.data_ptr(), 0, self.cap, self.nb.data_ptr())
        m = Matches(self.ia.data_ptr(), self.ib.data_ptr(), 0, self.cap, self.nm.data_ptr())
        return ka, kb, m

    def call(self, ws_bytes=None, ws_offset=0):
        ka, kb, m = self.views()
        torch.cuda.synchronize()
        return self.lib.s5_estimate(ref(ka), ref(kb), ref(m), ref(self.sa), ref(self.sb), ref(self.config),
                                    C.c_void_p(self.mask.data_ptr()), C.c_void_p(self.pinned.data_ptr()),
                                    C.c_void_p(self.ws.data_ptr() + ws_offset),
                                    self.bytes if ws_bytes is None else ws_bytes, stream())

    def run(self) -> dict:
        assert self.call() == 0
        torch.cuda.synchronize()
        r = HomographyResult.from_buffer_copy(self.pinned.numpy().tobytes())
        return {"H": np.array(r.H[:]), "H_s": np.array(r.H_s[:]), "num_matches": r.num_matches,
                "num_inliers": r.num_inliers, "inlier_ratio": r.inlier_ratio,
                "inlier_coverage": r.inlier_coverage, "reproj_residual": r.reproj_residual, "status": r.status}

    def mask_host(self):
        return self.mask[:self.n].cpu().numpy()


def ref_available() -> bool:
    return REF_STAGES.exists()

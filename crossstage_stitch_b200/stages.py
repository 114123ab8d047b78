"""Python mirror of the stage API over torch CUDA tensors, and the plain
per-pair runner.

Function names and argument meaning follow the reference's C++ stage API
(src/s2_s3/s2.hpp:26-39, src/s2_s3/s3.hpp:19-30, src/s4/s4.hpp:25-60,
src/s5/s5.hpp:23-39); every call goes through the C ABI of libstitch_b200.so
and returns the Status code. PairRunner reproduces the reference harness's
fixed-config pair run (harness/pipeline_runner.cu:335-416): buffers are
allocated once for the largest image and K, then each pair runs
S2(A), S2(B), S3(A), S3(B), S4, S5 on one stream and synchronises once
(with pyramid levels > 1, S2+S3 of each image is one pyramid call).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _abi
from ._abi import (BINARY_U8, GRAY8, Descriptors, HomographyResult, ImageView, Keypoints, Matches,
                   PyramidConfig, S2Config, S4Config, S5Config, ScaleInfo, StageError, Status, Top2)

ref = C.byref


def lib():
    return _abi.load()


def stream_handle(stream: torch.cuda.Stream | None = None) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def ptr(t: torch.Tensor | None) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


def image_view(img: torch.Tensor, width: int | None = None, height: int | None = None) -> ImageView:
    """GRAY8 view of a (rows, pitch) uint8 device tensor; the visible width and
    height default to the tensor's shape."""
    assert img.dtype == torch.uint8 and img.dim() == 2 and img.is_cuda
    h = img.shape[0] if height is None else height
    w = img.shape[1] if width is None else width
    return ImageView(img.data_ptr(), w, h, img.stride(0), GRAY8)


def make_scale_info(w: int, h: int, s: float = 1.0) -> ScaleInfo:
    out = ScaleInfo()
    st = lib().stitch_make_scale_info(w, h, s, ref(out))
    if st != 0:
        raise StageError("make_scale_info", st)
    return out


def check(where: str, status: int) -> None:
    if status != Status.OK:
        raise StageError(where, status)


@dataclass
class Knobs:
    """Per-pair knobs: the reference's stage Config values
    (src/s2_s3/s2.hpp:19-23, src/s4/s4.hpp:8-11, src/s5/s5.hpp:11-19) with
    the harness defaults (harness/harness_types.hpp:23-29), plus the pyramid
    levels knob (levels 1 is the reference's single-level S2/S3)."""
    fast_threshold: int = 20
    max_keypoints: int = 1000
    harris_k: float = 0.04
    ratio: float = 0.8
    cross_check: bool = False
    hypotheses: int = 2000
    batch_size: int = 64
    refinement_steps: int = 1
    threshold: float = 3.0
    seed: int = 0
    generation: int = 1
    levels: int = 1
    scale_factor: float = 1.2

    def s2(self) -> S2Config:
        return S2Config(self.fast_threshold, self.max_keypoints, self.harris_k)

    def s4(self) -> S4Config:
        c = S4Config()
        c.ratio_threshold = self.ratio
        c.cross_check = 1 if self.cross_check else 0
        return c

    def s5(self, previous: int = 0) -> S5Config:
        return S5Config(self.hypotheses, previous, self.batch_size, self.refinement_steps, self.threshold,
                        self.seed, self.generation)

    def pyramid(self) -> PyramidConfig:
        return PyramidConfig(self.levels, self.scale_factor)


def result_dict(r: HomographyResult) -> dict:
    return {"H": np.array(r.H[:], np.float64).reshape(3, 3), "H_s": np.array(r.H_s[:], np.float64).reshape(3, 3),
            "num_matches": r.num_matches, "num_inliers": r.num_inliers, "inlier_ratio": r.inlier_ratio,
            "inlier_coverage": r.inlier_coverage, "reproj_residual": r.reproj_residual,
            "status": Status(r.status)}


@dataclass
class ImageFeatures:
    """Device buffers of one image's S2/S3 outputs."""
    capacity: int
    device: torch.device
    x: torch.Tensor = field(init=False)
    y: torch.Tensor = field(init=False)
    response: torch.Tensor = field(init=False)
    count: torch.Tensor = field(init=False)
    desc: torch.Tensor = field(init=False)

    def __post_init__(self):
        n = max(self.capacity, 1)
        self.x = torch.empty(n, dtype=torch.float32, device=self.device)
        self.y = torch.empty(n, dtype=torch.float32, device=self.device)
        self.response = torch.empty(n, dtype=torch.float32, device=self.device)
        self.count = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.desc = torch.zeros((n, 32), dtype=torch.uint8, device=self.device)

    def keypoints(self, capacity: int | None = None) -> Keypoints:
        return Keypoints(self.x.data_ptr(), self.y.data_ptr(), self.response.data_ptr(),
                         self.capacity if capacity is None else capacity, self.count.data_ptr())

    def descriptors(self) -> Descriptors:
        return Descriptors(BINARY_U8, 32, self.desc.stride(0), self.desc.data_ptr())


def workspace(nbytes: int, device) -> torch.Tensor:
    # cudaMalloc-backed torch storage starts 256-byte aligned (512 in practice).
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


class PairRunner:
    """The plain per-pair form: the drop-in stages called one pair at a time
    on one stream, exactly as the reference harness calls them."""

    def __init__(self, max_w: int, max_h: int, max_k: int, max_r: int = 8192, device: str | int = "cuda",
                 cross_check: bool = False, stage_lib=None):
        """stage_lib: an object with the stitch_* stage entry points of
        include/stitch_b200.h (default: this library)."""
        self.device = torch.device(device)
        self.L = L = stage_lib if stage_lib is not None else lib()
        self.max_w, self.max_h, self.max_k = max_w, max_h, max_k
        self.img = [torch.zeros((max_h, max_w), dtype=torch.uint8, device=self.device) for _ in range(2)]
        self.feat = [ImageFeatures(max_k, self.device) for _ in range(2)]
        n = max(max_k, 1)
        self.idx_a = torch.empty(n, dtype=torch.int32, device=self.device)
        self.idx_b = torch.empty(n, dtype=torch.int32, device=self.device)
        self.dist = torch.empty(n, dtype=torch.float32, device=self.device)
        self.mcount = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.mask = torch.zeros(n, dtype=torch.uint8, device=self.device)
        b = C.c_size_t()
        check("s2_workspace_bytes", L.stitch_s2_workspace_bytes(max_w, max_h, ref(S2Config(20, max_k, 0.04)), ref(b)))
        self.s2_bytes = b.value
        self.ws2 = [workspace(self.s2_bytes, self.device) for _ in range(2)]
        check("s3_workspace_bytes", L.stitch_s3_workspace_bytes(max_w, max_h, ref(b)))
        self.s3_bytes = b.value
        self.ws3 = workspace(self.s3_bytes, self.device)
        c4 = S4Config()
        c4.ratio_threshold = 0.8
        c4.cross_check = 1 if cross_check else 0
        check("s4_workspace_bytes", L.stitch_s4_workspace_bytes(max_k, max_k, ref(c4), ref(b)))
        self.s4_bytes = b.value
        self.ws4 = workspace(self.s4_bytes, self.device)
        check("s5_workspace_bytes", L.stitch_s5_workspace_bytes(ref(S5Config(max_r, 0, 64, 1, 3.0, 0, 1)), ref(b)))
        self.s5_bytes = b.value
        self.ws5 = workspace(self.s5_bytes, self.device)
        self.pinned = torch.zeros(C.sizeof(HomographyResult), dtype=torch.uint8, pin_memory=True)
        self.result = HomographyResult.from_address(self.pinned.data_ptr())
        self.wsp: dict[tuple[int, float], tuple[torch.Tensor, int]] = {}

    def pyramid_workspace(self, knobs: Knobs) -> tuple[torch.Tensor, int]:
        """Workspace of the pyramid S2/S3 call for the largest image and K at
        these levels (allocated on first use)."""
        key = (knobs.levels, float(np.float32(knobs.scale_factor)))
        if key not in self.wsp:
            b = C.c_size_t()
            check("pyramid_workspace_bytes", self.L.stitch_pyramid_workspace_bytes(
                self.max_w, self.max_h, ref(S2Config(20, self.max_k, 0.04)), ref(knobs.pyramid()), ref(b)))
            self.wsp[key] = (workspace(b.value, self.device), b.value)
        return self.wsp[key]

    def matches_view(self, capacity: int) -> Matches:
        return Matches(self.idx_a.data_ptr(), self.idx_b.data_ptr(), self.dist.data_ptr(), capacity,
                       self.mcount.data_ptr())

    def enqueue(self, wa: int, ha: int, wb: int, hb: int, knobs: Knobs, stream=None,
                scale_a: ScaleInfo | None = None, scale_b: ScaleInfo | None = None,
                images: tuple[torch.Tensor, torch.Tensor] | None = None) -> None:
        """Enqueues S2..S5 (no sync) for the pair in self.img[0/1], or in
        `images` (two device uint8 tensors) when given."""
        L = self.L
        s = stream_handle(stream)
        k = knobs.max_keypoints
        dims = ((wa, ha), (wb, hb))
        imgs = self.img if images is None else images
        c2 = knobs.s2()
        if knobs.levels > 1:
            wsp, nbytes = self.pyramid_workspace(knobs)
            for i in range(2):
                iv = image_view(imgs[i], *dims[i])
                check("pyramid_detect_describe", L.stitch_pyramid_detect_describe(
                    ref(iv), ref(c2), ref(knobs.pyramid()), ref(self.feat[i].keypoints(k)),
                    ref(self.feat[i].descriptors()), ptr(wsp), nbytes, s))
        else:
            for i in range(2):
                iv = image_view(imgs[i], *dims[i])
                check("s2_detect", L.stitch_s2_detect(ref(iv), ref(c2), ref(self.feat[i].keypoints(k)),
                                                      ptr(self.ws2[i]), self.s2_bytes, s))
            for i in range(2):
                iv = image_view(imgs[i], *dims[i])
                check("s3_describe", L.stitch_s3_describe(ref(iv), ref(self.feat[i].keypoints(k)),
                                                          ref(self.feat[i].descriptors()), ptr(self.ws3),
                                                          self.s3_bytes, s))
        ka, kb = self.feat[0].keypoints(k), self.feat[1].keypoints(k)
        da, db = self.feat[0].descriptors(), self.feat[1].descriptors()
        m = self.matches_view(k)
        check("s4_match", L.stitch_s4_match(ref(ka), ref(da), ref(kb), ref(db), ref(knobs.s4()), ref(m),
                                            ptr(self.ws4), self.s4_bytes, s))
        sa = scale_a if scale_a is not None else make_scale_info(wa, ha, 1.0)
        sb = scale_b if scale_b is not None else make_scale_info(wb, hb, 1.0)
        check("s5_estimate", L.stitch_s5_estimate(ref(ka), ref(kb), ref(m), ref(sa), ref(sb), ref(knobs.s5()),
                                                  ptr(self.mask), C.c_void_p(self.pinned.data_ptr()),
                                                  ptr(self.ws5), self.s5_bytes, s))

    def upload(self, gray_a: np.ndarray, gray_b: np.ndarray) -> None:
        for i, g in enumerate((gray_a, gray_b)):
            h, w = g.shape
            self.img[i][:h, :w].copy_(torch.from_numpy(np.ascontiguousarray(g)), non_blocking=False)

    def run(self, gray_a: np.ndarray, gray_b: np.ndarray, knobs: Knobs, stream=None) -> dict:
        """Uploads one pair, runs the chain, synchronises, returns the result."""
        self.upload(gray_a, gray_b)
        (ha, wa), (hb, wb) = gray_a.shape, gray_b.shape
        self.enqueue(wa, ha, wb, hb, knobs, stream)
        (stream or torch.cuda.current_stream()).synchronize()
        return result_dict(self.result)

    def download(self) -> dict:
        """Features, matches and mask of the last completed run (host copies)."""
        out = {}
        for i, tag in enumerate("ab"):
            f = self.feat[i]
            n = int(f.count.item())
            out[f"kp_{tag}"] = torch.stack([f.x[:n], f.y[:n], f.response[:n]], 1).cpu().numpy()
            out[f"desc_{tag}"] = f.desc[:n].cpu().numpy()
        n = int(self.mcount.item())
        out["idx_a"] = self.idx_a[:n].cpu().numpy()
        out["idx_b"] = self.idx_b[:n].cpu().numpy()
        out["distance"] = self.dist[:n].cpu().numpy()
        out["mask"] = self.mask[:n].cpu().numpy()
        return out

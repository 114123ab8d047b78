"""S6 for Python callers: the B -> A canvas geometry and the feather render of
two device RGB8 images, over the C ABI (stitch_s6_*).

Mirrors src/s6/geometry.hpp:43-44 (prepare_geometry) and src/s6/s6.hpp:44-47
(render): the geometry is host arithmetic; render() enqueues one kernel on
the current torch stream and returns without synchronising.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi
from ._abi import GRAY8, RGB8, ImageView, S6Geometry, S6Policy, StageError, Status


def default_policy() -> S6Policy:
    p = S6Policy()
    _abi.load().stitch_s6_default_policy(C.byref(p))
    return p


def prepare_geometry(width_a: int, height_a: int, width_b: int, height_b: int, H,
                     policy: S6Policy | None = None) -> S6Geometry:
    """The canvas and A -> B inverse for H (B -> A, 3x3); raises StageError
    with the status (DEGENERATE, INSUFFICIENT_WORKSPACE, INVALID_ARGUMENT)."""
    h = np.ascontiguousarray(np.asarray(H, np.float64).reshape(9))
    g = S6Geometry()
    st = _abi.load().stitch_s6_prepare_geometry(width_a, height_a, width_b, height_b,
                                                h.ctypes.data_as(C.POINTER(C.c_double)),
                                                C.byref(policy) if policy is not None else None, C.byref(g))
    if st != Status.OK:
        raise StageError("s6 prepare_geometry", st)
    return g


def rgb_view(t: torch.Tensor, width: int | None = None) -> ImageView:
    """ImageView of a (h, >= 3 w) uint8 CUDA tensor holding packed RGB rows,
    or of a contiguous (h, w, 3) tensor."""
    if t.dim() == 3:
        h, w, _ = t.shape
        return ImageView(t.data_ptr(), w, h, t.stride(0), RGB8)
    h = t.shape[0]
    return ImageView(t.data_ptr(), width if width is not None else t.shape[1] // 3, h, t.stride(0), RGB8)


def render(a: torch.Tensor, b: torch.Tensor, geometry: S6Geometry, output: torch.Tensor | None = None,
           mask: torch.Tensor | None = None, statistics: torch.Tensor | None = None):
    """Feather render of device RGB8 images a, b ((h, w, 3) uint8 CUDA) onto
    the canvas of geometry. Returns (panorama (H, W, 3), mask (H, W) 0/1);
    statistics, when given, is a 2-element int64/uint64 CUDA tensor that
    receives {union_pixels, overlap_pixels}."""
    g = geometry
    dev = a.device
    if output is None:
        output = torch.empty((g.height, g.width, 3), dtype=torch.uint8, device=dev)
    if mask is None:
        mask = torch.empty((g.height, g.width), dtype=torch.uint8, device=dev)
    va, vb, vo = rgb_view(a), rgb_view(b), rgb_view(output)
    vm = ImageView(mask.data_ptr(), g.width, g.height, mask.stride(0), GRAY8)
    stats = None if statistics is None else C.cast(statistics.data_ptr(), C.POINTER(C.c_uint64))
    st = _abi.load().stitch_s6_render(C.byref(va), C.byref(vb), C.byref(g), _abi.S6_FEATHER, C.byref(vo),
                                      C.byref(vm), None, 0, C.c_void_p(torch.cuda.current_stream(dev).cuda_stream),
                                      stats)
    if st != Status.OK:
        raise StageError("s6 render", st)
    return output, mask

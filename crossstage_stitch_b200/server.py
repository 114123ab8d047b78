"""Served form: a native request loop (C ABI stitch_server_*) that admits
image pairs of uneven size under an HBM budget and batches them
continuously; see csrc/server.cu."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi, replicas
from ._abi import Request, ServerConfig, ServerResult, StageError
from .stages import Knobs, result_dict


def pinned_image(gray) -> torch.Tensor:
    """A pinned host uint8 tensor, (rows, cols) GRAY8 or (rows, cols, 3) RGB8,
    holding `gray`."""
    if isinstance(gray, torch.Tensor) and gray.is_pinned() and gray.dtype == torch.uint8:
        return gray
    t = torch.empty(tuple(gray.shape), dtype=torch.uint8, pin_memory=True)
    t.copy_(torch.as_tensor(np.ascontiguousarray(gray)))
    return t


class Server:
    """Owns the device arena (its size is the admission budget) and the
    native server. Images passed to submit() are kept alive until their
    result has been polled."""

    def __init__(self, arena_bytes: int = 8 << 30, max_batch: int = 64, streams: int = 2, device=None):
        self.lib = _abi.load()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.arena = torch.empty(arena_bytes, dtype=torch.uint8, device=self.device)
        cfg = ServerConfig(self.arena.data_ptr(), arena_bytes, self.device.index, max_batch, streams)
        h = C.c_void_p()
        st = self.lib.stitch_server_create(C.byref(cfg), C.byref(h))
        if st != 0:
            raise StageError("stitch_server_create", st)
        self.handle = h
        self.held: dict[int, tuple] = {}
        self._buf = (ServerResult * 256)()

    def submit(self, gray_a, gray_b, knobs: Knobs, tag: int, scale_a=None, scale_b=None, s1_scale: float = 1.0,
               retry_hypotheses: int = 0, retry_min_inliers: int = 0, panorama_capacity: int = 0) -> int:
        st, r, held = self.request(gray_a, gray_b, knobs, tag, scale_a, scale_b, s1_scale, retry_hypotheses,
                                   retry_min_inliers, panorama_capacity)
        return st if st != 0 else self.submit_request(r, held)

    def request(self, gray_a, gray_b, knobs: Knobs, tag: int, scale_a=None, scale_b=None, s1_scale: float = 1.0,
                retry_hypotheses: int = 0, retry_min_inliers: int = 0, panorama_capacity: int = 0):
        """(0, request, host buffers) for submit_request(); the arguments are
        submit()'s."""
        """Queues one pair; returns the status code (0 = queued). (rows, cols, 3)
        images are RGB8: the server converts and resizes them with S1 at
        s1_scale on the device and returns H in their original coordinates.
        retry_hypotheses > knobs.hypotheses: a result that is not OK or has
        fewer than retry_min_inliers inliers is retried once by extending the
        saved S5 search to retry_hypotheses. panorama_capacity > 0 (RGB8
        requests): the server also renders the S6 feather panorama of the
        original images from the returned H, for canvases of up to that many
        pixels; poll() then returns it as "panorama" (h, w, 3) and "mask"."""
        a, b = pinned_image(gray_a), pinned_image(gray_b)
        r = Request()
        r.host_a, r.host_b = a.data_ptr(), b.data_ptr()
        r.width_a, r.height_a, r.pitch_a = a.shape[1], a.shape[0], a.stride(0)
        r.width_b, r.height_b, r.pitch_b = b.shape[1], b.shape[0], b.stride(0)
        r.rgb = 1 if a.dim() == 3 else 0
        r.scale = s1_scale if r.rgb else 0.0
        r.retry_hypotheses, r.retry_min_inliers = retry_hypotheses, retry_min_inliers
        if scale_a is not None:
            r.scale_a = scale_a
        if scale_b is not None:
            r.scale_b = scale_b
        r.s2, r.s4, r.s5, r.pyramid = knobs.s2(), knobs.s4(), knobs.s5(), knobs.pyramid()
        r.tag = tag
        pano = mask = None
        if panorama_capacity > 0:
            pano = torch.empty(3 * panorama_capacity, dtype=torch.uint8, pin_memory=True)
            mask = torch.empty(panorama_capacity, dtype=torch.uint8, pin_memory=True)
            r.host_panorama, r.host_mask, r.panorama_capacity = pano.data_ptr(), mask.data_ptr(), panorama_capacity
        return 0, r, (a, b, pano, mask)

    def submit_request(self, r: Request, held) -> int:
        """Queues a request built by request(); `held` stays alive until its
        result is polled."""
        self.held[r.tag] = held
        st = self.lib.stitch_server_submit(self.handle, C.byref(r))
        if st != 0:
            del self.held[r.tag]
        return st

    def poll(self) -> list[dict]:
        out = []
        while True:
            n = C.c_int()
            st = self.lib.stitch_server_poll(self.handle, self._buf, len(self._buf), C.byref(n))
            if st != 0:
                raise StageError("stitch_server_poll", st)
            for i in range(n.value):
                r = self._buf[i]
                d = result_dict(r.result) if r.status == 0 else {"status": r.status}
                d.update(tag=r.tag, submit_ms=r.submit_ms, launch_ms=r.launch_ms, done_ms=r.done_ms,
                         latency_ms=r.done_ms - r.submit_ms, batch_pairs=r.batch_pairs, run_status=r.status,
                         attempts=r.attempts, render_status=r.render_status)
                held = self.held.pop(r.tag, None)
                if r.render_status == 0 and held is not None:
                    w, h = r.canvas_width, r.canvas_height
                    d.update(panorama=held[2][:3 * w * h].numpy().reshape(h, w, 3).copy(),
                             mask=held[3][:w * h].numpy().reshape(h, w).copy(), canvas=(w, h),
                             origin=(r.origin_x, r.origin_y), union_pixels=r.union_pixels,
                             overlap_pixels=r.overlap_pixels)
                out.append(d)
            if n.value < len(self._buf):
                return out

    def outstanding(self) -> int:
        return self.lib.stitch_server_outstanding(self.handle)

    def close(self) -> None:
        """Finishes the queued work and stops the server; results not polled
        by then are dropped."""
        if getattr(self, "handle", None):
            self.lib.stitch_server_destroy(self.handle)
            self.handle = None

    def drain(self, timeout_s: float = 120.0) -> list[dict]:
        import time
        out, t0 = [], time.time()
        while self.outstanding() > 0:
            out += self.poll()
            if time.time() - t0 > timeout_s:
                raise TimeoutError(f"{self.outstanding()} requests still outstanding")
            time.sleep(0.0005)
        return out + self.poll()

    def __del__(self):
        self.close()


class MultiServer:
    """One Server per GPU of the node and a least-loaded dispatcher over
    their arenas: pairs are independent, so a request goes to the GPU with
    the most free admission budget (its footprint from
    stitch_server_request_bytes) and no collective is involved. Results
    carry "gpu", the index into `devices`."""

    def __init__(self, devices, arena_bytes: int = 8 << 30, max_batch: int = 64, streams: int = 2):
        self.devices = list(devices)
        self.servers = [Server(arena_bytes, max_batch, streams, device=d) for d in self.devices]
        self.dispatch = replicas.LeastLoadedDispatcher([arena_bytes] * len(self.devices))
        self.lib = _abi.load()

    def submit(self, gray_a, gray_b, knobs: Knobs, tag: int, **kw) -> int:
        head = self.servers[0]
        st, r, held = head.request(gray_a, gray_b, knobs, tag, **kw)
        if st != 0:
            return st
        nbytes = C.c_size_t()
        st = self.lib.stitch_server_request_bytes(C.byref(r), C.byref(nbytes))
        if st != 0:
            return st
        try:
            gpu = self.dispatch.place(tag, nbytes.value)
        except ValueError:
            return int(_abi.Status.INSUFFICIENT_WORKSPACE)
        st = self.servers[gpu].submit_request(r, held)
        if st != 0:
            self.dispatch.release(tag)
        return st

    def poll(self) -> list[dict]:
        out = []
        for g, srv in enumerate(self.servers):
            for res in srv.poll():
                self.dispatch.release(res["tag"])
                res["gpu"] = g
                out.append(res)
        return out

    def outstanding(self) -> int:
        return sum(s.outstanding() for s in self.servers)

    def drain(self, timeout_s: float = 120.0) -> list[dict]:
        import time
        out, t0 = [], time.time()
        while self.outstanding() > 0:
            out += self.poll()
            if time.time() - t0 > timeout_s:
                raise TimeoutError(f"{self.outstanding()} requests still outstanding")
            time.sleep(0.0005)
        return out + self.poll()

    def close(self) -> None:
        for s in self.servers:
            s.close()

"""Batched form: many uneven pairs registered by one launch per stage kernel,
optionally replayed as a captured CUDA graph (C ABI stitch_batch_*)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi
from ._abi import Descriptors, HomographyResult, ImageView, Keypoints, Matches, PairDesc, StageError
from .stages import Knobs, result_dict


def pair_desc(img_a: torch.Tensor, img_b: torch.Tensor, knobs: Knobs, size_a=None, size_b=None) -> PairDesc:
    """Descriptor of one pair over device uint8 images (rows, pitch); sizes
    default to the tensors' shapes."""
    wa, ha = size_a if size_a else (img_a.shape[1], img_a.shape[0])
    wb, hb = size_b if size_b else (img_b.shape[1], img_b.shape[0])
    d = PairDesc()
    d.image_a = ImageView(img_a.data_ptr(), wa, ha, img_a.stride(0), 1)
    d.image_b = ImageView(img_b.data_ptr(), wb, hb, img_b.stride(0), 1)
    d.s2, d.s4, d.s5 = knobs.s2(), knobs.s4(), knobs.s5()
    d.pyramid = knobs.pyramid()
    return d


class Batch:
    """Plan + workspace of one batch. The images must stay alive (and at the
    same addresses) while the plan is used."""

    def __init__(self, descs: list[PairDesc], device=None, tuning: dict | None = None):
        """tuning: launch shapes of the plan (the fields of
        _abi.BatchTuning; missing or 0 fields keep their defaults)."""
        self.lib = _abi.load()
        self.n = len(descs)
        arr = (PairDesc * self.n)(*descs)
        plan = C.c_void_p()
        nbytes = C.c_size_t()
        bad = C.c_int(-1)
        t = None
        if tuning:
            t = _abi.BatchTuning(**{k: int(v) for k, v in tuning.items()})
        st = self.lib.stitch_batch_create_tuned(self.n, arr, C.byref(t) if t is not None else None, C.byref(plan),
                                                C.byref(nbytes), C.byref(bad))
        if st != 0:
            raise StageError(f"stitch_batch_create (pair {bad.value})", st)
        self.plan = plan
        self.bytes = nbytes.value
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.ws = torch.empty(self.bytes, dtype=torch.uint8, device=self.device)
        self.results = torch.zeros(self.n * C.sizeof(HomographyResult), dtype=torch.uint8, pin_memory=True)
        self.captured = False

    def __del__(self):
        if getattr(self, "plan", None):
            self.lib.stitch_batch_destroy(self.plan)
            self.plan = None

    def _stream(self, stream):
        s = stream if stream is not None else torch.cuda.current_stream()
        return C.c_void_p(s.cuda_stream)

    def enqueue(self, stream=None, copy_results=True) -> None:
        st = self.lib.stitch_batch_enqueue(self.plan, C.c_void_p(self.ws.data_ptr()), self.bytes,
                                           C.c_void_p(self.results.data_ptr() if copy_results else 0),
                                           self._stream(stream))
        if st != 0:
            raise StageError("stitch_batch_enqueue", st)

    def capture(self, stream=None, copy_results=True) -> None:
        s = stream or torch.cuda.Stream()
        with torch.cuda.stream(s):
            st = self.lib.stitch_batch_capture(self.plan, C.c_void_p(self.ws.data_ptr()), self.bytes,
                                               C.c_void_p(self.results.data_ptr() if copy_results else 0),
                                               C.c_void_p(s.cuda_stream))
        s.synchronize()
        if st != 0:
            raise StageError("stitch_batch_capture", st)
        self.captured = True

    def set_marks(self, events: list | None) -> None:
        """events: one torch.cuda.Event(enable_timing=True) per name in
        _abi.BATCH_MARKS, recorded after the matching kernel group."""
        if events is None:
            st = self.lib.stitch_batch_set_marks(self.plan, None, 0)
        else:
            for e in events:   # torch creates the CUDA event on first record
                e.record()
            arr = (C.c_void_p * len(events))(*[e.cuda_event for e in events])
            st = self.lib.stitch_batch_set_marks(self.plan, arr, len(events))
        if st != 0:
            raise StageError("stitch_batch_set_marks", st)

    def launch(self, stream=None) -> None:
        st = self.lib.stitch_batch_launch(self.plan, self._stream(stream))
        if st != 0:
            raise StageError("stitch_batch_launch", st)

    def result(self, i: int) -> dict:
        size = C.sizeof(HomographyResult)
        r = HomographyResult.from_buffer_copy(self.results.numpy()[i * size:(i + 1) * size].tobytes())
        return result_dict(r)

    def outputs(self, i: int) -> dict:
        """Host copies of pair i's keypoints, descriptors, matches and mask."""
        ka, kb, m = Keypoints(), Keypoints(), Matches()
        da, db = Descriptors(), Descriptors()
        mask = C.c_void_p()
        res = C.c_void_p()
        st = self.lib.stitch_batch_pair_outputs(self.plan, C.c_void_p(self.ws.data_ptr()), i, C.byref(ka),
                                                C.byref(kb), C.byref(da), C.byref(db), C.byref(m), C.byref(mask),
                                                C.byref(res))
        if st != 0:
            raise StageError("stitch_batch_pair_outputs", st)
        base = self.ws.data_ptr()

        def view(ptr, count, dtype):
            off = ptr - base
            itemsize = torch.empty(0, dtype=dtype).element_size()
            return self.ws[off:off + count * itemsize].view(dtype)

        out = {}
        for tag, k, d in (("a", ka, da), ("b", kb, db)):
            n = int(view(k.d_count, 1, torch.int32).item())
            xs = view(k.x, n, torch.float32)
            ys = view(k.y, n, torch.float32)
            rs = view(k.response, n, torch.float32)
            out[f"kp_{tag}"] = torch.stack([xs, ys, rs], 1).cpu().numpy() if n else np.zeros((0, 3), np.float32)
            out[f"desc_{tag}"] = view(d.data, n * 32, torch.uint8).reshape(n, 32).cpu().numpy()
        nm = int(view(m.d_count, 1, torch.int32).item())
        out["idx_a"] = view(m.idx_a, nm, torch.int32).cpu().numpy()
        out["idx_b"] = view(m.idx_b, nm, torch.int32).cpu().numpy()
        out["distance"] = view(m.distance, nm, torch.float32).cpu().numpy()
        out["mask"] = view(mask.value, nm, torch.uint8).cpu().numpy()
        return out


class StreamingBatches:
    """The batched form over a stream of batches of one shape.

    All images of a step live in one contiguous buffer (image `side` of pair
    p at byte layout[p][side], rows of pitch_of(width) bytes), so a step's inputs
    move with one host-to-device copy. Two device slots, each with its own
    captured graph and compute stream, alternate: step() copies the pinned
    host buffer into the free slot on a copy stream and launches that slot's
    graph on the slot's stream when the copy lands, so the copy of one step
    overlaps the registration of the previous one, and a step's first kernels
    may start on SMs that the previous step's last kernels leave idle. A
    slot's results stay valid until the step after next is launched;
    wait(slot) then result(slot, i) reads them. The host buffer of a step must
    not be refilled before that step's copy has finished (use two host
    buffers, alternating)."""

    def __init__(self, sizes: list[tuple[int, int, int, int]], knobs: list[Knobs], device=None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.sizes = list(sizes)
        self.layout, cursor = [], 0
        for (wa, ha, wb, hb) in self.sizes:
            offs = []
            for (w, h) in ((wa, ha), (wb, hb)):
                offs.append(cursor)
                cursor += -(-self.pitch_of(w) * h // 256) * 256
            self.layout.append(tuple(offs))
        self.nbytes = max(cursor, 1)
        self.slots = [torch.empty(self.nbytes, dtype=torch.uint8, device=self.device) for _ in range(2)]
        self.copy_stream = torch.cuda.Stream(self.device)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(2)]  # compute stream of each slot
        self.batches = []
        for buf, stream in zip(self.slots, self.streams):
            descs = []
            for (wa, ha, wb, hb), (oa, ob), k in zip(self.sizes, self.layout, knobs):
                d = PairDesc()
                d.image_a = ImageView(buf.data_ptr() + oa, wa, ha, self.pitch_of(wa), 1)
                d.image_b = ImageView(buf.data_ptr() + ob, wb, hb, self.pitch_of(wb), 1)
                d.s2, d.s4, d.s5 = k.s2(), k.s4(), k.s5()
                d.pyramid = k.pyramid()
                descs.append(d)
            b = Batch(descs, self.device)
            b.capture(stream)
            self.batches.append(b)
        self.copied = [torch.cuda.Event() for _ in range(2)]
        self.done = [torch.cuda.Event() for _ in range(2)]
        for e, stream in zip(self.done, self.streams):
            e.record(stream)
        self.next = 0

    @staticmethod
    def pitch_of(width: int) -> int:
        return -(-width // 16) * 16

    def host_buffer(self) -> torch.Tensor:
        """A pinned host buffer of this layout."""
        return torch.zeros(self.nbytes, dtype=torch.uint8, pin_memory=True)

    def fill(self, host: torch.Tensor, pair: int, gray_a: np.ndarray, gray_b: np.ndarray) -> None:
        """Writes one pair's GRAY8 images into a host buffer of this layout."""
        for side, g in enumerate((gray_a, gray_b)):
            h, w = g.shape
            off, pitch = self.layout[pair][side], self.pitch_of(w)
            host[off:off + pitch * h].view(h, pitch)[:, :w].copy_(torch.from_numpy(np.ascontiguousarray(g)))

    def step(self, host: torch.Tensor) -> int:
        """Queues one step (copy, then registration); returns its slot."""
        s = self.next
        self.next ^= 1
        self.copy_stream.wait_event(self.done[s])  # the slot's previous step has finished
        with torch.cuda.stream(self.copy_stream):
            self.slots[s].copy_(host, non_blocking=True)
        self.copied[s].record(self.copy_stream)
        self.streams[s].wait_event(self.copied[s])
        self.batches[s].launch(self.streams[s])
        self.done[s].record(self.streams[s])
        return s

    def wait(self, slot: int) -> None:
        self.done[slot].synchronize()

    def result(self, slot: int, i: int) -> dict:
        return self.batches[slot].result(i)

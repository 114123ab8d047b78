"""s4_forward_neighbors (src/s4/s4.cu:265-272): after s4_match, the forward
Top2 of every query row sits at offset 0 of the S4 workspace, where the
reference's controller features read it (harness/pipeline_runner.cu:446-450).
Through the C ABI: the pointer returned is the workspace itself, its rows
equal s4_knn_top2 and the CPU oracle bit for bit, for both matchers and with
the mutual check on and off; a short or misaligned workspace, capacity_a 0
and a null output are INVALID_ARGUMENT."""
import ctypes as C

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi
from crossstage_stitch_b200._abi import BINARY_U8, Descriptors, Keypoints, Matches, S4Config, Status
from oracle import c_oracle

pytestmark = pytest.mark.gpu

TOP2 = np.dtype([("first_distance", "<f8"), ("second_distance", "<f8"), ("first_index", "<i4"),
                 ("second_index", "<i4")])


def planted(nq, nt, seed):
    rng = np.random.default_rng(seed)
    q = rng.integers(0, 256, (nq, 32), dtype=np.uint8)
    t = rng.integers(0, 256, (nt, 32), dtype=np.uint8)
    for qi in rng.choice(nq, size=nq // 3, replace=False):
        row = np.unpackbits(q[qi]).copy()
        row[rng.choice(256, size=int(rng.binomial(256, 0.05)), replace=False)] ^= 1
        t[rng.integers(0, nt)] = np.packbits(row)
    t[5] = t[9]   # an exact tie of train rows: the lower index wins
    return q, t


@pytest.mark.parametrize("matcher", [0, 1], ids=["popc", "tensor"])
@pytest.mark.parametrize("cross", [False, True])
def test_forward_neighbors_is_the_forward_top2(cuda, matcher, cross):
    L = _abi.load()
    before = L.stitch_s4_matcher()
    assert L.stitch_s4_set_matcher(matcher) == 0
    try:
        q, t = planted(1200, 1700, 31 + cross)
        dq, dt = torch.from_numpy(q).to(cuda), torch.from_numpy(t).to(cuda)
        cq = torch.tensor([q.shape[0]], dtype=torch.int32, device=cuda)
        ct = torch.tensor([t.shape[0]], dtype=torch.int32, device=cuda)
        ka, kb = Keypoints(0, 0, 0, q.shape[0], cq.data_ptr()), Keypoints(0, 0, 0, t.shape[0], ct.data_ptr())
        da, db = Descriptors(BINARY_U8, 32, 32, dq.data_ptr()), Descriptors(BINARY_U8, 32, 32, dt.data_ptr())
        cfg = S4Config()
        cfg.ratio_threshold = 0.8
        cfg.cross_check = 1 if cross else 0
        nb = C.c_size_t()
        assert L.stitch_s4_workspace_bytes(q.shape[0], t.shape[0], C.byref(cfg), C.byref(nb)) == 0
        ws = torch.zeros(nb.value + 256, dtype=torch.uint8, device=cuda)
        n = q.shape[0]
        ia, ib = torch.empty(n, dtype=torch.int32, device=cuda), torch.empty(n, dtype=torch.int32, device=cuda)
        dist, mc = torch.empty(n, dtype=torch.float32, device=cuda), torch.zeros(1, dtype=torch.int32, device=cuda)
        m = Matches(ia.data_ptr(), ib.data_ptr(), dist.data_ptr(), n, mc.data_ptr())
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert L.stitch_s4_match(C.byref(ka), C.byref(da), C.byref(kb), C.byref(db), C.byref(cfg), C.byref(m),
                                 C.c_void_p(ws.data_ptr()), nb.value, s) == 0
        top = torch.zeros(n * 24, dtype=torch.uint8, device=cuda)
        assert L.stitch_s4_knn_top2(C.byref(ka), C.byref(da), C.byref(kb), C.byref(db),
                                    C.c_void_p(top.data_ptr()), s) == 0
        out = C.c_void_p()
        assert L.stitch_s4_forward_neighbors(n, t.shape[0], C.byref(cfg), C.c_void_p(ws.data_ptr()), nb.value,
                                             C.byref(out)) == 0
        assert out.value == ws.data_ptr()
        torch.cuda.synchronize()
        fwd = np.frombuffer(ws[:n * 24].cpu().numpy().tobytes(), TOP2)
        direct = np.frombuffer(top.cpu().numpy().tobytes(), TOP2)
        want = c_oracle.top2(q, t)
        for f in TOP2.names:
            assert np.array_equal(fwd[f], direct[f]), f
            assert np.array_equal(fwd[f], want[f]), f
        # host-only rejections, in the reference's order
        p = C.c_void_p(ws.data_ptr())
        assert L.stitch_s4_forward_neighbors(n, t.shape[0], C.byref(cfg), p, nb.value - 1,
                                             C.byref(out)) == Status.INVALID_ARGUMENT
        assert L.stitch_s4_forward_neighbors(n, t.shape[0], C.byref(cfg), C.c_void_p(ws.data_ptr() + 4), nb.value,
                                             C.byref(out)) == Status.INVALID_ARGUMENT
        assert L.stitch_s4_forward_neighbors(0, t.shape[0], C.byref(cfg), p, nb.value,
                                             C.byref(out)) == Status.INVALID_ARGUMENT
        assert L.stitch_s4_forward_neighbors(n, t.shape[0], C.byref(cfg), None, nb.value,
                                             C.byref(out)) == Status.INVALID_ARGUMENT
        assert L.stitch_s4_forward_neighbors(n, t.shape[0], C.byref(cfg), p, nb.value, None) \
            == Status.INVALID_ARGUMENT
    finally:
        L.stitch_s4_set_matcher(before)

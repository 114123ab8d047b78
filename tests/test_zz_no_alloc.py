"""stitch_s4_match_static: S4 matching for callers that cannot allocate
device memory (their host process owns every device allocation, or their
loop cannot afford cudaMalloc's device-wide synchronisation). It uses a
scratch array held in the library's own device memory instead of a caller
workspace. This test calls it through the C ABI twice in a row and checks
each result against the workspace entry point stitch_s4_match on the same
inputs: match indices and distances must be identical (bit-exact, the
tolerance every S4 test here uses). It also checks that a request beyond the
scratch limit is refused without writing the output count.

The file name sorts last so a run that stops at the first failure has
already run every other test; it passes alone in a fresh process too."""
import ctypes as C

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi
from crossstage_stitch_b200._abi import Descriptors, Keypoints, Matches, S4Config

pytestmark = pytest.mark.gpu


def planted(nq, nt, seed):
    rng = np.random.default_rng(seed)
    q = rng.integers(0, 256, (nq, 32), dtype=np.uint8)
    t = rng.integers(0, 256, (nt, 32), dtype=np.uint8)
    for qi in rng.choice(nq, size=nq // 3, replace=False):
        row = np.unpackbits(q[qi]).copy()
        row[rng.choice(256, size=int(rng.binomial(256, 0.05)), replace=False)] ^= 1
        t[rng.integers(0, nt)] = np.packbits(row)
    return q, t


class Side:
    def __init__(self, rows: np.ndarray, dev):
        self.rows = torch.from_numpy(rows).to(dev)
        self.count = torch.tensor([rows.shape[0]], dtype=torch.int32, device=dev)
        self.kp = Keypoints(0, 0, 0, rows.shape[0], self.count.data_ptr())
        self.desc = Descriptors(0, 32, 32, self.rows.data_ptr())


class Out:
    def __init__(self, cap, dev):
        self.ia = torch.full((cap,), -1, dtype=torch.int32, device=dev)
        self.ib = torch.full((cap,), -1, dtype=torch.int32, device=dev)
        self.d = torch.zeros(cap, dtype=torch.float32, device=dev)
        self.n = torch.full((1,), 0x7f7f7f7f, dtype=torch.int32, device=dev)
        self.m = Matches(self.ia.data_ptr(), self.ib.data_ptr(), self.d.data_ptr(), cap, self.n.data_ptr())

    def host(self):
        k = int(self.n.item())
        return self.ia[:k].cpu().numpy(), self.ib[:k].cpu().numpy(), self.d[:k].cpu().numpy()


@pytest.mark.parametrize("cross", [False, True])
def test_static_scratch_matches_workspace_entry_point(cross):
    assert torch.cuda.is_available()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = _abi.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    cfg = S4Config()
    cfg.ratio_threshold = 0.8
    cfg.cross_check = 1 if cross else 0
    cases = [planted(1500, 1700, 21), planted(3000, 800, 22)]
    for q, t in cases:   # two calls in a row on different inputs share the scratch
        a, b = Side(q, dev), Side(t, dev)
        want = Out(q.shape[0], dev)
        nbytes = C.c_size_t()
        assert L.stitch_s4_workspace_bytes(q.shape[0], t.shape[0], C.byref(cfg), C.byref(nbytes)) == 0
        ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
        assert L.stitch_s4_match(C.byref(a.kp), C.byref(a.desc), C.byref(b.kp), C.byref(b.desc), C.byref(cfg),
                                 C.byref(want.m), C.c_void_p(ws.data_ptr()), nbytes.value, stream) == 0
        got = Out(q.shape[0], dev)
        assert L.stitch_s4_match_static(C.byref(a.kp), C.byref(a.desc), C.byref(b.kp), C.byref(b.desc),
                                        C.byref(cfg), C.byref(got.m), stream) == 0
        torch.cuda.synchronize()
        w, g = want.host(), got.host()
        assert w[0].size > 0
        for x, y in zip(w, g):
            assert np.array_equal(x, y)


def test_static_scratch_rejects_oversize_request():
    dev = torch.device("cuda", 0)
    L = _abi.load()
    cfg = S4Config()
    cfg.ratio_threshold = 0.8
    cfg.cross_check = 1
    big = 200000   # needs more than the 4 MiB scratch with the mutual check
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    rows = torch.zeros(16, dtype=torch.uint8, device=dev)
    kp = Keypoints(0, 0, 0, big, cnt.data_ptr())
    desc = Descriptors(0, 32, 0, rows.data_ptr())   # stride 0 never read: the size check comes first
    out = Out(1, dev)
    out.m.capacity = big
    st = L.stitch_s4_match_static(C.byref(kp), C.byref(desc), C.byref(kp), C.byref(desc), C.byref(cfg),
                                  C.byref(out.m), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _abi.Status.INSUFFICIENT_WORKSPACE
    torch.cuda.synchronize()
    assert int(out.n.item()) == 0x7f7f7f7f

"""stitch_s4_match_static: S4 matching for callers that cannot allocate
device memory (their host process owns every device allocation, or their
loop cannot afford cudaMalloc's device-wide synchronisation). It uses a
scratch array held in the library's own device memory instead of a caller
workspace.

The tests call it through the C ABI, two calls in a row, and check each
result against the workspace entry point stitch_s4_match on the same inputs
and against the CPU oracle: match indices and distances must be identical
(bit-exact, the tolerance every S4 test here uses). Each matcher (__popc and
tensor cores) and the FLOAT32 layout run right after a larger call, so
anything left in the shared scratch by that call would show. A request
beyond the scratch limit is refused without writing the output count.

The file name sorts last so a run that stops at the first failure has
already run every other test; it passes alone in a fresh process too."""
import ctypes as C

import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi
from crossstage_stitch_b200._abi import BINARY_U8, FLOAT32, Descriptors, Keypoints, Matches, S4Config
from oracle import c_oracle

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


def floats(nq, nt, dim, seed):
    rng = np.random.default_rng(seed)
    t = rng.standard_normal((nt, dim)).astype(np.float32)
    q = rng.standard_normal((nq, dim)).astype(np.float32)
    pick = rng.choice(nq, size=nq // 2, replace=False)
    q[pick] = t[rng.integers(0, nt, pick.size)] + 0.05 * rng.standard_normal((pick.size, dim)).astype(np.float32)
    return q, t


class Side:
    def __init__(self, rows: np.ndarray, dev):
        self.rows = torch.from_numpy(np.ascontiguousarray(rows)).to(dev)
        self.count = torch.tensor([rows.shape[0]], dtype=torch.int32, device=dev)
        self.kp = Keypoints(0, 0, 0, rows.shape[0], self.count.data_ptr())
        if rows.dtype == np.float32:
            self.desc = Descriptors(FLOAT32, rows.shape[1], 4 * rows.shape[1], self.rows.data_ptr())
        else:
            self.desc = Descriptors(BINARY_U8, 32, 32, self.rows.data_ptr())


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


@pytest.fixture
def lib():
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)
    L = _abi.load()
    before = L.stitch_s4_matcher()
    yield L
    L.stitch_s4_set_matcher(before)


def run_both(L, q, t, cross, dev):
    """stitch_s4_match (caller workspace) and stitch_s4_match_static on the
    same inputs; returns both host results."""
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    cfg = S4Config()
    cfg.ratio_threshold = 0.8
    cfg.cross_check = 1 if cross else 0
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
    return want.host(), got.host()


def oracle_matches(q, t, cross, l2):
    fwd = c_oracle.top2(q, t, None, None, l2)
    rev = c_oracle.top2(t, q, None, None, l2) if cross else None
    return c_oracle.accept(fwd, rev, 0.8, l2)


@pytest.mark.parametrize("matcher", [0, 1], ids=["popc", "tensor"])
@pytest.mark.parametrize("cross", [False, True])
def test_static_scratch_matches_workspace_entry_point(lib, matcher, cross):
    dev = torch.device("cuda", 0)
    assert lib.stitch_s4_set_matcher(matcher) == 0
    # the larger call first: the second call reuses a scratch that holds its data
    cases = [planted(3000, 2600, 22), planted(1500, 1700, 21)]
    for n, (q, t) in enumerate(cases):
        w, g = run_both(lib, q, t, cross, dev)
        assert w[0].size > 0
        for x, y in zip(w, g):
            assert np.array_equal(x, y)
        if n == 1:   # the oracle on the smaller case
            for x, y in zip(oracle_matches(q, t, cross, False), g):
                assert np.array_equal(x, y)


@pytest.mark.parametrize("cross", [False, True])
def test_static_scratch_float32_after_a_larger_binary_call(lib, cross):
    dev = torch.device("cuda", 0)
    big_q, big_t = planted(4000, 3000, 23)
    w, g = run_both(lib, big_q, big_t, cross, dev)
    for x, y in zip(w, g):
        assert np.array_equal(x, y)
    q, t = floats(300, 420, 24, 24)
    for _ in range(2):   # two calls in a row
        w, g = run_both(lib, q, t, cross, dev)
        assert w[0].size > 0
        for x, y in zip(w, g):
            assert np.array_equal(x, y)
    for x, y in zip(oracle_matches(q, t, cross, True), g):
        assert np.array_equal(x, y)


def test_static_scratch_rejects_oversize_request(lib):
    dev = torch.device("cuda", 0)
    cfg = S4Config()
    cfg.ratio_threshold = 0.8
    cfg.cross_check = 1
    big = 200000   # needs more than the 4 MiB scratch with the mutual check
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    rows = torch.zeros((big, 32), dtype=torch.uint8, device=dev)
    kp = Keypoints(0, 0, 0, big, cnt.data_ptr())
    desc = Descriptors(BINARY_U8, 32, 32, rows.data_ptr())   # a valid request, only too large
    out = Out(big, dev)
    st = lib.stitch_s4_match_static(C.byref(kp), C.byref(desc), C.byref(kp), C.byref(desc), C.byref(cfg),
                                    C.byref(out.m), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _abi.Status.INSUFFICIENT_WORKSPACE
    torch.cuda.synchronize()
    assert int(out.n.item()) == 0x7f7f7f7f

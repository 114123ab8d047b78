"""The C S4 oracle against the reference's own S4 expectations
(tests/test_s4_cuda.cu:60-94 sort-all-distances oracle, :185-245 edge and
tile cases) and against brute force with NumPy."""
import numpy as np
import pytest

from oracle import c_oracle


def brute_top2(a, b, l2=False):
    out = []
    for q in a:
        if l2:
            d = [sum((float(x) - float(y)) ** 2 for x, y in zip(q, t)) for t in b]
        else:
            d = [int(np.unpackbits(np.bitwise_xor(q, t)).sum()) for t in b]
        order = sorted(range(len(b)), key=lambda i: (d[i], i))
        f = (d[order[0]], order[0]) if order else (np.inf, -1)
        s = (d[order[1]], order[1]) if len(order) > 1 else (np.inf, -1)
        out.append((f[0], s[0], f[1], s[1]))
    return out


@pytest.mark.parametrize("dim", [1, 31, 32, 33, 65])
def test_binary_tiles(dim):
    n_a, n_b = 40, 37
    i = np.arange(n_a * dim)
    a = ((i * 73 + i // dim * 19) % 256).astype(np.uint8).reshape(n_a, dim)
    j = np.arange(n_b * dim)
    b = a.reshape(-1)[(j + 3 * dim) % a.size].reshape(n_b, dim)
    got = c_oracle.top2(a, b)
    want = brute_top2(a, b)
    for g, w in zip(got, want):
        assert (g["first_distance"], g["second_distance"], g["first_index"], g["second_index"]) == w


def test_float_l2_and_overflow():
    a = np.array([[-3.4028235e38]], np.float32)
    b = np.array([[3.4028235e38 / 2], [3.4028235e38]], np.float32)
    t = c_oracle.top2(a, b, l2=True)
    ia, ib, d = c_oracle.accept(t, None, 0.9, l2=True)
    assert list(ia) == [0] and np.isinf(d[0])
    e = c_oracle.top2(np.array([[0, 0]], np.float32), np.array([[3, 4], [30, 40]], np.float32), l2=True)
    ia, ib, d = c_oracle.accept(e, None, 0.8, l2=True)
    assert list(ib) == [0] and d[0] == 5


def test_edges_reference_cases():
    u8 = lambda *v: np.array(v, np.uint8).reshape(-1, 1)
    f32 = lambda *v: np.array(v, np.float32).reshape(-1, 1)
    for cross in (False, True):
        def run(a, b, ratio=0.8, ca=None, cb=None, l2=False):
            f = c_oracle.top2(a, b, ca, cb, l2)
            r = c_oracle.top2(b, a, cb, ca, l2) if cross and len(b) else None
            return c_oracle.accept(f, r, ratio, l2)[0]
        assert run(u8(0), u8(0, 0)).size == 0          # two zero distances never pass
        assert run(u8(0), u8(0)).size == 0             # fewer than two neighbours
        assert run(u8(0), u8(1, 2)).size == 0
        assert run(u8(0), u8(1, 3), 0.5).size == 0
        assert run(f32(0), f32(0, 2), np.nextafter(0, 1), l2=True).size == 1
        assert run(u8(0, 1), u8(0, 255), ca=0).size == 0
        assert run(u8(0, 1), u8(0, 255), ca=3).size == 0   # invalid count -> empty
        assert run(u8(0, 1), u8(0, 255), cb=-1).size == 0
    # equal A descriptors compete for B0: the mutual check keeps A0
    f = c_oracle.top2(np.zeros((2, 1), np.float32), np.array([[0], [10]], np.float32), l2=True)
    r = c_oracle.top2(np.array([[0], [10]], np.float32), np.zeros((2, 1), np.float32), l2=True)
    ia, _, _ = c_oracle.accept(f, r, 0.8, l2=True)
    assert list(ia) == [0]


def test_ties_across_tiles():
    train = np.full((260, 1), 20, np.float32)
    train[[3, 129, 258]] = 1
    t = c_oracle.top2(np.zeros((1, 1), np.float32), train, l2=True)[0]
    assert t["first_index"] == 3 and t["second_index"] == 129

"""The tcgen05 kind::i8 matcher (descriptor bits as +-1 int8, Hamming =
(256 - dot) / 2 from tensor-core dot products) against the oracle, on the
same cases as the __popc kernel: edges, ties across train tiles, planted
partners at every shape including 8192 x 8192, counts below capacity, and
the whole batched chain against the per-pair chain run with __popc. Every
train-stage width runs (matcher kinds 1, 2, 3: 256, 128 and 64 train rows
per MMA stage), and the pipelined kernel (kind 4)."""
import numpy as np
import pytest
import torch

from crossstage_stitch_b200 import _abi, batch, stages, synth

from .test_gpu_s4 import check, planted, u8

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[1, 2, 3, 4], ids=["stage256", "stage128", "stage64", "pipelined"])
def tc(cuda, request):
    from .gpu_util import Lib
    lib = Lib("ours")
    L = _abi.load()
    assert L.stitch_s4_set_matcher(request.param) == 0 and L.stitch_s4_matcher() == request.param
    yield lib
    L.stitch_s4_set_matcher(1)
    assert L.stitch_s4_tc_errors() == 0, "an MMA completion wait ran out"


@pytest.mark.parametrize("shape", [(1, 1), (5, 300), (128, 256), (129, 257), (1000, 1000), (2000, 3000),
                                   (300, 20000), (4096, 64)])
@pytest.mark.parametrize("cross", [False, True])
def test_tc_planted_vs_oracle(tc, shape, cross):
    q, t = planted(*shape)
    check(tc, q, t, cross=cross, pad_a=0, pad_b=0)


def test_tc_counts_below_capacity_and_padding(tc):
    q, t = planted(700, 900, seed=3)
    check(tc, q, t, cross=True, ca=650, cb=811, pad_a=16, pad_b=16)


def test_tc_ties_and_extremes(tc):
    # identical rows (distance 0), complements (distance 256) and exact ties
    base = np.random.default_rng(1).integers(0, 256, (1, 32), dtype=np.uint8)
    t = np.concatenate([base ^ 0xff, base, base, base ^ 0x01, base ^ 0xff] * 60)
    q = np.concatenate([base, base ^ 0xff, base ^ 0x01, np.zeros((1, 32), np.uint8)])
    check(tc, q, t, cross=True, pad_a=0, pad_b=0)


def test_tc_full_microbenchmark_size(tc):
    q, t = planted(8192, 8192)
    ia, ib, d = check(tc, q, t, pad_a=0, pad_b=0)
    assert ia.size > 0.2 * 8192


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
def test_tc_batched_chain_equals_popc_per_pair(cuda, kind):
    L = _abi.load()
    cases = []
    for i in range(3):
        p = synth.config0_pair(60 + i)
        cases.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=2000, seed=600 + i, levels=8,
                                                        cross_check=i == 1)))
    runner = stages.PairRunner(512, 512, 2000, cross_check=True)
    assert L.stitch_s4_set_matcher(0) == 0
    want = []
    for a, b, k in cases:
        res = runner.run(a, b, k)
        want.append((res, runner.download()))
    assert L.stitch_s4_set_matcher(kind) == 0
    try:
        imgs = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b, _ in cases]
        bt = batch.Batch([batch.pair_desc(ia, ib, k) for (ia, ib), (_, _, k) in zip(imgs, cases)])
        bt.enqueue()
        torch.cuda.synchronize()
        for i, (res, dl) in enumerate(want):
            got = bt.outputs(i)
            for key in ("idx_a", "idx_b", "distance", "mask"):
                assert np.array_equal(got[key], dl[key]), (i, key)
            np.testing.assert_array_equal(bt.result(i)["H"], res["H"])
        assert L.stitch_s4_tc_errors() == 0
    finally:
        L.stitch_s4_set_matcher(1)

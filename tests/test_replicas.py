"""The N > 1 path on CPU: pairs are independent, so ranks register disjoint
shares with no collective on the data path; the job's time is the slowest
rank's (max over ranks); served requests are placed on the least-loaded GPU.
The world_size-2 case runs as two gloo processes on this host, each running
the oracle chain on its share of small synthetic pairs."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from crossstage_stitch_b200 import replicas

N_PER_RANK = 2


def test_pair_indices_partition():
    got = [list(replicas.pair_indices(5, r)) for r in range(4)]
    flat = [i for g in got for i in g]
    assert flat == list(range(20)) and len(set(flat)) == 20
    with pytest.raises(ValueError):
        replicas.pair_indices(-1, 0)


def test_max_over_ranks_without_a_group():
    assert replicas.max_over_ranks([1.5, 2.0]) == [1.5, 2.0]


def test_least_loaded_dispatcher():
    d = replicas.LeastLoadedDispatcher([100, 100, 60])
    assert d.place("a", 50) == 0          # all free: lowest index
    assert d.place("b", 50) == 1          # GPU 1 now has the most free budget
    assert d.place("c", 10) == 2          # 60 free beats 50, 50
    assert d.place("d", 40) == 0          # 50, 50, 50: lowest index
    assert d.used == [90, 50, 10]
    assert d.place("e", 80) == 1          # GPU 2's budget is too small; GPU 1 has more free than 0
    assert d.place("f", 30) == 2          # 10, -30, 50 free
    assert d.used == [90, 130, 40]
    assert d.release("a") == 0 and d.used == [40, 130, 40]
    with pytest.raises(ValueError):
        d.place("big", 101)               # larger than every budget
    with pytest.raises(ValueError):
        d.place("b", 1)                   # already placed
    with pytest.raises(ValueError):
        replicas.LeastLoadedDispatcher([])


def register(g):
    """Pair g of the registration workload through the CPU oracle chain."""
    from crossstage_stitch_b200 import stages, synth
    from oracle import chain
    p = synth.config0_pair(g)
    res = chain.run_pair(p.gray_a, p.gray_b, stages.Knobs(max_keypoints=300, hypotheses=200, seed=g))
    return g, int(res["status"]), int(res["num_inliers"]), np.asarray(res["H"]).ravel().tolist()


def rank_main(rank, world, port, queue):
    import time

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t0 = time.perf_counter()
        mine = [register(g) for g in replicas.pair_indices(N_PER_RANK, rank)]
        elapsed = time.perf_counter() - t0
        (t_max,) = replicas.max_over_ranks([elapsed])
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            queue.put((t_max, elapsed, gathered))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_register_disjoint_pairs():
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    t_max, t0, gathered = queue.get(timeout=10)
    assert t_max >= t0 > 0
    flat = [r for share in gathered for r in share]
    assert [r[0] for r in flat] == list(range(world * N_PER_RANK))
    # each rank's results equal the single-process run of the same pairs
    for g, status, inliers, h in flat:
        _, status1, inliers1, h1 = register(g)
        assert status == status1 == 0 and inliers == inliers1 > 0
        assert np.array_equal(h, h1)


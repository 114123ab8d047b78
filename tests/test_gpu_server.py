"""The served form: requests of uneven size and knobs, submitted while
others are on the GPU, are admitted under the arena budget, batched
continuously, and each result equals the same pair registered alone by the
plain per-pair path (bit for bit: status, match and inlier counts, H)."""
import time

import numpy as np
import pytest

from crossstage_stitch_b200 import stages, synth
from crossstage_stitch_b200.server import Server

pytestmark = pytest.mark.gpu


def requests():
    out = []
    for i in range(6):
        p = synth.config0_pair(30 + i)
        out.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=1000, seed=300 + i, levels=8)))
    for i in range(4):
        p, kn = synth.mixed_pair(i)
        if p.gray_a.shape[0] > 1100:
            continue
        out.append((p.gray_a, p.gray_b, stages.Knobs(max_keypoints=kn["max_keypoints"],
                                                      fast_threshold=kn["fast_threshold"],
                                                      hypotheses=kn["hypotheses"], seed=400 + i, levels=8)))
    p = synth.config0_pair(40)
    out.append((p.gray_a, p.gray_b[:300, :420].copy(), stages.Knobs(max_keypoints=500, seed=7)))  # single level
    rng = np.random.default_rng(4)
    tiny = rng.integers(0, 256, (60, 200), dtype=np.uint8)
    out.append((tiny, tiny.copy(), stages.Knobs(max_keypoints=100, hypotheses=64, seed=2, levels=8)))
    return out


@pytest.fixture(scope="module")
def reqs(cuda):
    return requests()


@pytest.fixture(scope="module")
def alone(reqs):
    W = max(max(a.shape[1], b.shape[1]) for a, b, _ in reqs)
    H = max(max(a.shape[0], b.shape[0]) for a, b, _ in reqs)
    K = max(k.max_keypoints for _, _, k in reqs)
    runner = stages.PairRunner(W, H, K, max_r=8000)
    return [runner.run(a, b, k) for a, b, k in reqs]


def same(got, want):
    assert got["run_status"] == 0
    assert got["status"] == want["status"]
    assert got["num_matches"] == want["num_matches"] and got["num_inliers"] == want["num_inliers"]
    np.testing.assert_array_equal(got["H"], want["H"])
    np.testing.assert_array_equal(got["H_s"], want["H_s"])


def test_results_equal_alone_in_the_mix(reqs, alone):
    srv = Server(arena_bytes=2 << 30, max_batch=8, streams=2)
    got = {}
    order = list(range(len(reqs))) * 2   # every request twice, in two waves
    for n, i in enumerate(order):
        a, b, k = reqs[i]
        assert srv.submit(a, b, k, tag=n) == 0
        if n % 3 == 2:
            time.sleep(0.002)             # let batches start while more arrive
        for r in srv.poll():
            got[r["tag"]] = r
    for r in srv.drain():
        got[r["tag"]] = r
    srv.close()
    assert len(got) == len(order)
    batches = {r["batch_pairs"] for r in got.values()}
    assert max(batches) > 1               # some requests really ran together
    for n, i in enumerate(order):
        same(got[n], alone[i])
        assert got[n]["submit_ms"] <= got[n]["launch_ms"] <= got[n]["done_ms"]


def test_admission_under_a_small_budget(reqs, alone):
    # a 512x512 8-level pair needs about 5 MB: room for two at a time
    srv = Server(arena_bytes=12 << 20, max_batch=64, streams=3)
    for n in range(8):
        a, b, k = reqs[n % 6]
        assert srv.submit(a, b, k, tag=n) == 0
    res = srv.drain()
    srv.close()
    assert len(res) == 8
    assert max(r["batch_pairs"] for r in res) <= 2   # the budget split the work
    for r in res:
        same(r, alone[r["tag"] % 6])


def test_rejections(reqs):
    srv = Server(arena_bytes=2 << 20, max_batch=4, streams=1)
    a, b, k = reqs[0]
    assert srv.submit(a, b, k, tag=1) == 2                     # larger than the whole arena
    bad = stages.Knobs(max_keypoints=100, ratio=1.5)
    assert srv.submit(a[:100, :100].copy(), b[:100, :100].copy(), bad, tag=2) == 1
    assert srv.outstanding() == 0
    srv.close()


def test_rgb_requests_run_s1_on_the_device(cuda):
    """RGB8 requests: the server's S1 + registration equals S1 through the
    stage call followed by the plain per-pair chain with the same ScaleInfo
    (H in original coordinates)."""
    import ctypes as C

    import torch

    from crossstage_stitch_b200 import _abi
    from crossstage_stitch_b200._abi import ImageView, ScaleInfo

    L = _abi.load()
    rng = np.random.default_rng(11)
    cases = []
    for i, scale in enumerate((1.0, 0.5, 0.75)):
        p = synth.config0_pair(50 + i)
        # RGB views whose S1 gray is close to the synthetic gray scene
        noise = rng.integers(-3, 4, p.gray_a.shape + (3,))
        a = np.clip(p.gray_a[..., None].astype(int) + noise, 0, 255).astype(np.uint8)
        b = np.clip(p.gray_b[..., None].astype(int) + noise[::-1], 0, 255).astype(np.uint8)
        cases.append((a, b, scale, stages.Knobs(max_keypoints=800, seed=500 + i, levels=8)))
    srv = Server(arena_bytes=1 << 30, max_batch=8, streams=2)
    for n, (a, b, scale, k) in enumerate(cases):
        assert srv.submit(a, b, k, tag=n, s1_scale=scale) == 0
    got = {r["tag"]: r for r in srv.drain()}
    srv.close()
    runner = stages.PairRunner(512, 512, 800)
    for n, (a, b, scale, k) in enumerate(cases):
        h, w, _ = a.shape
        ta = torch.from_numpy(a.reshape(h, 3 * w)).cuda()
        tb = torch.from_numpy(b.reshape(h, 3 * w)).cuda()
        si_a, si_b = ScaleInfo(), ScaleInfo()
        assert L.stitch_make_scale_info(w, h, scale, C.byref(si_a)) == 0
        assert L.stitch_make_scale_info(w, h, scale, C.byref(si_b)) == 0
        ga = torch.zeros((si_a.work_h, si_a.work_w), dtype=torch.uint8, device="cuda")
        gb = torch.zeros((si_b.work_h, si_b.work_w), dtype=torch.uint8, device="cuda")
        va, vb = ImageView(ta.data_ptr(), w, h, ta.stride(0), 0), ImageView(tb.data_ptr(), w, h, tb.stride(0), 0)
        oa = ImageView(ga.data_ptr(), si_a.work_w, si_a.work_h, ga.stride(0), 1)
        ob = ImageView(gb.data_ptr(), si_b.work_w, si_b.work_h, gb.stride(0), 1)
        s2a, s2b = ScaleInfo(), ScaleInfo()
        assert L.stitch_s1_preprocess(C.byref(va), C.byref(vb), scale, C.byref(oa), C.byref(ob), C.byref(s2a),
                                      C.byref(s2b), None) == 0
        torch.cuda.synchronize()
        runner.enqueue(si_a.work_w, si_a.work_h, si_b.work_w, si_b.work_h, k, scale_a=si_a, scale_b=si_b,
                       images=(ga, gb))
        torch.cuda.synchronize()
        want = stages.result_dict(runner.result)
        same(got[n], want)


def test_retry_extends_the_saved_search(cuda):
    """R escalation without resampling: a request retried from R = 24 to
    R = 2000 on its resident state gives the result of a fresh R = 2000 run;
    a request that passes its bar keeps its first result."""
    from dataclasses import replace
    p = synth.config0_pair(70)
    base = stages.Knobs(max_keypoints=1000, hypotheses=24, seed=77, levels=8)
    srv = Server(arena_bytes=1 << 30, max_batch=8, streams=2)
    assert srv.submit(p.gray_a, p.gray_b, base, tag=0, retry_hypotheses=2000, retry_min_inliers=10 ** 9) == 0
    assert srv.submit(p.gray_a, p.gray_b, base, tag=1, retry_hypotheses=2000, retry_min_inliers=0) == 0
    assert srv.submit(p.gray_a, p.gray_b, replace(base, seed=78), tag=2) == 0
    got = {r["tag"]: r for r in srv.drain()}
    srv.close()
    runner = stages.PairRunner(512, 512, 1000, max_r=2000)
    full = runner.run(p.gray_a, p.gray_b, replace(base, hypotheses=2000))
    short = runner.run(p.gray_a, p.gray_b, base)
    other = runner.run(p.gray_a, p.gray_b, replace(base, seed=78))
    assert got[0]["attempts"] == 2 and got[1]["attempts"] == 1 and got[2]["attempts"] == 1
    same(got[0], full)
    same(got[1], short)
    same(got[2], other)


def test_rgb_requests_render_their_panorama(cuda):
    """S6 in the served form: the panorama and mask of each RGB request equal
    the feather render of its original images under the returned H (the
    stage call on the same GPU, and the oracle bit for bit); a canvas above
    the request's capacity reports INSUFFICIENT_WORKSPACE with the
    registration result intact; a GRAY8 request cannot ask for one."""
    import torch

    from crossstage_stitch_b200 import render
    from oracle import c_oracle

    rng = np.random.default_rng(21)
    cases = []
    for i, scale in enumerate((1.0, 0.5)):
        p = synth.config0_pair(80 + i)
        noise = rng.integers(-3, 4, p.gray_a.shape + (3,))
        a = np.clip(p.gray_a[..., None].astype(int) + noise, 0, 255).astype(np.uint8)
        b = np.clip(p.gray_b[..., None].astype(int) + noise[::-1], 0, 255).astype(np.uint8)
        cases.append((a, b, scale, stages.Knobs(max_keypoints=800, seed=800 + i, levels=8)))
    srv = Server(arena_bytes=1 << 30, max_batch=8, streams=2)
    for n, (a, b, scale, k) in enumerate(cases):
        assert srv.submit(a, b, k, tag=n, s1_scale=scale, panorama_capacity=4 << 20) == 0
    a, b, scale, k = cases[0]
    assert srv.submit(a, b, k, tag=10, s1_scale=scale, panorama_capacity=1000) == 0  # too small a canvas
    assert srv.submit(a, b, k, tag=11, s1_scale=scale) == 0                           # no panorama
    gray = synth.config0_pair(80)
    assert srv.submit(gray.gray_a, gray.gray_b, k, tag=12, panorama_capacity=1 << 20) != 0
    got = {r["tag"]: r for r in srv.drain()}
    srv.close()
    for n, (a, b, scale, k) in enumerate(cases):
        r = got[n]
        assert r["status"] == 0 and r["render_status"] == 0
        H = r["H"]
        g = render.prepare_geometry(a.shape[1], a.shape[0], b.shape[1], b.shape[0], H)
        assert r["canvas"] == (g.width, g.height) and r["origin"] == (g.origin_x, g.origin_y)
        stats = torch.zeros(2, dtype=torch.int64, device="cuda")
        pano, mask = render.render(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), g, statistics=stats)
        torch.cuda.synchronize()
        assert np.array_equal(r["panorama"], pano.cpu().numpy()) and np.array_equal(r["mask"], mask.cpu().numpy())
        assert [r["union_pixels"], r["overlap_pixels"]] == stats.tolist()
        st, og = c_oracle.s6_geometry(a.shape[1], a.shape[0], b.shape[1], b.shape[0], H)
        opano, omask, ostats = c_oracle.s6_feather(a, b, og)
        assert st == 0 and np.array_equal(r["panorama"], opano) and np.array_equal(r["mask"], omask)
        assert (r["union_pixels"], r["overlap_pixels"]) == ostats
    assert got[10]["status"] == 0 and got[10]["render_status"] == 2
    np.testing.assert_array_equal(got[10]["H"], got[0]["H"])
    assert got[11]["render_status"] == -1 and "panorama" not in got[11]
    np.testing.assert_array_equal(got[11]["H"], got[0]["H"])


def test_multi_server_places_and_returns(reqs, alone):
    """The multi-GPU served form on the GPUs this host has (one here):
    requests placed by the least-loaded dispatcher come back with their GPU
    index and the results of the plain per-pair path."""
    import torch

    from crossstage_stitch_b200.server import MultiServer

    devices = list(range(torch.cuda.device_count()))
    ms = MultiServer(devices, arena_bytes=1 << 30, max_batch=8, streams=2)
    for n, (a, b, k) in enumerate(reqs):
        assert ms.submit(a, b, k, tag=n) == 0
    got = {r["tag"]: r for r in ms.drain()}
    ms.close()
    assert sorted(got) == list(range(len(reqs)))
    assert ms.dispatch.used == [0] * len(devices) and not ms.dispatch.placed
    for n, want in enumerate(alone):
        assert got[n]["gpu"] in range(len(devices))
        same(got[n], want)

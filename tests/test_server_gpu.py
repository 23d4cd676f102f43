"""Build server (lvbh_server_*): continuous batching under an HBM budget.

Each request's result must be the same, word for word, built in the mix of a busy server as
built alone with lvbh_build_soup: Morton keys, permutation, parent links, every BVHNode and
triangle word, and the quantisation box.  Requests are device or pinned-host soups, with and
without MODEL_BOUNDS; a request with a non-finite vertex fails alone.
"""
import threading
import time

import numpy as np
import pytest

from test_parity_gpu import assert_same

pytestmark = pytest.mark.gpu


def request_soups(count, seed, lo=1024, hi=200_000):
    from lvbh import scenes
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count))).astype(int)
    return [scenes.clustered_soup(int(n), seed=seed * 7919 + i) for i, n in enumerate(sizes)]


def result_np(res):
    return {"nodes": res.nodes.cpu().numpy().view(np.uint32), "tris": res.tris.cpu().numpy(),
            "parents": res.parents.cpu().numpy(), "leaf_index": res.leaf_index.cpu().numpy().view(np.uint32),
            "morton": res.morton.cpu().numpy().view(np.uint32), "bounds": res.bounds}


def alone(builder, tri, bounds):
    import torch
    return builder.build_soup(torch.from_numpy(tri).cuda(), bounds).to_numpy()


def bounds_for(tri, i):
    if i % 3:
        return None
    v = np.concatenate([tri[:, 0:3], tri[:, 4:7], tri[:, 8:11]])
    return np.concatenate([v.min(0) - 0.01, v.max(0) + 0.02]).astype(np.float32)


def test_server_same_alone_and_in_mix(builder):
    import torch
    from lvbh.server import Server
    soups = request_soups(48, seed=1)
    srv = Server(0, hbm_budget=6 << 30, slots=3, max_batch_tris=1 << 21, max_batch_reqs=64)
    try:
        tickets = []
        for i, tri in enumerate(soups):
            src = torch.from_numpy(tri).cuda() if i % 2 else torch.from_numpy(tri).pin_memory()
            tickets.append(srv.submit(src, bounds_for(tri, i)))
            if i % 8 == 7:
                time.sleep(0.002)  # let some arrive while others are on the GPU
        for i, t in enumerate(tickets):
            res, info = srv.wait(t)
            assert info["status"] == 0 and info["num_tris"] == soups[i].shape[0]
            got = result_np(res)
            ref = alone(builder, soups[i], bounds_for(soups[i], i))
            assert_same(got, ref, f"request {i}")
            np.testing.assert_array_equal(got["bounds"].view(np.uint32), ref["bounds"].view(np.uint32))
            srv.release(t)
        st = srv.stats()
        assert st["completed"] == len(soups) and st["failed"] == 0
        assert st["max_batch_seen"] > 1, st  # coalescing happened
        assert st["bytes_in_use"] == 0
    finally:
        srv.close()


def test_server_admission_under_budget(builder):
    """Results of all requests together exceed the result memory: batches wait for releases
    and every request still completes with the right tree."""
    import torch
    from lvbh.server import Server
    from lvbh import scenes
    n = 600_000
    base = scenes.clustered_soup(n, seed=77)
    dev = torch.from_numpy(base).cuda()
    srv = Server(0, hbm_budget=1536 << 20, slots=2, max_batch_tris=1 << 21, max_batch_reqs=16)
    try:
        st0 = srv.stats()
        per_req = 128 * n
        count = int(st0["result_bytes"] // per_req) * 3 + 2  # about three budgets' worth
        sizes = [n - 1000 * k for k in range(count)]
        tickets = [srv.submit(dev[:m]) for m in sizes]
        done = []

        def consumer():
            for t, m in zip(tickets, sizes):
                res, info = srv.wait(t)
                done.append((m, result_np(res), info))
                srv.release(t)

        th = threading.Thread(target=consumer)
        th.start()
        th.join(timeout=300)
        assert not th.is_alive()
        assert len(done) == count
        for m, got, info in done[:: max(1, count // 4)]:
            assert_same(got, alone(builder, base[:m], None), f"prefix {m}")
        st = srv.stats()
        assert st["completed"] == count
        assert st["admission_waits"] > 0
        assert st["peak_bytes"] <= st["result_bytes"]
    finally:
        srv.close()


def test_server_bad_request_fails_alone(builder):
    import lvbh
    import torch
    from lvbh.server import Server
    soups = request_soups(6, seed=4, hi=50_000)
    soups[2] = soups[2].copy()
    soups[2][17, 4] = np.nan
    srv = Server(0, hbm_budget=2 << 30, slots=1, max_batch_tris=1 << 20, max_batch_reqs=16)
    try:
        # hold the single slot with a first request so that the rest coalesce into one batch
        tickets = [srv.submit(torch.from_numpy(t).cuda()) for t in soups]
        for i, t in enumerate(tickets):
            if i == 2:
                with pytest.raises(lvbh.LvbhError) as e:
                    srv.wait(t)
                assert e.value.code == lvbh._native.EINVAL
            else:
                res, _ = srv.wait(t)
                assert_same(result_np(res), alone(builder, soups[i], None), f"request {i}")
            srv.release(t)
        assert srv.stats()["failed"] == 1
    finally:
        srv.close()


def test_server_empty_and_oversize():
    import lvbh
    import torch
    from lvbh.server import Server
    srv = Server(0, hbm_budget=1 << 30, slots=1, max_batch_tris=1 << 16, max_batch_reqs=8)
    try:
        t = srv.submit(torch.zeros((0, 12), dtype=torch.float32, device="cuda"))
        res, info = srv.wait(t)
        assert info["status"] == 0 and res.nodes.shape[0] == 0
        srv.release(t)
        with pytest.raises(lvbh.LvbhError) as e:
            srv.submit(torch.zeros(((1 << 16) + 1, 12), dtype=torch.float32, device="cuda"))
        assert e.value.code == lvbh._native.EINVAL
    finally:
        srv.close()

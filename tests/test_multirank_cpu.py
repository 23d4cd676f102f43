"""bench.py's multi-rank host logic on CPU: two `gloo` ranks on 127.0.0.1.

The build does not shard (a global bounds reduction and a global sort), so N GPUs run N
replicas: every rank times its own builds, the reported time is the slowest rank's and the
reported throughput is all ranks' triangles over that time.  These tests run that plumbing
with world size 2 - process-group set-up from the torchrun environment, the barrier, the
max-over-ranks reduction - and check that the reference arm prints from rank 0 only.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    for p in (REPO, os.path.join(REPO, "webgpu-lvbh-demo_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import bench
    try:
        w, r, local = bench.dist_setup()
        # each rank's per-step time differs; the reported one is the slowest rank's
        ms = bench.max_over_ranks(1.5 * (rank + 1), w)
        bench.barrier(w)
        # the reference arm: rank 0 alone runs and prints, the others return without work
        buf = io.StringIO()

        class Args:
            workload, warmup, steps = "tiny", 3, 1

        if r != 0:
            with redirect_stdout(buf):
                bench.run_reference(Args, w, r)
        q.put((r, w, local, dist.get_backend(), ms, buf.getvalue()))
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put(("error", repr(e)))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_two_gloo_ranks_max_and_reference_arm():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = []
    try:
        for _ in procs:
            results.append(q.get(timeout=120))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(r[0] != "error" for r in results), results
    results.sort()
    assert [r[0] for r in results] == [0, 1]
    for rank, world, local, backend, ms, out in results:
        assert world == 2 and local == rank and backend == "gloo"
        assert ms == pytest.approx(3.0)  # max of 1.5 and 3.0 on both ranks
        assert out == ""                 # rank 1 printed nothing for the reference arm
    assert all(p.exitcode == 0 for p in procs)


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    import bench
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (1, 0, 0)
    assert bench.max_over_ranks(2.5, w) == 2.5
    bench.barrier(w)  # a no-op for one rank

"""The multi-GPU layout of bench.py (replicas: one independent bar per rank,
no data-path collective), exercised on the CPU with two gloo ranks: the
process group, the barrier and the max-over-ranks timing every rank takes in
the same order, and the per-rank bars."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    from taylor_b200 import cases
    r, w, dist = bench.dist_setup(world, backend="gloo")
    try:
        bench.barrier(dist)
        worst = bench.max_over_ranks(10.0 + r, dist)      # each rank's "device time"
        case = cases.taylor_bar(h=1.6e-3, seed=1 + r)     # the replica's own bar, as run_ours seeds it
        q.put((r, w, worst, float(case["coo"][0, 0])))
        bench.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[0] for g in got] == [0, 1] and all(g[1] == 2 for g in got)
    assert all(g[2] == 11.0 for g in got)               # the max over ranks, seen by every rank
    assert got[0][3] != got[1][3]                       # independent replicas (own jitter seed)

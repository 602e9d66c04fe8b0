"""The N>1 path of bench.py on CPU: independent replicas, one process per rank,
timed as the maximum over ranks and counted as the sum (gloo, world size 2).
A single graph does not shard, so this is the only exchange the path has."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    # host ranks on gloo even where a GPU is present
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import bench

    class A:
        impl = "engine"

    w, r, local, pg = bench.dist_setup(A())
    try:
        bench.barrier(pg)
        # rank r "took" 1.5 + r seconds and swept 1000 * (r + 1) edges
        t, e = bench.reduce_max_sum(pg, w, local, 1.5 + r, 1000.0 * (r + 1))
        bench.barrier(pg)
        q.put((r, w, t, e))
    finally:
        pg.destroy_process_group()


def test_replicas_max_time_sum_work():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for r, w, t, e in res:
        assert w == 2
        assert t == 2.5  # slowest rank
        assert e == 3000.0  # all ranks' work

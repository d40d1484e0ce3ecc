"""bench.py --gpus N runs N independent replicas (the path does not shard):
the only cross-rank work is the barrier around the timed region and the
max over ranks of the device times.  Checked here with two gloo ranks on
the CPU."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    r, w, local = bench.dist_env()
    d = bench.Dist(w)
    d.barrier()
    mx = d.max(10.0 * (r + 1))
    d.barrier()
    d.close()
    q.put((r, w, local, mx))


def test_two_gloo_ranks_barrier_and_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    assert codes == [0, 0]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 0, 20.0), (1, 2, 1, 20.0)]


def test_single_rank_needs_no_process_group():
    import bench
    d = bench.Dist(1)
    d.barrier()
    assert d.max(3.5) == 3.5
    d.close()

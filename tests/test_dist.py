"""bench.py's rank helpers on world size 2 with the gloo backend on CPU: the
rendezvous, the barrier and the max-over-ranks reduction that turns per-rank
device times into the job's time (the path itself runs replicas only)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup(None, backend="gloo")
    bench.barrier(pg)
    m = bench.max_over_ranks(pg, 10.0 + r)
    bench.barrier(pg)
    pg.destroy_process_group()
    q.put((r, w, local, m))


def test_rank_helpers_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[3] == 11.0 for o in out)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        w, r, local, pg = bench.dist_setup(None)
        assert (w, r, local, pg) == (1, 0, 0, None)
        assert bench.max_over_ranks(pg, 3.5) == 3.5
    finally:
        os.environ.update(env)

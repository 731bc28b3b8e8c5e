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


def _slab_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from cubismnova_b200 import partition as P
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s = P.ZSlab((2, 2, 5), (4, 4, 4), rank, world)
    # stand-ins for the packed planes: rank-tagged host tensors
    low = torch.full((3, 8, 8, 5), 100.0 * rank + 1)
    high = torch.full((3, 8, 8, 5), 100.0 * rank + 2)
    from_up, from_down = P.exchange_messages(s, low, high)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, s.z0, s.z1, float(from_up[0, 0, 0, 0]), float(from_down[0, 0, 0, 0])))


@pytest.mark.parametrize("world", [2, 3])
def test_slab_ghost_messages_gloo(world):
    """The ghost exchange's messages over gloo: a slab's high ghost layer gets
    the lowest planes of the slab above, its low ghost layer the top planes of
    the slab below (a ring along z; with two ranks both neighbours are the
    same rank and the two messages still land in the right layers)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    out = sorted(q.get(timeout=10) for _ in range(world))
    sys.path.insert(0, ROOT)
    from cubismnova_b200 import partition as P
    layers = P.split_layers(5, world)
    for r, z0, z1, up, down in out:
        assert (z0, z1) == layers[r]
        assert up == 100.0 * ((r + 1) % world) + 1
        assert down == 100.0 * ((r - 1) % world) + 2


def test_split_layers_and_slab_geometry():
    sys.path.insert(0, ROOT)
    from cubismnova_b200 import partition as P
    assert P.split_layers(5, 2) == [(0, 3), (3, 5)]
    assert P.split_layers(4, 3) == [(0, 2), (2, 3), (3, 4)]
    with pytest.raises(ValueError):
        P.split_layers(2, 3)
    s = P.ZSlab((2, 2, 4), (8, 8, 8), 1, 2)
    assert s.nb == (2, 2, 4) and (s.z0, s.z1) == (2, 4) and (s.down, s.up) == (0, 0)
    # the slab's z extent: its 2 layers and one ghost layer each side, same cell size
    assert s.begin[2] == 1 * 8 / 32 and s.end[2] == 5 * 8 / 32
    assert s.global_block(0) == -1 and s.global_block(4) == 8 and s.global_block(11) == 15
    assert s.global_block(12) == -1
    assert s._span("send_low", 3) == ((0, 0, 8), (16, 16, 11))
    assert s._span("recv_high", 3) == ((0, 0, 24), (16, 16, 27))

"""Multi-rank host logic on CPU (gloo, world size 2): max-over-ranks timing and
the replica partition of independent units."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        got = bench.barrier_max(float(rank + 1) * 1.5, ws)
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_barrier_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 3.0


@pytest.mark.parametrize("n,ws", [(64, 8), (7, 2), (3, 4), (1, 1), (0, 3)])
def test_replica_shares_partition(n, ws):
    shares = bench.replica_shares(n, ws)
    assert len(shares) == ws
    flat = [i for s in shares for i in s]
    assert flat == list(range(n))
    sizes = [len(s) for s in shares]
    assert max(sizes) - min(sizes) <= 1


_SMALL_BLOB = dict(name="blob L3", kind="blob", level=3, radius=12.0, nq=40, eps_in=4.0, eps_out=80.0,
                   kappa=0.125, seed=7)


def _workload_worker(rank, ws, port, out):
    """Each rank builds its own seeded system, as bench.py does under torchrun, and all
    ranks gather a digest of every rank's inputs and the max of their sizes."""
    import hashlib

    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        tri, qpos, q = bench.make_workload(_SMALL_BLOB, rank)
        h = hashlib.sha256(tri.tobytes() + qpos.tobytes() + q.tobytes()).digest()[:8]
        mine = torch.tensor([int.from_bytes(h, "little") & 0x7FFFFFFFFFFFFFFF, len(tri)], dtype=torch.int64)
        allv = [torch.zeros(2, dtype=torch.int64) for _ in range(ws)]
        dist.all_gather(allv, mine)
        out[rank] = [tuple(int(x) for x in v) for v in allv]
    finally:
        dist.destroy_process_group()


def test_ranks_solve_distinct_systems_of_one_size():
    """bench.py under torchrun: rank 0 solves the configuration's own system and every
    other rank a different seeded system of the same size (no replicated solves)."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_workload_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert out[0] == out[1]
    (h0, n0), (h1, n1) = out[0]
    assert h0 != h1 and n0 == n1 == 1280
    tri, qpos, q = bench.make_workload(_SMALL_BLOB)
    import hashlib
    h = hashlib.sha256(tri.tobytes() + qpos.tobytes() + q.tobytes()).digest()[:8]
    assert h0 == int.from_bytes(h, "little") & 0x7FFFFFFFFFFFFFFF

"""Multi-rank chain scheduling on CPU ranks (gloo, world size 2): the cyclic task split with energy rotation covers every
task exactly once, and the sum of disjoint shares equals the serial result bit for bit (test/test_mpi.f90:114-121)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from asr_b200 import distributed as D


def test_task_split_covers_every_task_once():
    for world in (1, 2, 3, 4, 8):
        for ntask, ntg in ((54 * 48, 48), (17, 5), (7, 7)):
            seen = np.concatenate([D.rank_tasks(ntask, ntg, world, r) for r in range(world)])
            assert np.array_equal(np.sort(seen), np.arange(ntask))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ngroup, nz = 6, 13

    def compute(q, j):     # stands in for the GPU chains: a deterministic complex value per (group, energy)
        return np.sin(q * 1.7 + j * 0.31) + 1j * np.cos(q * 0.3 - j * 1.1) / (1.0 + q + j)

    gz = D.chain_greens_distributed(ngroup, nz, compute, dist)
    out[rank] = gz.tobytes()
    dist.barrier()
    dist.destroy_process_group()


def test_disjoint_share_sum_is_bitwise_serial():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    ngroup, nz = 6, 13
    q, j = np.meshgrid(np.arange(ngroup), np.arange(nz))
    serial = np.sin(q * 1.7 + j * 0.31) + 1j * np.cos(q * 0.3 - j * 1.1) / (1.0 + q + j)
    for r in range(world):
        gz = np.frombuffer(out[r], dtype=np.complex128).reshape(nz, ngroup)
        assert np.array_equal(gz, serial)


def _dead_rank_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=3))
    if rank == 1:
        return   # a rank that leaves between steps and never joins the collective
    try:
        D.sum_disjoint(np.ones(4, np.complex128), dist)
        out[rank] = "no error"
    except Exception as e:   # the short process-group timeout ends the collective with an error
        out[rank] = type(e).__name__


@pytest.mark.timeout(120)
def test_missing_rank_is_detected_by_timeout():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_dead_rank_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert out.get(0) not in (None, "no error")

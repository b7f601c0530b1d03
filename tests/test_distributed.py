"""Multi-rank paths on CPU ranks (gloo, world size 2), with the oracle and the host-side fraction adjoint as the per-rank
compute:

* chain tasks: the reference's cyclic split with energy rotation (src/asr_class_scf.f90:1095-1097), per energy and in
  energy blocks, covers every task once; real edc chains of each rank's share (the oracle's edc_green_blk) summed as
  disjoint shares (par_sum_z, src/asr_mpi.F90:155-164) equal the serial chains bit for bit (test/test_mpi.f90:114-121);
* KPM: the random vectors split over the ranks and one all-reduce of the weighted moments equal the serial moments;
* adjoint: per-rank sums of fraction gradients over the rank's (chain, energy) lanes, summed by one all-reduce, equal the
  serial sum;
* a rank that never joins ends the others' collective through the process-group timeout.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from asr_b200 import distributed as D

NZ, NBE = 13, 4


def test_task_split_covers_every_task_once():
    for world in (1, 2, 3, 4, 8):
        for ntask, ntg in ((54 * 48, 48), (17, 5), (7, 7)):
            seen = np.concatenate([D.rank_tasks(ntask, ntg, world, r) for r in range(world)])
            assert np.array_equal(np.sort(seen), np.arange(ntask))


def test_block_split_covers_every_lane_once():
    for world in (1, 2, 3, 8):
        for ngroup, nz, nbe in ((54, 192, 32), (6, 13, 4), (5, 7, 0)):
            lanes = [D.rank_lanes(ngroup, nz, nbe, world, r) for r in range(world)]
            flat = np.concatenate([q * nz + j for q, j in lanes])
            assert np.array_equal(np.sort(flat), np.arange(ngroup * nz))


def test_vector_range_partitions_the_vectors():
    for world in (1, 2, 3, 5, 8):
        for nvec in (64, 63, 9):
            rs = [D.vector_range(nvec, world, r) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == nvec
            assert all(rs[k][1] == rs[k + 1][0] for k in range(world - 1))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _chain_setup():
    from asr_b200 import synthetic as S
    from oracle import oracle as O
    from tests import cases as K
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=2, maxrank=1)
    oop = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 2, 1, case["flippable"])
    groups = []
    for cen in (1, 2):
        ed = S.edc_params(S.draw_species(2, 3), cen)
        for l0 in (1, 3, 5):   # one-dimensional under D4h
            groups.append((ed, cen, l0))
    z = np.linspace(-0.7, 0.5, NZ) + 0.03j
    return oop, groups, z


def _oracle_chains(oop, groups, z, q, j):
    """G of the lanes (group q, energy j): the oracle's edc_green_blk per group over that group's energies."""
    out = np.zeros(q.size, np.complex128)
    for gq in np.unique(q):
        ed, cen, l0 = groups[gq]
        sel = np.nonzero(q == gq)[0]
        oop.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        oop.unfreeze()
        oop.freeze_any(1, cen)
        oop.set_start(l0)
        out[sel] = oop.edc_green_blk(ed, z[j[sel]], l0, 16)[0]
    return out


def _kpm_setup():
    from asr_b200 import kpm, synthetic as S
    nbr, spc, bvec, _ = kpm.fcc_supercell(3, [0.66, 0.14, 0.20], -0.10, seed=4, sweeps=2)
    block, block0 = S.sk_blocks(bvec, 4)
    c, d, o, e = S.plain_params(S.draw_species(3, 4))
    return nbr, spc, c, d, o, e, block, block0


def _cf_lanes(golden_path, lanes):
    """Gradient of sum_L w_L G_L(a, b) over the lanes L = (chain, energy) with respect to the chain coefficients, each lane
    through the library's host-side fraction adjoint (asr_cf_adjoint)."""
    import json

    from asr_b200 import _lib
    gold = json.load(open(golden_path))
    ga = np.zeros((2, 24), np.complex128)
    gb = np.zeros((2, 24), np.complex128)
    for c, zj in lanes:
        ch = gold["cr1" if c == 0 else "cr2"]
        a = np.array(ch["re_a"]) + 1j * np.array(ch["im_a"])
        b = np.array(ch["re_b"]) + 1j * np.array(ch["im_b"])
        z0 = complex(*gold["zc1" if c == 0 else "zc2"])
        z = z0 + 0.01 * zj
        w = complex(np.cos(0.3 * zj), np.sin(0.7 * zj))
        ab, bb, g = np.zeros(48), np.zeros(48), np.zeros(2)
        pd = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
        _lib.check(_lib.lib().asr_cf_adjoint(pd(np.ascontiguousarray(a).view(np.float64)),
                                             pd(np.ascontiguousarray(b).view(np.float64)), 24, z.real, z.imag,
                                             _lib.TAILS["hull"], w.real, w.imag, pd(ab), pd(bb), pd(g)))
        ga[c] += ab.view(np.complex128)
        gb[c] += bb.view(np.complex128)
    return np.stack([ga, gb])


def _worker(rank, world, port, out, golden_path):
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    oop, groups, z = _chain_setup()
    for nbe in (0, NBE):
        gz = D.chain_greens_distributed(len(groups), NZ, lambda q, j: _oracle_chains(oop, groups, z, q, j), dist, nbe=nbe)
        out[(rank, "chains", nbe)] = gz.tobytes()
    nbr, spc, c, d, o, e, block, block0 = _kpm_setup()
    mu = D.kpm_moments_distributed(
        16, lambda v0, n: O.kpm_moments(nbr, spc, c, d, o, e, block, block0, 0.0, 3.0, 24, v0, n, 11), dist)
    out[(rank, "kpm")] = mu.tobytes()
    lanes = [(ch, zj) for ch in (0, 1) for zj in range(10)]
    mine = [lanes[k] for k in range(len(lanes)) if k % world == rank]
    out[(rank, "grad")] = D.gradient_sum(_cf_lanes(golden_path, mine), dist).tobytes()
    dist.barrier()
    dist.destroy_process_group()


def test_world2_chains_kpm_and_gradients_equal_serial():
    from oracle import oracle as O
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "terminators.json")
    mp.spawn(_worker, args=(world, port, out, golden), nprocs=world, join=True)
    # serial: every lane on one process
    oop, groups, z = _chain_setup()
    q, j = np.meshgrid(np.arange(len(groups)), np.arange(NZ))
    serial = _oracle_chains(oop, groups, z, q.ravel(), j.ravel()).reshape(NZ, len(groups))
    nbr, spc, c, d, o, e, block, block0 = _kpm_setup()
    mu_serial = O.kpm_moments(nbr, spc, c, d, o, e, block, block0, 0.0, 3.0, 24, 0, 16, 11)
    lanes = [(ch, zj) for ch in (0, 1) for zj in range(10)]
    grad_serial = _cf_lanes(golden, lanes)
    for r in range(world):
        for nbe in (0, NBE):
            gz = np.frombuffer(out[(r, "chains", nbe)], dtype=np.complex128).reshape(NZ, len(groups))
            assert np.array_equal(gz, serial)
        mu = np.frombuffer(out[(r, "kpm")], dtype=np.float64)
        assert np.max(np.abs(mu - mu_serial)) <= 1e-12 * np.max(np.abs(mu_serial))
        gr = np.frombuffer(out[(r, "grad")], dtype=np.complex128).reshape(grad_serial.shape)
        assert np.max(np.abs(gr - grad_serial)) <= 1e-13 * np.max(np.abs(grad_serial))


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

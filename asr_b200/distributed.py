"""Chain tasks, KPM vectors and adjoint gradients over several GPUs, one process per GPU (torch.distributed over NCCL;
gloo for CPU tests).

The reference splits the chain tasks of ``chain_greens`` cyclically over MPI ranks with an energy rotation,
``mod(t - 1 + (t - 1) / ntg, nr) == rk`` (src/asr_class_scf.f90:1095-1097), where a task is one energy (nbe = 0) or one
block of nbe energies (ntg tasks per group), and sums the disjoint shares of the Green function array with one Allreduce
(``par_sum_z``, src/asr_mpi.F90:155-164; src/asr_class_scf.f90:1043-1051).  Every entry is non-zero on exactly one rank,
so the sum is bitwise the same on every rank in any order (test/test_mpi.f90:114-121).  Each GPU holds its own copy of
the operator (tens of MB), so there are no remote loads; the exchange is that sum.  The KPM moments are averages over
random vectors: each rank takes a contiguous range of the vectors and one all-reduce sums the weighted moments.  The
adjoint's parameter gradient is a sum over the chains, so each rank's partial gradient is summed by one all-reduce.
"""
from __future__ import annotations

import numpy as np


def rank_tasks(ntask: int, ntg: int, world: int, rank: int) -> np.ndarray:
    """0-based task indices of this rank: task t (1-based) belongs to rank mod(t - 1 + (t - 1) / ntg, world)."""
    t = np.arange(ntask)
    return t[(t + t // ntg) % world == rank]


def task_lanes(tasks: np.ndarray, nz: int):
    """Task t = (group q, energy j) with the energy fastest (t = q nz + j): the (group, energy) pairs of the tasks."""
    return tasks // nz, tasks % nz


def rank_lanes(ngroup: int, nz: int, nbe: int, world: int, rank: int):
    """(group, energy) pairs (0-based) of this rank's tasks: nbe = 0, one energy per task; nbe > 0, blocks of nbe
    consecutive energies per task (the last block of a group may be shorter), blocks fastest within a group, as the
    reference numbers them (jb fastest, then start orbital, component and spin, src/asr_class_scf.f90:1098-1108)."""
    if nbe <= 0:
        q, j = task_lanes(rank_tasks(ngroup * nz, nz, world, rank), nz)
        return q, j
    nbk = (nz + nbe - 1) // nbe
    tasks = rank_tasks(ngroup * nbk, nbk, world, rank)
    qs, js = [], []
    for t in tasks:
        q, jb = divmod(int(t), nbk)
        j = np.arange(jb * nbe, min(nz, (jb + 1) * nbe))
        qs.append(np.full(j.size, q))
        js.append(j)
    if not qs:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    return np.concatenate(qs), np.concatenate(js)


def sum_disjoint(gz_local: np.ndarray, dist, device=None) -> np.ndarray:
    """``par_sum_z``: all-reduce (sum) of disjoint complex shares; exact because each entry has one non-zero term."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(gz_local).view(np.float64).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy().view(np.complex128).reshape(gz_local.shape)


def chain_greens_distributed(ngroup: int, nz: int, compute, dist, device=None, nbe: int = 0) -> np.ndarray:
    """gz (nz, ngroup): this rank computes its tasks through ``compute(groups, energies) -> values`` (one complex value
    per (group, energy) lane; on a GPU ``chains_run_lanes``), the shares are summed over the ranks."""
    world, rank = dist.get_world_size(), dist.get_rank()
    q, j = rank_lanes(ngroup, nz, nbe, world, rank)
    gz = np.zeros((nz, ngroup), np.complex128)
    if q.size:
        gz[j, q] = compute(q, j)
    return sum_disjoint(gz, dist, device)


def vector_range(nvec: int, world: int, rank: int):
    """Contiguous range [v0, v1) of the random vectors of this rank (sizes differ by at most one)."""
    base, extra = divmod(nvec, world)
    v0 = rank * base + min(rank, extra)
    return v0, v0 + base + (1 if rank < extra else 0)


def kpm_moments_distributed(nvec: int, moments, dist, device=None) -> np.ndarray:
    """KPM moments averaged over nvec random vectors split over the ranks: ``moments(v0, n)`` returns the average over
    the vectors v0 .. v0 + n - 1 of this rank (``Supercell.kpm_moments`` with v0); the ranks' averages weighted by their
    vector counts are summed by one all-reduce."""
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    v0, v1 = vector_range(nvec, world, rank)
    local = np.asarray(moments(v0, v1 - v0), np.float64) * ((v1 - v0) / nvec) if v1 > v0 else None
    if local is None:
        raise ValueError("kpm_moments_distributed: more ranks than random vectors")
    t = torch.from_numpy(np.ascontiguousarray(local).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def gradient_sum(grad_local: np.ndarray, dist, device=None) -> np.ndarray:
    """The adjoint's parameter gradient over all ranks: each rank's sum over its own chains, summed by one all-reduce."""
    import torch
    g = np.ascontiguousarray(grad_local)
    cplx = np.iscomplexobj(g)
    t = torch.from_numpy((g.view(np.float64) if cplx else g.astype(np.float64)).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = t.cpu().numpy()
    return out.view(np.complex128).reshape(g.shape) if cplx else out.reshape(g.shape)

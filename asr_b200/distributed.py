"""Chain tasks over several GPUs, one process per GPU (torch.distributed over NCCL; gloo for CPU tests).

The reference splits the chain tasks of ``chain_greens`` cyclically over MPI ranks with an energy rotation,
``mod(t - 1 + (t - 1) / ntg, nr) == rk`` (src/asr_class_scf.f90:1095-1097), and sums the disjoint shares of the Green
function array with one Allreduce (``par_sum_z``, src/asr_mpi.F90:155-164; src/asr_class_scf.f90:1043-1051).  Every entry
is non-zero on exactly one rank, so the sum is bitwise the same on every rank in any order (test/test_mpi.f90:114-121).
Each GPU holds its own copy of the operator (tens of MB), so there are no remote loads; the only exchange is that sum.
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


def sum_disjoint(gz_local: np.ndarray, dist, device=None) -> np.ndarray:
    """``par_sum_z``: all-reduce (sum) of disjoint complex shares; exact because each entry has one non-zero term."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(gz_local).view(np.float64).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy().view(np.complex128).reshape(gz_local.shape)


def chain_greens_distributed(ngroup: int, nz: int, compute, dist, device=None) -> np.ndarray:
    """gz (nz, ngroup): this rank computes its tasks through ``compute(groups, energies) -> values`` (one complex value
    per task), the shares are summed over the ranks.  ``compute`` is the GPU chain run in production."""
    world, rank = dist.get_world_size(), dist.get_rank()
    tasks = rank_tasks(ngroup * nz, nz, world, rank)
    q, j = task_lanes(tasks, nz)
    gz = np.zeros((nz, ngroup), np.complex128)
    if tasks.size:
        gz[j, q] = compute(q, j)
    return sum_disjoint(gz, dist, device)

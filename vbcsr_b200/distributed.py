"""Multi-GPU KPM by sharding, one process per GPU (torch.distributed).

The KPM recurrence has no exchange step: every random vector's Chebyshev
sequence is independent, and so is every Hamiltonian of a batch.  So the
work is split across ranks with H replicated and no collective inside the
recurrence; one all-reduce of the moments (M doubles per Hamiltonian) ends
the job.  This is the layout of the reference's random-vector loop
(examples/ex08_graphene_dos.py:66-156, examples/inp_nanocrystal_dos/kpm.py:40-74)
spread over processes instead of over OpenMP threads.

* :func:`column_shard` / :func:`rademacher_columns`: random-vector column c
  is drawn from its own seeded stream, so any split of the columns over
  ranks reproduces exactly the vectors (and the moments) of one process.
* :func:`hamiltonian_shard`: a batch of Hamiltonians split by work (nnz x
  moments), largest first onto the least loaded rank.
* :func:`kpm_moments_sharded` / :func:`batched_kpm_moments_sharded`: run the
  local part with a moment function (the device recurrence by default) and
  all-reduce.
"""
from __future__ import annotations

import numpy as np


def column_shard(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous column range [c0, c1) of `rank` (balanced to within one)."""
    base, extra = divmod(total, world)
    c0 = rank * base + min(rank, extra)
    return c0, c0 + base + (1 if rank < extra else 0)


def rademacher_columns(N: int, c0: int, c1: int, seed: int) -> np.ndarray:
    """+-1 vectors for global columns [c0, c1): column c from the stream
    (seed, c), independent of how columns are split."""
    out = np.empty((N, c1 - c0))
    for j, c in enumerate(range(c0, c1)):
        rng = np.random.default_rng([seed, c])
        out[:, j] = np.where(rng.random(N) < 0.5, -1.0, 1.0)
    return out


def hamiltonian_shard(costs, world: int) -> list[list[int]]:
    """Indices of the Hamiltonians each rank runs: longest-processing-time
    first onto the least loaded rank (deterministic: ties by index)."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def _allreduce_sum(arr: np.ndarray, group=None) -> np.ndarray:
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return arr
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def _device_moments(H, V, M, precision="fp64", two_moment=True):
    """Moments of one (rescaled) BlockCSR H and vectors V on this process's GPU."""
    import ctypes as C

    import torch

    from . import _capi

    dm = _capi.DeviceMatrix.create(H.block_sizes, H.row_ptr, H.col_ind, H.values)
    R = V.shape[1]
    ld = 1 if R == 1 else ((R * 8 + 63) // 64) * 8
    V0 = torch.zeros((H.N, ld), dtype=torch.float64, device="cuda")
    V0[:, :R] = torch.from_numpy(V).cuda()
    mu = torch.zeros(M, dtype=torch.float64, device="cuda")
    _capi.call("vbg_kpm_moments", dm.h, R, ld, C.c_void_p(V0.data_ptr()), int(M), {"fp64": 0, "fp32": 1}[precision],
               int(two_moment), 1, C.c_void_p(mu.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return mu.cpu().numpy()


def kpm_moments_sharded(H, num_moments: int, total_vectors: int, seed: int = 0, group=None, moment_fn=None,
                        precision: str = "fp64") -> np.ndarray:
    """Unnormalised moments sum_r <r|T_n(H)|r> over `total_vectors` Rademacher
    vectors split by column across the ranks of `group` (H already rescaled,
    replicated on every rank); identical to one process running all columns.
    moment_fn(H, V, M) computes the local moments (default: the device
    recurrence)."""
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    c0, c1 = column_shard(total_vectors, world, rank)
    fn = moment_fn or (lambda h, v, m: _device_moments(h, v, m, precision))
    local = fn(H, rademacher_columns(H.N, c0, c1, seed), num_moments) if c1 > c0 else np.zeros(num_moments)
    return _allreduce_sum(np.asarray(local, dtype=np.float64), group)


def batched_kpm_moments_sharded(hamiltonians, num_moments: int, vectors_each: int, seed: int = 0, group=None,
                                moment_fn=None) -> np.ndarray:
    """Moments of every Hamiltonian of a batch, the batch split across ranks
    by work; Hamiltonian i's vectors come from the stream seed + i, so the
    result does not depend on the split.  Returns [count x num_moments]."""
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    costs = [h.nnz for h in hamiltonians]
    mine = hamiltonian_shard(costs, world)[rank]
    out = np.zeros((len(hamiltonians), num_moments))
    fn = moment_fn or _device_moments
    for i in mine:
        h = hamiltonians[i]
        out[i] = fn(h, rademacher_columns(h.N, 0, vectors_each, seed + i), num_moments)
    return _allreduce_sum(out, group)

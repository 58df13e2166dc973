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

A row-partitioned apply (the reference's distributed mult) is the one path
with an exchange: :func:`row_partition`, :func:`halo_plan` (or
:func:`halo_plan_from_global`), :func:`exchange_ghosts` and
:class:`RowPartitionedOperator` below.
"""
from __future__ import annotations

from dataclasses import dataclass, field

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


# --------------------------------------------------- row-partitioned apply
# The reference distributes a matrix by contiguous block rows (sorted owned
# global indices and their displacements, vbcsr/core/dist_graph.hpp:362-470),
# numbers the columns a rank reads but does not own as ghosts after its own
# rows, ordered by owner rank and then global id (dist_graph.hpp:419-436),
# learns who needs which of its rows by an exchange of requests
# (build_comm_pattern, dist_graph.hpp:662-760) and, before each mult, packs
# the requested rows per destination and receives every ghost row straight
# into the ghost region with one all-to-all (DistVector::sync_ghosts,
# dist_vector.hpp:224-266).  Here each rank is one process with one GPU: the
# same plan, the exchange an all_to_all_single on device tensors (NCCL) into
# the ghost rows, and the local product the library's apply on a square
# local matrix of owned + ghost block rows whose ghost rows hold no blocks.


def row_partition(H, world: int) -> list[tuple[int, int]]:
    """Contiguous block-row ranges [r0, r1), one per rank, cut where the
    running count of stored values passes k / world of the total."""
    start = H.slot_offsets()[H.row_ptr]  # value offset at each row start
    total = float(start[-1])
    cuts = [0]
    for k in range(1, world):
        c = int(np.searchsorted(start, total * k / world, side="left"))
        cuts.append(min(max(c, cuts[-1]), H.n))
    cuts.append(H.n)
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


@dataclass
class LocalRows:
    """The block rows [r0, r1) one rank owns; columns are global block ids."""

    r0: int
    r1: int
    block_sizes: np.ndarray  # sizes of the owned rows
    row_ptr: np.ndarray      # local, from 0
    col_ind: np.ndarray      # global block ids
    values: np.ndarray       # slot order, row-major blocks


def local_rows(H, r0: int, r1: int) -> LocalRows:
    """Rows [r0, r1) of a global BlockCSR."""
    off = H.slot_offsets()
    s0, s1 = int(H.row_ptr[r0]), int(H.row_ptr[r1])
    return LocalRows(r0, r1, np.asarray(H.block_sizes[r0:r1], np.int32),
                     np.asarray(H.row_ptr[r0:r1 + 1] - s0, np.int64), np.asarray(H.col_ind[s0:s1], np.int64),
                     H.values[off[s0]:off[s1]])


@dataclass
class HaloPlan:
    """One rank's view of a row-partitioned matrix and its ghost exchange.

    Local block ids: owned rows 0 .. n_owned - 1 (global r0 + i), then the
    ghosts in `ghosts` order (owner rank, then global id).  `send_rows` are
    the scalar rows of this rank's owned X that it packs, grouped by
    destination rank in the order that rank's ghosts expect them;
    `send_counts` / `recv_counts` are scalar rows per peer rank."""

    rank: int
    world: int
    displs: np.ndarray        # first global block row of each rank, world + 1
    ghosts: np.ndarray        # global block ids
    block_sizes: np.ndarray   # owned, then ghosts
    row_ptr: np.ndarray       # owned rows
    col_ind: np.ndarray       # local block ids
    send_rows: np.ndarray
    send_counts: list = field(default_factory=list)
    recv_counts: list = field(default_factory=list)
    slot_perm: np.ndarray = None  # local slot s holds the owned rows' original slot slot_perm[s]

    @property
    def n_owned(self) -> int:
        return int(self.displs[self.rank + 1] - self.displs[self.rank])

    @property
    def N_owned(self) -> int:
        return int(np.sum(self.block_sizes[:self.n_owned]))

    @property
    def N_local(self) -> int:
        return int(np.sum(self.block_sizes))

    def local_values(self, values):
        """The owned rows' values (their original slot order, columns
        ascending by global id) in the local slot order (columns ascending
        by local id)."""
        values = np.asarray(values)
        n0 = self.n_owned
        rows = np.repeat(np.arange(n0), np.diff(self.row_ptr))
        bsz = np.asarray(self.block_sizes, np.int64)
        sizes = np.empty(len(self.slot_perm), np.int64)
        sizes[self.slot_perm] = bsz[rows] * bsz[self.col_ind]  # sizes in the original order
        off = np.zeros(len(sizes) + 1, np.int64)
        np.cumsum(sizes, out=off[1:])
        lens = sizes[self.slot_perm]
        starts = off[self.slot_perm]
        if lens.sum() == 0:
            return values[:0].copy()
        first = np.concatenate([[0], np.cumsum(lens)[:-1]])
        idx = np.repeat(starts - first, lens) + np.arange(lens.sum())
        return values[idx]

    def local_matrix(self, values):
        """The square local matrix (owned + ghost block rows, ghost rows
        empty) as a BlockCSR; `values` in the owned rows' original slot
        order."""
        from .workloads import BlockCSR

        rp = np.concatenate([self.row_ptr, np.full(len(self.ghosts), self.row_ptr[-1])]).astype(np.int32)
        return BlockCSR(np.asarray(self.block_sizes, np.int32), rp, np.asarray(self.col_ind, np.int32),
                        self.local_values(values))

    def same_as(self, other: "HaloPlan") -> bool:
        return (self.rank == other.rank and self.world == other.world and np.array_equal(self.displs, other.displs)
                and np.array_equal(self.ghosts, other.ghosts)
                and np.array_equal(self.block_sizes, other.block_sizes)
                and np.array_equal(self.row_ptr, other.row_ptr) and np.array_equal(self.col_ind, other.col_ind)
                and np.array_equal(self.send_rows, other.send_rows)
                and np.array_equal(self.slot_perm, other.slot_perm)
                and list(self.send_counts) == list(other.send_counts)
                and list(self.recv_counts) == list(other.recv_counts))


def _owner(displs: np.ndarray, gids: np.ndarray) -> np.ndarray:
    return np.searchsorted(displs, gids, side="right") - 1


def _finish_plan(rank, world, displs, loc: LocalRows, ghosts, ghost_sizes, requested):
    """Local numbering, columns remapped, pack list; `requested[d]` are the
    global ids rank d asked this rank for (in d's ghost order)."""
    n_owned = loc.r1 - loc.r0
    bsz = np.concatenate([np.asarray(loc.block_sizes, np.int64), np.asarray(ghost_sizes, np.int64)])
    # global -> local ids: owned by offset, ghosts by position (sorted ids)
    cols = np.asarray(loc.col_ind, np.int64)
    own = (cols >= loc.r0) & (cols < loc.r1)
    local = np.empty_like(cols)
    local[own] = cols[own] - loc.r0
    local[~own] = n_owned + np.searchsorted(ghosts, cols[~own])
    so = np.zeros(n_owned + 1, np.int64)
    np.cumsum(loc.block_sizes, out=so[1:])
    send, send_counts = [], []
    for d in range(world):
        ids = np.asarray(requested[d], np.int64) - loc.r0
        rows = [np.arange(so[i], so[i + 1]) for i in ids]
        send.extend(rows)
        send_counts.append(int(sum(len(r) for r in rows)))
    gown = _owner(displs, ghosts) if len(ghosts) else np.zeros(0, np.int64)
    recv_counts = [int(np.sum(np.asarray(ghost_sizes)[gown == r])) for r in range(world)]
    send_rows = np.concatenate(send).astype(np.int64) if send else np.zeros(0, np.int64)
    # local columns ascending within each row (ghosts owned by lower ranks
    # move behind the owned columns)
    rows = np.repeat(np.arange(n_owned), np.diff(np.asarray(loc.row_ptr, np.int64)))
    perm = np.lexsort((local, rows))
    return HaloPlan(rank, world, np.asarray(displs, np.int64), np.asarray(ghosts, np.int64), bsz.astype(np.int32),
                    np.asarray(loc.row_ptr, np.int64), local[perm], send_rows, send_counts, recv_counts, perm)


def _ghost_ids(loc: LocalRows) -> np.ndarray:
    """Columns read but not owned, ascending: with contiguous owned ranges in
    rank order this is the order (owner rank, global id)."""
    cols = np.asarray(loc.col_ind, np.int64)
    return np.unique(cols[(cols < loc.r0) | (cols >= loc.r1)])


def halo_plan_from_global(H, parts: list[tuple[int, int]], rank: int) -> HaloPlan:
    """The plan of `rank` computed from the whole matrix (no communication):
    what every rank needs is read off its rows directly."""
    world = len(parts)
    displs = np.array([p[0] for p in parts] + [parts[-1][1]], np.int64)
    locs = [local_rows(H, *p) for p in parts]
    ghosts = [_ghost_ids(l) for l in locs]
    mine = locs[rank]
    requested = []
    for d in range(world):
        g = ghosts[d]
        requested.append(g[_owner(displs, g) == rank] if len(g) else g)
    gs = np.asarray(H.block_sizes, np.int64)[ghosts[rank]]
    return _finish_plan(rank, world, displs, mine, ghosts[rank], gs, requested)


def _a2a(send: np.ndarray, send_counts, recv_counts, group, dtype=np.int64) -> np.ndarray:
    """all_to_all_single of a 1-D array (CPU tensors for gloo, CUDA for NCCL)."""
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    src = torch.from_numpy(np.ascontiguousarray(send, dtype=dtype)).to(dev)
    out = torch.empty(int(sum(recv_counts)), dtype=src.dtype, device=dev)
    dist.all_to_all_single(out, src, [int(c) for c in recv_counts], [int(c) for c in send_counts], group=group)
    return out.cpu().numpy()


def halo_plan(loc: LocalRows, group=None) -> HaloPlan:
    """The plan built the way the reference builds its communication
    pattern: the owned ranges are gathered, every rank sends each owner the
    ids of the ghosts it owns (counts first, then the ids), and the owners
    answer with the ghosts' block sizes.  Collective over `group`."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    mine = torch.tensor([loc.r0, loc.r1], dtype=torch.int64, device=dev)
    allr = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(allr, mine, group=group)
    ranges = [tuple(int(v) for v in t.cpu()) for t in allr]
    if any(ranges[k][1] != ranges[k + 1][0] for k in range(world - 1)) or ranges[0][0] != 0:
        raise ValueError("ranks must own contiguous block-row ranges in rank order")
    displs = np.array([r[0] for r in ranges] + [ranges[-1][1]], np.int64)
    ghosts = _ghost_ids(loc)
    gown = _owner(displs, ghosts) if len(ghosts) else np.zeros(0, np.int64)
    req_counts = np.bincount(gown, minlength=world).astype(np.int64)
    in_counts = _a2a(req_counts, [1] * world, [1] * world, group)
    requested_flat = _a2a(ghosts, req_counts, in_counts, group)
    cuts = np.concatenate([[0], np.cumsum(in_counts)])
    requested = [requested_flat[cuts[d]:cuts[d + 1]] for d in range(world)]
    if any(((q < loc.r0) | (q >= loc.r1)).any() for q in requested):
        raise RuntimeError("a rank requested a block row this rank does not own")
    # the owners answer with the block sizes of the requested rows
    sizes_out = np.asarray(loc.block_sizes, np.int64)[requested_flat - loc.r0] if len(requested_flat) \
        else np.zeros(0, np.int64)
    ghost_sizes = _a2a(sizes_out, in_counts, req_counts, group)
    return _finish_plan(rank, world, displs, loc, ghosts, ghost_sizes, requested)


def exchange_ghosts(xl, plan: HaloPlan, group=None) -> None:
    """Fills the ghost rows of the local X (a tensor of N_local rows, on the
    process group's device) from their owners: the rows other ranks need
    are packed in `send_rows` order and one all_to_all_single writes every
    received row straight into the ghost region (rows N_owned ..), as
    DistVector::sync_ghosts does (dist_vector.hpp:224-266)."""
    import torch
    import torch.distributed as dist

    if plan.world == 1:
        return
    idx = torch.from_numpy(plan.send_rows).to(xl.device)
    send = xl.index_select(0, idx)
    recv = xl[plan.N_owned:]
    if xl.is_complex():
        send = torch.view_as_real(send)
        recv = torch.view_as_real(recv)
    dist.all_to_all_single(recv, send, list(plan.recv_counts), list(plan.send_counts), group=group)


class RowPartitionedOperator:
    """y = A x for one rank's block rows of a row-partitioned matrix on this
    process's GPU: the ghost exchange (:func:`exchange_ghosts`, NCCL), then
    the library's apply on the local matrix.  x and y are this rank's owned
    rows (device tensors, vectors or [rows x k] multivectors)."""

    def __init__(self, plan: HaloPlan, values, group=None):
        import torch

        from . import _capi

        self.plan = plan
        self.group = group
        L = plan.local_matrix(values)
        self.dtype = torch.complex128 if np.iscomplexobj(L.values) else torch.float64
        self.dm = _capi.DeviceMatrix.create(L.block_sizes, L.row_ptr, L.col_ind, L.values, dtype=L.values.dtype)
        self._bufs = {}

    def _buffers(self, k):
        import torch

        if k not in self._bufs:
            es = 16 if self.dtype == torch.complex128 else 8
            ld = 1 if k == 1 else ((k * es + 15) // 16 * 16) // es
            shape = (self.plan.N_local,) if k == 1 else (self.plan.N_local, ld)
            self._bufs[k] = (torch.zeros(shape, dtype=self.dtype, device="cuda"),
                             torch.zeros(shape, dtype=self.dtype, device="cuda"), ld)
        return self._bufs[k]

    def mult(self, x, ghosts=None):
        """y (owned rows) = A x.  `ghosts` (the ghost rows of x) skips the
        exchange: the caller already has them."""
        import ctypes as C

        import torch

        from . import _capi

        k = 1 if x.dim() == 1 else int(x.shape[1])
        xl, yl, ld = self._buffers(k)
        n0 = self.plan.N_owned
        if k == 1:
            xl[:n0].copy_(x)
        else:
            xl[:n0, :k].copy_(x)
        if ghosts is not None:
            if k == 1:
                xl[n0:].copy_(ghosts)
            else:
                xl[n0:, :k].copy_(ghosts)
        else:
            exchange_ghosts(xl, self.plan, self.group)
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        vp = C.c_void_p
        if k == 1:
            _capi.call("vbg_spmv", self.dm.h, vp(xl.data_ptr()), vp(yl.data_ptr()), s)
            return yl[:n0].clone()
        _capi.call("vbg_spmm", self.dm.h, k, ld, vp(xl.data_ptr()), vp(yl.data_ptr()), s)
        return yl[:n0, :k].clone()

"""Seeded synthetic block-sparse workloads (host side, numpy).

Each generator returns a :class:`BlockCSR`: block sizes, row pointers, sorted
global block columns and the values in slot order (row-major blocks), i.e.
exactly what ``vbg_matrix_create`` and the reference's construct_serial +
add_block path consume.

* :func:`random_symmetric_blocks` -- random symmetric variable-block pattern
  (diagonal plus mirrored random neighbours), values U[-1, 1] symmetrised.
* :func:`tmd_lattice` -- tight-binding Hamiltonian of a TMD-like triangular
  lattice (one 5-orbital metal site and two 3-orbital chalcogen sites per
  cell), rescaled into [-0.95, 0.95] by its Gershgorin bound.
* :func:`banded_decaying` -- banded, exponentially decaying symmetric matrix
  whose spectrum maps into McWeeny's basin after scale/shift.
* :func:`ring_blocks` -- the ring test matrix of the reference's SpGEMM tests.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class BlockCSR:
    block_sizes: np.ndarray  # int32 [n]
    row_ptr: np.ndarray  # int32 [n+1]
    col_ind: np.ndarray  # int32 [nnzb]
    values: np.ndarray  # float64/complex128 [nnz], slot order, row-major blocks

    @property
    def n(self) -> int:
        return len(self.block_sizes)

    @property
    def nnzb(self) -> int:
        return len(self.col_ind)

    @property
    def nnz(self) -> int:
        return len(self.values)

    @property
    def N(self) -> int:
        return int(np.sum(self.block_sizes))

    def slot_offsets(self) -> np.ndarray:
        rows = np.repeat(np.arange(self.n), np.diff(self.row_ptr))
        sizes = self.block_sizes[rows].astype(np.int64) * self.block_sizes[self.col_ind].astype(np.int64)
        off = np.zeros(self.nnzb + 1, np.int64)
        np.cumsum(sizes, out=off[1:])
        return off

    def to_dense(self) -> np.ndarray:
        so = np.zeros(self.n + 1, np.int64)
        np.cumsum(self.block_sizes, out=so[1:])
        D = np.zeros((so[-1], so[-1]), dtype=self.values.dtype)
        off = self.slot_offsets()
        for i in range(self.n):
            r = self.block_sizes[i]
            for s in range(self.row_ptr[i], self.row_ptr[i + 1]):
                j = self.col_ind[s]
                c = self.block_sizes[j]
                D[so[i] : so[i] + r, so[j] : so[j] + c] += self.values[off[s] : off[s + 1]].reshape(r, c)
        return D

    def scalar_offsets(self) -> np.ndarray:
        so = np.zeros(self.n + 1, np.int64)
        np.cumsum(self.block_sizes, out=so[1:])
        return so


def _assemble(n, bsz, rows, cols, blocks_by_shape, dtype=np.float64) -> BlockCSR:
    """rows/cols: int arrays of block coordinates (one entry per block, no
    duplicates); blocks_by_shape: list of (index array into rows/cols, value
    array [m, r, c]).  Sorts into CSR order and scatters values."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    order = np.lexsort((cols, rows))
    inv = np.empty_like(order)
    inv[order] = np.arange(len(order))
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    col_ind = cols[order]
    srows = rows[order]
    sizes = bsz[srows].astype(np.int64) * bsz[col_ind].astype(np.int64)
    off = np.zeros(len(order) + 1, np.int64)
    np.cumsum(sizes, out=off[1:])
    values = np.zeros(off[-1], dtype=dtype)
    for idx, vals in blocks_by_shape:
        if len(idx) == 0:
            continue
        m, r, c = vals.shape
        start = off[inv[idx]]
        tgt = start[:, None] + np.arange(r * c)[None, :]
        values[tgt.ravel()] = vals.reshape(m, r * c).ravel()
    return BlockCSR(bsz.astype(np.int32), row_ptr.astype(np.int32), col_ind.astype(np.int32), values)


def _symmetric_from_bonds(n, bsz, bi, bj, rng, hop_sampler, onsite_sampler, dtype=np.float64, phase=None):
    """Builds H = H^T (or H^H) from undirected bonds (bi < bj) plus diagonal
    blocks.  hop_sampler(m, r, c) -> [m, r, c]; onsite_sampler(m, r) -> [m, r, r]
    (symmetrised here)."""
    bi = np.asarray(bi, np.int64)
    bj = np.asarray(bj, np.int64)
    rows = [np.arange(n), bi, bj]
    cols = [np.arange(n), bj, bi]
    nb = len(bi)
    groups = []
    # diagonal blocks, grouped by size
    for r in np.unique(bsz):
        ids = np.nonzero(bsz == r)[0]
        B = onsite_sampler(len(ids), int(r))
        B = 0.5 * (B + np.swapaxes(B, 1, 2).conj())
        groups.append((ids, B.astype(dtype)))
    # bonds grouped by (r, c)
    ri, cj = bsz[bi], bsz[bj]
    keys = ri.astype(np.int64) * 1000 + cj
    for key in np.unique(keys):
        sel = np.nonzero(keys == key)[0]
        r, c = int(key // 1000), int(key % 1000)
        B = hop_sampler(len(sel), r, c).astype(dtype)
        if phase is not None:
            B = B * np.exp(1j * phase[sel])[:, None, None]
        groups.append((n + sel, B))
        groups.append((n + nb + sel, np.swapaxes(B, 1, 2).conj()))
    return _assemble(n, bsz, np.concatenate(rows), np.concatenate(cols), groups, dtype=dtype)


def random_symmetric_blocks(n_blocks: int = 5000, size_min: int = 4, size_max: int = 8, neighbours: int = 6,
                            seed: int = 1) -> BlockCSR:
    """Diagonal + for each i, `neighbours` distinct j != i mirrored to (j, i);
    entries U[-1, 1], symmetrised so A = A^T (off-diagonal B_ji = B_ij^T,
    diagonal (B + B^T)/2).  ~12 off-diagonal + 1 diagonal block per row."""
    rng = np.random.default_rng(seed)
    bsz = rng.integers(size_min, size_max + 1, size=n_blocks).astype(np.int64)
    src = np.repeat(np.arange(n_blocks), neighbours)
    # distinct j != i per row: sample from n-1 values and skip i
    draws = np.empty((n_blocks, neighbours), np.int64)
    for i in range(n_blocks):
        d = rng.choice(n_blocks - 1, size=neighbours, replace=False)
        draws[i] = d + (d >= i)
    dst = draws.ravel()
    a = np.minimum(src, dst)
    b = np.maximum(src, dst)
    pairs = np.unique(a * n_blocks + b)
    bi, bj = pairs // n_blocks, pairs % n_blocks
    return _symmetric_from_bonds(
        n_blocks, bsz, bi, bj, rng,
        hop_sampler=lambda m, r, c: rng.uniform(-1.0, 1.0, size=(m, r, c)),
        onsite_sampler=lambda m, r: rng.uniform(-1.0, 1.0, size=(m, r, r)),
    )


# Metal (5 orbitals) at fractional (0, 0); two chalcogens (3 orbitals each) at
# (1/3, 1/3), one above and one below the metal plane.
TMD_SITE_SIZES = (5, 3, 3)
_NN_MX = ((0, 0), (-1, 0), (0, -1))  # metal (cell c) -> chalcogen cells c + d
_IN_PLANE = ((1, 0), (0, 1), (1, -1))  # half of the 6 in-plane neighbours


def tmd_lattice(L: int = 200, seed: int = 2, hop_sigma: float = 0.5, onsite_sigma: float = 0.2,
                disorder: float = 0.0, dtype=np.float64, bond_phase: bool = False, rescale: float = 0.95,
                Ly: int | None = None):
    """TMD-like triangular-lattice tight-binding Hamiltonian on an L x Ly
    periodic supercell.  Bonds: metal-chalcogen nearest neighbours (each metal
    to both chalcogens of 3 cells), metal-metal and chalcogen-chalcogen
    (same layer) in-plane neighbours (6 each), and the vertical
    chalcogen-chalcogen pair of each cell: 35 blocks per cell.  Hopping
    blocks ~ N(0, hop_sigma), on-site blocks ~ N(0, onsite_sigma) symmetrised,
    optional on-site disorder U(-W/2, W/2) on the diagonal, optional random
    bond phases (complex Hermitian).  Returns (BlockCSR rescaled so that its
    Gershgorin bound is `rescale`, the bound g of the unscaled matrix)."""
    Ly = L if Ly is None else Ly
    rng = np.random.default_rng(seed)
    ncell = L * Ly
    n = 3 * ncell
    bsz = np.tile(np.array(TMD_SITE_SIZES, np.int64), ncell)
    ix, iy = np.meshgrid(np.arange(L), np.arange(Ly), indexing="xy")
    ix, iy = ix.ravel(), iy.ravel()
    cell = iy * L + ix

    def cid(dx, dy):
        return ((iy + dy) % Ly) * L + (ix + dx) % L

    bi, bj = [], []

    def add(a, b):
        a = np.asarray(a)
        b = np.asarray(b)
        bi.append(np.minimum(a, b))
        bj.append(np.maximum(a, b))

    for dx, dy in _NN_MX:
        for site in (1, 2):
            add(3 * cell, 3 * cid(dx, dy) + site)
    for dx, dy in _IN_PLANE:
        for site in (0, 1, 2):
            add(3 * cell + site, 3 * cid(dx, dy) + site)
    add(3 * cell + 1, 3 * cell + 2)
    bi = np.concatenate(bi)
    bj = np.concatenate(bj)
    keep = bi != bj
    key = np.unique(bi[keep] * n + bj[keep])
    bi, bj = key // n, key % n
    phase = rng.uniform(0, 2 * np.pi, size=len(bi)) if bond_phase else None
    cdtype = np.complex128 if (bond_phase or np.dtype(dtype) == np.complex128) else np.float64
    H = _symmetric_from_bonds(
        n, bsz, bi, bj, rng,
        hop_sampler=lambda m, r, c: rng.normal(0.0, hop_sigma, size=(m, r, c)),
        onsite_sampler=lambda m, r: rng.normal(0.0, onsite_sigma, size=(m, r, r)),
        dtype=cdtype, phase=phase,
    )
    if disorder:
        so = H.scalar_offsets()
        eps = rng.uniform(-disorder / 2, disorder / 2, size=so[-1])
        add_diagonal(H, eps)
    g = gershgorin_bound(H)
    if rescale:
        H.values *= rescale / g
    return H, g


def add_diagonal(H: BlockCSR, d: np.ndarray) -> None:
    """In place: H_ii += d_i on the diagonal blocks (rows without a diagonal
    block are left alone)."""
    off = H.slot_offsets()
    so = H.scalar_offsets()
    rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
    diag = np.nonzero(H.col_ind == rows)[0]  # at most one per row (columns are distinct)
    drow = rows[diag]
    r = H.block_sizes[drow].astype(np.int64)
    t = np.arange(int(r.sum())) - np.repeat(np.cumsum(r) - r, r)
    tgt = np.repeat(off[diag], r) + t * (np.repeat(r, r) + 1)
    H.values[tgt] += d[np.repeat(so[drow], r) + t]


def scalar_coords(H: BlockCSR):
    """(scalar row, scalar col) of every stored value, slot order."""
    so = H.scalar_offsets()
    rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
    r = H.block_sizes[rows].astype(np.int64)
    c = H.block_sizes[H.col_ind].astype(np.int64)
    sizes = r * c
    blk = np.repeat(np.arange(H.nnzb), sizes)
    off = H.slot_offsets()
    local = np.arange(H.nnz) - off[blk]
    cc = c[blk]
    return so[rows][blk] + local // cc, so[H.col_ind][blk] + local % cc


def gershgorin_bound(H: BlockCSR) -> float:
    """max over scalar rows of sum_j |H_ij|: each block's rows are runs of c
    consecutive values (row-major), summed with one reduceat."""
    off = H.slot_offsets()
    so = H.scalar_offsets()
    rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
    r = H.block_sizes[rows].astype(np.int64)
    c = H.block_sizes[H.col_ind].astype(np.int64)
    t = np.arange(int(r.sum())) - np.repeat(np.cumsum(r) - r, r)
    starts = np.repeat(off[:-1], r) + t * np.repeat(c, r)
    if len(starts) == 0:
        return 0.0
    sums = np.add.reduceat(np.abs(H.values), starts)
    radii = np.bincount(np.repeat(so[rows], r) + t, weights=sums, minlength=H.N)
    return float(radii.max())


def banded_decaying(n_blocks: int = 20000, size_min: int = 4, size_max: int = 8, neighbours: int = 8,
                    band: int = 32, decay: float = 4.0, seed: int = 3) -> BlockCSR:
    """Symmetric, banded, exponentially decaying variable-block matrix: for each
    i draw `neighbours` j = i + U{-band..band} \\ {0} (mirrored), entries
    U[-1, 1] * exp(-|i-j| / decay)."""
    rng = np.random.default_rng(seed)
    bsz = rng.integers(size_min, size_max + 1, size=n_blocks).astype(np.int64)
    off = rng.integers(1, band + 1, size=(n_blocks, neighbours)) * rng.choice([-1, 1], size=(n_blocks, neighbours))
    src = np.repeat(np.arange(n_blocks), neighbours)
    dst = src + off.ravel()
    ok = (dst >= 0) & (dst < n_blocks)
    src, dst = src[ok], dst[ok]
    a, b = np.minimum(src, dst), np.maximum(src, dst)
    pairs = np.unique(a * n_blocks + b)
    bi, bj = pairs // n_blocks, pairs % n_blocks
    dist = np.abs(bi - bj).astype(np.float64)
    # decay applied per bond after sampling
    H = _symmetric_from_bonds(
        n_blocks, bsz, bi, bj, rng,
        hop_sampler=lambda m, r, c: rng.uniform(-1.0, 1.0, size=(m, r, c)),
        onsite_sampler=lambda m, r: rng.uniform(-1.0, 1.0, size=(m, r, r)),
    )
    rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
    fac = np.exp(-np.abs(rows - H.col_ind) / decay)
    sizes = H.block_sizes[rows].astype(np.int64) * H.block_sizes[H.col_ind]
    H.values *= np.repeat(fac, sizes)
    return H


def ring_blocks(n_blocks: int = 4, block_size: int = 2, diag: float = 1.0, off: float = 0.5,
                directed: bool = True) -> BlockCSR:
    """Ring of uniform blocks: diagonal blocks diag*I and off*I on the ring
    neighbour(s): (i, i+1 mod n) when directed -- the matrix of the
    reference's SpGEMM ring tests (tests/test_spmm.py:40-90, 93-200) -- else
    both i-1 and i+1."""
    n = n_blocks
    bsz = np.full(n, block_size, np.int64)
    rows, cols = [], []
    for i in range(n):
        nb = {i, (i + 1) % n} if directed else {(i - 1) % n, i, (i + 1) % n}
        for j in sorted(nb):
            rows.append(i)
            cols.append(j)
    rows = np.array(rows)
    cols = np.array(cols)
    eye = np.eye(block_size)
    vals = np.stack([(diag if r == c else off) * eye for r, c in zip(rows, cols)])
    return _assemble(n, bsz, rows, cols, [(np.arange(len(rows)), vals)])


def from_dense_blocks(bsz, pattern_rows, pattern_cols, dense: np.ndarray) -> BlockCSR:
    """Cuts the given block pattern out of a dense matrix."""
    bsz = np.asarray(bsz, np.int64)
    so = np.zeros(len(bsz) + 1, np.int64)
    np.cumsum(bsz, out=so[1:])
    groups = []
    vals = [dense[so[i] : so[i] + bsz[i], so[j] : so[j] + bsz[j]] for i, j in zip(pattern_rows, pattern_cols)]
    # group by shape
    shapes = {}
    for k, v in enumerate(vals):
        shapes.setdefault(v.shape, []).append(k)
    for shp, ks in shapes.items():
        groups.append((np.array(ks), np.stack([vals[k] for k in ks])))
    return _assemble(len(bsz), bsz, pattern_rows, pattern_cols, groups, dtype=dense.dtype)


def random_pattern(n_blocks: int, size_min: int, size_max: int, per_row: int, seed: int, dtype=np.float64,
                   symmetric_pattern: bool = False) -> BlockCSR:
    """Random (non-symmetric) pattern with the diagonal plus `per_row` random
    columns per row, entries U[0, 1) (+ i U[0, 1) for complex)."""
    rng = np.random.default_rng(seed)
    bsz = rng.integers(size_min, size_max + 1, size=n_blocks).astype(np.int64)
    rows, cols = [], []
    for i in range(n_blocks):
        cs = set(rng.choice(n_blocks, size=min(per_row, n_blocks), replace=False).tolist())
        cs.add(i)
        for j in sorted(cs):
            rows.append(i)
            cols.append(j)
            if symmetric_pattern and j != i:
                rows.append(j)
                cols.append(i)
    key = np.unique(np.array(rows, np.int64) * n_blocks + np.array(cols, np.int64))
    rows, cols = key // n_blocks, key % n_blocks
    groups = []
    shp = bsz[rows] * 1000 + bsz[cols]
    for k in np.unique(shp):
        sel = np.nonzero(shp == k)[0]
        r, c = int(k // 1000), int(k % 1000)
        v = rng.random((len(sel), r, c))
        if np.dtype(dtype) == np.complex128:
            v = v + 1j * rng.random((len(sel), r, c))
        groups.append((sel, v))
    return _assemble(n_blocks, bsz, rows, cols, groups, dtype=dtype)


def block_diagonal(mats) -> tuple[BlockCSR, np.ndarray]:
    """Block-diagonal concatenation of square BlockCSR matrices (same value
    dtype); returns it and the block-row boundaries of the parts (n_parts + 1)."""
    seg = np.zeros(len(mats) + 1, np.int64)
    for i, m in enumerate(mats):
        seg[i + 1] = seg[i] + m.n
    bsz = np.concatenate([m.block_sizes for m in mats]).astype(np.int32)
    rp = [np.zeros(1, np.int64)]
    ci = []
    base = 0
    for i, m in enumerate(mats):
        rp.append(m.row_ptr[1:].astype(np.int64) + base)
        ci.append(m.col_ind.astype(np.int64) + seg[i])
        base += m.nnzb
    row_ptr = np.concatenate(rp).astype(np.int32)
    col_ind = np.concatenate(ci).astype(np.int32)
    values = np.concatenate([m.values for m in mats])
    return BlockCSR(bsz, row_ptr, col_ind, values), seg.astype(np.int32)


def _tmd_member(args):
    L, s, disorder = args
    return tmd_lattice(int(L), seed=int(s), disorder=disorder)[0]


def tmd_disorder_batch(count: int, side_min: int, side_max: int, disorder: float = 1.0, seed: int = 4,
                       workers: int = 0):
    """`count` disorder realisations of the TMD lattice with supercell sides
    drawn uniform in [side_min, side_max] and on-site disorder U(-W/2, W/2),
    each rescaled into [-0.95, 0.95].  The first k members of a larger batch
    with the same seed are this batch of k.  workers > 1 builds them in that
    many processes (started with `spawn`, so callers that already use CUDA
    may do it)."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(side_min, side_max + 1, size=count)
    tasks = [(int(L), int(rng.integers(1 << 30)), disorder) for L in sides]
    if workers and workers > 1 and count > 1:
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(min(workers, count)) as pool:
            return pool.map(_tmd_member, tasks, chunksize=1)
    return [_tmd_member(t) for t in tasks]

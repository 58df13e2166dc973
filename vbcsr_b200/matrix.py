"""VBCSR: the reference's SciPy-compatible matrix class (vbcsr/matrix.py) on the
B200 engine.  Same constructors, operators and LinearOperator hooks; the work
runs through the ``vbcsr_core`` host core and the C ABI beneath it.

Differences from the reference, all deliberate:
* construction fills values in bulk (one call) instead of one ``add_block``
  pybind call per block; the resulting matrix is identical;
* the wrapper's ``graph`` is re-read from the core after operations that may
  change the pattern (axpy/axpby/filter), so a union-pattern result stays
  usable (the reference's wrapper keeps a stale graph there);
* only serial (single-rank) communicators are supported;
* SciPy >= 1.15 reads the operator's array namespace (``_xp``) that
  ``LinearOperator.__init__`` sets, which neither class calls; the reference's
  ``matvec`` / ``cg`` then fail with AttributeError, this class supplies the
  namespace that SciPy gives its own operators.
"""
from __future__ import annotations

from typing import Any, List, Optional, Tuple

import numpy as np
from scipy.sparse.linalg import LinearOperator

from . import _core
from .multivector import DistMultiVector
from .vector import DistVector

vbcsr_core = _core.load()
AssemblyMode = vbcsr_core.AssemblyMode

# The array namespace SciPy's LinearOperator.__init__ records (None on SciPy
# versions without one), taken from an operator SciPy builds itself.
_SCIPY_XP = getattr(LinearOperator(dtype=np.float64, shape=(1, 1), matvec=lambda v: v), "_xp", None)


def _slot_sizes(bsz: np.ndarray, row_ptr: np.ndarray, col_ind: np.ndarray) -> np.ndarray:
    rows = np.repeat(np.arange(len(bsz)), np.diff(row_ptr))
    return np.asarray(bsz)[rows].astype(np.int64) * np.asarray(bsz)[col_ind].astype(np.int64)


class VBCSR(LinearOperator):
    """Variable Block Compressed Sparse Row matrix on one B200."""

    if _SCIPY_XP is not None:
        _xp = _SCIPY_XP

    def __init__(self, graph: Any, dtype: type = np.float64, comm: Any = None):
        self.graph = graph
        self.dtype = np.dtype(dtype)
        self.comm = comm
        if self.dtype == np.dtype(np.float64):
            self._core = vbcsr_core.BlockSpMat_Double(graph)
        elif self.dtype == np.dtype(np.complex128):
            self._core = vbcsr_core.BlockSpMat_Complex(graph)
        else:
            raise TypeError(f"unsupported dtype {self.dtype}; use float64 or complex128")
        self.shape = tuple(int(s) for s in self._core.shape)

    @classmethod
    def _wrap_core(cls, core: Any, dtype, comm: Any, shape: Optional[Tuple[int, int]] = None,
                   global_nnz: Optional[int] = None) -> "VBCSR":
        obj = cls.__new__(cls)
        obj.graph = core.graph
        obj.dtype = np.dtype(dtype)
        obj.comm = comm
        obj._core = core
        obj.shape = shape if shape is not None else tuple(int(s) for s in core.shape)
        return obj

    def _refresh_graph(self) -> None:
        self.graph = self._core.graph

    # ---- properties (matrix.py:99-250) ----
    @property
    def ndim(self) -> int:
        return 2

    @property
    def nnz(self) -> int:
        return int(self._core.global_nnz)

    @property
    def matrix_kind(self) -> str:
        return self._core.matrix_kind

    @property
    def local_nnz(self) -> int:
        return int(self._core.local_nnz)

    @property
    def local_block_nnz(self) -> int:
        return int(self._core.local_block_nnz)

    @property
    def configured_page_size(self) -> int:
        return int(self._core.configured_page_size)

    @property
    def vendor_backend_name(self) -> str:
        return str(self._core.vendor_backend_name)

    @property
    def vendor_launch_count(self) -> int:
        return int(self._core.vendor_launch_count)

    def reset_vendor_launch_count(self) -> None:
        self._core.reset_vendor_launch_count()

    @property
    def page_size(self) -> int:
        return int(self._core.page_size)

    @page_size.setter
    def page_size(self, value: int) -> None:
        self._core.set_page_size(int(value))

    def set_page_size(self, value: int) -> None:
        self._core.set_page_size(int(value))

    @property
    def shape_class_count(self) -> int:
        return int(self._core.shape_class_count)

    @property
    def has_contiguous_layout(self) -> bool:
        return bool(self._core.has_contiguous_layout)

    def pack_contiguous(self) -> None:
        self._core.pack_contiguous()

    @property
    def T(self) -> "VBCSR":
        return self.transpose()

    def transpose(self) -> "VBCSR":
        """Conjugate (Hermitian) transpose A^H (conjugates complex data)."""
        return self._wrap_core(self._core.transpose(), self.dtype, self.comm, shape=(self.shape[1], self.shape[0]))

    def transpose_(self) -> None:
        self._core = self._core.transpose()
        self.graph = self._core.graph
        self.shape = (self.shape[1], self.shape[0])

    def conj_(self) -> None:
        self._core.conjugate()

    def conj(self) -> "VBCSR":
        obj = self.duplicate()
        obj.conj_()
        return obj

    def conjugate(self) -> "VBCSR":
        return self.conj()

    @property
    def real(self) -> "VBCSR":
        return self._wrap_core(self._core.real(), np.float64, self.comm, shape=self.shape)

    @property
    def imag(self) -> "VBCSR":
        return self._wrap_core(self._core.imag(), np.float64, self.comm, shape=self.shape)

    def __neg__(self) -> "VBCSR":
        return self * -1

    def __pos__(self) -> "VBCSR":
        return self

    def __getitem__(self, key):
        if isinstance(key, tuple) and len(key) == 2 and all(isinstance(k, int) for k in key):
            raise NotImplementedError("Scalar indexing is not supported; use get_block(...) for block access.")
        raise NotImplementedError("Slicing is not supported on VBCSR matrices.")

    def dot(self, other):
        return self @ other

    def copy(self) -> "VBCSR":
        return self.duplicate()

    def __len__(self) -> int:
        return self.shape[0]

    def __repr__(self):
        return f"<{self.shape[0]}x{self.shape[1]} VBCSR matrix of type {self.dtype} with {self.nnz} stored elements>"

    # ---- constructors (matrix.py:260-410, 877-976) ----
    @classmethod
    def create_serial(cls, global_blocks: int, block_sizes: List[int], adjacency: List[List[int]],
                      dtype: type = np.float64, comm: Any = None) -> "VBCSR":
        graph = vbcsr_core.DistGraph(comm)
        graph.construct_serial(int(global_blocks), [int(b) for b in block_sizes],
                               [[int(c) for c in row] for row in adjacency])
        return cls(graph, dtype, comm)

    @classmethod
    def create_distributed(cls, owned_indices: List[int], block_sizes: List[int], adjacency: List[List[int]],
                           dtype: type = np.float64, comm: Any = None) -> "VBCSR":
        graph = vbcsr_core.DistGraph(comm)
        graph.construct_distributed([int(i) for i in owned_indices], [int(b) for b in block_sizes],
                                    [[int(c) for c in row] for row in adjacency])
        return cls(graph, dtype, comm)

    @classmethod
    def create_distributed_flat(cls, owned_indices, block_sizes, adj_ptr, adj_ind, dtype: type = np.float64,
                                comm: Any = None) -> "VBCSR":
        graph = vbcsr_core.DistGraph(comm)
        graph.construct_distributed_flat(
            np.ascontiguousarray(owned_indices, dtype=np.int32),
            np.ascontiguousarray(block_sizes, dtype=np.int32),
            np.ascontiguousarray(adj_ptr, dtype=np.int64),
            np.ascontiguousarray(adj_ind, dtype=np.int32),
        )
        return cls(graph, dtype, comm)

    @classmethod
    def from_block_csr(cls, block_sizes, row_ptr, col_ind, values, dtype: type = np.float64, comm: Any = None):
        """Bulk constructor: block pattern (sorted columns per row) and values in
        slot order, row-major blocks -- the layout ``get_values`` returns."""
        n = len(block_sizes)
        mat = cls.create_distributed_flat(np.arange(n), block_sizes, row_ptr, col_ind, dtype=dtype, comm=comm)
        mat._core.set_values(np.ascontiguousarray(values, dtype=mat.dtype))
        return mat

    @classmethod
    def create_random(cls, global_blocks: int = 100, block_size_min: int = 1, block_size_max: int = 4,
                      density: float = 0.01, dtype: type = np.float64, seed: int = 42, comm: Any = None) -> "VBCSR":
        """Random connected matrix for benchmarking, drawing exactly the
        reference's random stream (matrix.py:331-410): np.random.seed(seed);
        block sizes by randint; per row the ring (i-1, i, i+1) plus
        np.random.choice(global_blocks, max(0, int(N*density)-2), replace=False)
        columns; then, block by block in row-major order, np.random.rand(r, c)
        (+ 1j*np.random.rand(r, c) for complex).  The values are drawn in one
        call instead of one per block -- the same stream, bulk-filled."""
        dtype = np.dtype(dtype)
        np.random.seed(seed)
        sizes = np.random.randint(block_size_min, block_size_max + 1, size=global_blocks)
        n_random = max(0, int(global_blocks * density) - 2)
        adj = []
        for i in range(global_blocks):
            nb = {(i - 1) % global_blocks, (i + 1) % global_blocks, i}
            if n_random > 0:
                nb.update(np.random.choice(global_blocks, size=n_random, replace=False).tolist())
            adj.append(sorted(nb))
        row_ptr = np.zeros(global_blocks + 1, np.int64)
        row_ptr[1:] = np.cumsum([len(a) for a in adj])
        col_ind = np.fromiter((c for a in adj for c in a), dtype=np.int64, count=int(row_ptr[-1]))
        blk = _slot_sizes(sizes, row_ptr, col_ind)
        total = int(blk.sum())
        if dtype == np.dtype(np.float64):
            values = np.random.rand(total)
        else:
            # per block: r*c real parts, then r*c imaginary parts
            raw = np.random.rand(2 * total)
            off = np.zeros(len(blk) + 1, np.int64)
            np.cumsum(blk, out=off[1:])
            blk_idx = np.repeat(np.arange(len(blk)), blk)
            local = np.arange(total) - off[blk_idx]
            values = raw[2 * off[blk_idx] + local] + 1j * raw[2 * off[blk_idx] + blk[blk_idx] + local]
        mat = cls.create_distributed_flat(np.arange(global_blocks), sizes, row_ptr, col_ind, dtype=dtype, comm=comm)
        mat._core.set_values(values.astype(dtype, copy=False))
        mat.assemble()
        return mat

    @classmethod
    def from_scipy(cls, spmat: Any, comm: Any = None, root: int = 0) -> "VBCSR":
        """SciPy BSR with square R x R blocks -> block size R; anything else ->
        CSR with block size 1 (matrix.py:877-976)."""
        import scipy.sparse as sp

        if spmat is None:
            raise ValueError("from_scipy requires a SciPy sparse matrix in serial mode.")
        if spmat.shape[0] != spmat.shape[1]:
            raise ValueError("VBCSR.from_scipy requires a square sparse matrix.")
        dtype = np.dtype(spmat.dtype)
        if sp.issparse(spmat) and spmat.format == "bsr":
            R, C = spmat.blocksize
            if R != C:
                raise ValueError("VBCSR requires square blocks (R == C) for BSR input.")
            if spmat.shape[0] % R != 0:
                raise ValueError("BSR input dimensions must be divisible by the block size.")
            n = spmat.shape[0] // R
            sizes = np.full(n, R)
            indptr = np.asarray(spmat.indptr)
            order = np.lexsort((spmat.indices, np.repeat(np.arange(n), np.diff(indptr))))
            values = np.asarray(spmat.data)[order].reshape(-1)
            col = np.asarray(spmat.indices)[order]
        else:
            csr = spmat.tocsr()
            n = csr.shape[0]
            sizes = np.ones(n, np.int64)
            indptr = np.asarray(csr.indptr)
            order = np.lexsort((csr.indices, np.repeat(np.arange(n), np.diff(indptr))))
            col = csr.indices[order]
            values = np.asarray(csr.data)[order]
        mat = cls.create_distributed_flat(np.arange(n), sizes, indptr.astype(np.int64), col, dtype=dtype, comm=comm)
        mat._core.set_values(np.ascontiguousarray(values, dtype=dtype))
        mat.assemble()
        return mat

    def create_vector(self) -> DistVector:
        cls = vbcsr_core.DistVector_Double if self.dtype == np.float64 else vbcsr_core.DistVector_Complex
        return DistVector(cls(self.graph), self.comm)

    def create_multivector(self, k: int) -> DistMultiVector:
        cls = vbcsr_core.DistMultiVector_Double if self.dtype == np.float64 else vbcsr_core.DistMultiVector_Complex
        return DistMultiVector(cls(self.graph, int(k)), self.comm)

    # ---- assembly / access ----
    def add_block(self, g_row: int, g_col: int, data: np.ndarray, mode=None) -> None:
        if mode is None:
            mode = AssemblyMode.ADD
        self._core.add_block(int(g_row), int(g_col), np.asarray(data, dtype=self.dtype), mode)

    def assemble(self) -> None:
        self._core.assemble()

    def get_block(self, g_row: int, g_col: int) -> Optional[np.ndarray]:
        l_row = self.graph.get_local_index(g_row)
        l_col = self.graph.get_local_index(g_col)
        if l_row == -1 or l_col == -1:
            return None
        data = self._core.get_block(l_row, l_col)
        return None if data.size == 0 else data

    # ---- apply (matrix.py:505-617) ----
    def _as_operand(self, x):
        if isinstance(x, np.ndarray):
            if x.ndim == 1:
                v = self.create_vector()
                v.from_numpy(x)
                return v
            if x.ndim == 2:
                mv = self.create_multivector(x.shape[1])
                mv.from_numpy(x)
                return mv
            raise ValueError("Input numpy array must be 1D or 2D")
        return x

    def mult(self, x, y=None):
        x = self._as_operand(x)
        if isinstance(x, DistVector):
            if y is None:
                y = self.create_vector()
            self._core.mult(x._core, y._core)
            return y
        if isinstance(x, DistMultiVector):
            if y is None:
                y = self.create_multivector(x.num_vectors)
            self._core.mult_dense(x._core, y._core)
            return y
        raise TypeError("mult expects DistVector, DistMultiVector, or numpy.ndarray")

    def mult_adjoint(self, x, y=None):
        x = self._as_operand(x)
        if isinstance(x, DistVector):
            if y is None:
                y = self.create_vector()
            self._core.mult_adjoint(x._core, y._core)
            return y
        if isinstance(x, DistMultiVector):
            if y is None:
                y = self.create_multivector(x.num_vectors)
            self._core.mult_dense_adjoint(x._core, y._core)
            return y
        raise TypeError("mult_adjoint expects DistVector, DistMultiVector, or numpy.ndarray")

    def _matvec(self, x: np.ndarray) -> np.ndarray:
        return self.mult(np.asarray(x).reshape(-1).astype(self.dtype, copy=False)).to_numpy().copy()

    def _matmat(self, X: np.ndarray) -> np.ndarray:
        return self.mult(np.asarray(X, dtype=self.dtype)).to_numpy().copy()

    def _rmatvec(self, x: np.ndarray) -> np.ndarray:
        return self.mult_adjoint(np.asarray(x).reshape(-1).astype(self.dtype, copy=False)).to_numpy().copy()

    def _rmatmat(self, X: np.ndarray) -> np.ndarray:
        return self.mult_adjoint(np.asarray(X, dtype=self.dtype)).to_numpy().copy()

    # ---- scalar / structural ops (matrix.py:619-830) ----
    def scale(self, alpha) -> None:
        self._core.scale(alpha)

    def fill(self, value) -> None:
        self._core.fill(value)

    def fill_random(self) -> None:
        self._core.fill_random()

    def copy_from(self, other: "VBCSR") -> None:
        if not isinstance(other, VBCSR):
            raise TypeError("copy_from expects a VBCSR matrix")
        self._core.copy_from(other._core)

    def axpby(self, alpha, x: "VBCSR", beta) -> None:
        if not isinstance(x, VBCSR):
            raise TypeError("axpby expects a VBCSR matrix")
        self._core.axpby(alpha, x._core, beta)
        self._refresh_graph()

    def shift(self, alpha) -> None:
        self._core.shift(alpha)

    def add_diagonal(self, v) -> None:
        if isinstance(v, np.ndarray):
            dv = self.create_vector()
            dv.from_numpy(v)
            v = dv
        if not isinstance(v, DistVector):
            raise TypeError("add_diagonal expects DistVector or numpy.ndarray")
        self._core.add_diagonal(v._core)

    def duplicate(self, independent_graph: bool = True) -> "VBCSR":
        return self._wrap_core(self._core.duplicate(independent_graph), self.dtype, self.comm, shape=self.shape)

    def __add__(self, other):
        if isinstance(other, VBCSR):
            res = self.duplicate()
            res += other
            return res
        return NotImplemented

    def __sub__(self, other):
        if isinstance(other, VBCSR):
            res = self.duplicate()
            res -= other
            return res
        return NotImplemented

    def __isub__(self, other):
        if isinstance(other, VBCSR):
            self._core.axpy(-1.0, other._core)
            self._refresh_graph()
            return self
        return NotImplemented

    def __iadd__(self, other):
        if isinstance(other, VBCSR):
            self._core.axpy(1.0, other._core)
            self._refresh_graph()
            return self
        return NotImplemented

    def __mul__(self, other):
        if np.isscalar(other):
            res = self.duplicate()
            res.scale(other)
            return res
        return NotImplemented

    def __imul__(self, other):
        if np.isscalar(other):
            self.scale(other)
            return self
        return NotImplemented

    def __rmul__(self, other):
        return self.__mul__(other)

    def __truediv__(self, other):
        if np.isscalar(other):
            return self.__mul__(1.0 / other)
        return NotImplemented

    def __itruediv__(self, other):
        if np.isscalar(other):
            self.scale(1.0 / other)
            return self
        return NotImplemented

    def __matmul__(self, other):
        if isinstance(other, VBCSR):
            return self.spmm(other)
        if isinstance(other, (DistVector, DistMultiVector, np.ndarray)):
            return self.mult(other)
        return NotImplemented

    def spmm(self, B: "VBCSR", threshold: float = 0.0, transA: bool = False, transB: bool = False) -> "VBCSR":
        if not isinstance(B, VBCSR):
            raise TypeError("B must be a VBCSR matrix")
        if self.dtype != B.dtype:
            raise TypeError("A and B must have the same dtype")
        core_C = self._core.spmm(B._core, float(threshold), bool(transA), bool(transB))
        return self._wrap_core(core_C, self.dtype, self.comm, shape=(self.shape[0], B.shape[1]))

    def spmm_hermitian(self, B: "VBCSR", threshold: float = 0.0, transA: bool = False) -> "VBCSR":
        if not isinstance(B, VBCSR):
            raise TypeError("B must be a VBCSR matrix")
        if self.dtype != B.dtype:
            raise TypeError("A and B must have the same dtype")
        core_C = self._core.spmm_hermitian(B._core, float(threshold), bool(transA))
        return self._wrap_core(core_C, self.dtype, self.comm, shape=(self.shape[0], B.shape[1]))

    # The reference core's fused triple products (BlockSpMat methods,
    # vbcsr/core/block_csr.hpp:1804-1853): upper block triangle, one drop of
    # the finished blocks; complete with complete_hermitian().
    def square_polynomial_upper(self, c2, c1, c0, threshold: float = 0.0) -> "VBCSR":
        """c2 A^2 + c1 A + c0 I for Hermitian A, upper block triangle."""
        core_C = self._core.square_polynomial_upper(complex(c2), complex(c1), complex(c0), float(threshold))
        return self._wrap_core(core_C, self.dtype, self.comm, shape=self.shape)

    def rarh_upper(self, B: "VBCSR", threshold: float = 0.0) -> "VBCSR":
        """A B A^H for Hermitian A and B, upper block triangle."""
        if not isinstance(B, VBCSR):
            raise TypeError("B must be a VBCSR matrix")
        return self._wrap_core(self._core.rarh_upper(B._core, float(threshold)), self.dtype, self.comm,
                               shape=self.shape)

    def rhar_upper(self, B: "VBCSR", threshold: float = 0.0) -> "VBCSR":
        """A^H B A for Hermitian B, upper block triangle."""
        if not isinstance(B, VBCSR):
            raise TypeError("B must be a VBCSR matrix")
        return self._wrap_core(self._core.rhar_upper(B._core, float(threshold)), self.dtype, self.comm,
                               shape=self.shape)

    def complete_hermitian(self) -> "VBCSR":
        """U + strict_lower(U^H) with Hermitized diagonal blocks, as a new matrix."""
        return self._wrap_core(self._core.complete_hermitian(), self.dtype, self.comm, shape=self.shape)

    def complete_hermitian_inplace(self) -> None:
        self._core.complete_hermitian_inplace()
        self._refresh_graph()

    def spmm_self(self, threshold: float = 0.0, transA: bool = False) -> "VBCSR":
        return self._wrap_core(self._core.spmm_self(float(threshold), bool(transA)), self.dtype, self.comm,
                               shape=self.shape)

    def get_block_density(self) -> float:
        return self._core.get_block_density()

    def filter_blocks(self, threshold: float = 0.0):
        self._core.filter_blocks(float(threshold))
        self._refresh_graph()

    def add(self, B: "VBCSR", alpha: float = 1.0, beta: float = 1.0) -> "VBCSR":
        if not isinstance(B, VBCSR):
            raise TypeError("B must be a VBCSR matrix")
        return self._wrap_core(self._core.add(B._core, alpha, beta), self.dtype, self.comm, shape=self.shape)

    def extract_submatrix(self, global_indices: List[int]) -> "VBCSR":
        return self._wrap_core(self._core.extract_submatrix(list(global_indices)), self.dtype, None)

    def insert_submatrix(self, submat: "VBCSR", global_indices: List[int]) -> None:
        self._core.insert_submatrix(submat._core, list(global_indices))

    def spmf(self, func_name: str, verbose: bool = False) -> "VBCSR":
        return self._wrap_core(self._core.spmf(func_name, verbose), self.dtype, self.comm, shape=self.shape)

    def to_dense(self) -> np.ndarray:
        return self._core.to_dense()

    def from_dense(self, data: np.ndarray) -> None:
        self._core.from_dense(np.asarray(data, dtype=self.dtype))

    @property
    def row_ptr(self) -> np.ndarray:
        return np.asarray(self._core.row_ptr, dtype=np.int32)

    @property
    def col_ind(self) -> np.ndarray:
        return np.asarray(self._core.col_ind, dtype=np.int32)

    def get_values(self) -> np.ndarray:
        return np.asarray(self._core.get_values(), dtype=self.dtype)

    def save_matrix_market(self, filename) -> None:
        self._core.save_matrix_market(str(filename))

    def to_scipy(self, format: Optional[str] = None):
        """Local matrix as SciPy BSR (uniform blocks) or CSR (matrix.py:992-1122)."""
        import scipy.sparse as sp

        values = self.get_values()
        row_ptr, col_ind = self.row_ptr, self.col_ind
        bsz = np.asarray(self.graph.block_sizes, np.int64)
        uniform = len(bsz) > 0 and np.all(bsz == bsz[0])
        fmt = format or ("bsr" if self.matrix_kind in ("csr", "bsr") else "csr")
        N = int(bsz.sum())
        if fmt == "bsr":
            if not uniform:
                raise ValueError("Cannot convert non-uniform VBCSR to BSR format.")
            R = int(bsz[0])
            out = sp.bsr_matrix((values.reshape(-1, R, R), col_ind, row_ptr), shape=(N, N))
            out.sort_indices()
            return out
        if fmt != "csr":
            raise ValueError(f"Unknown format: {fmt}")
        so = np.zeros(len(bsz) + 1, np.int64)
        np.cumsum(bsz, out=so[1:])
        rows = np.repeat(np.arange(len(bsz)), np.diff(row_ptr))
        c = bsz[col_ind]
        sizes = bsz[rows] * c
        blk = np.repeat(np.arange(len(col_ind)), sizes)
        off = np.zeros(len(col_ind) + 1, np.int64)
        np.cumsum(sizes, out=off[1:])
        local = np.arange(len(values)) - off[blk]
        srow = so[rows][blk] + local // c[blk]
        scol = so[col_ind][blk] + local % c[blk]
        out = sp.csr_matrix((values, (srow, scol)), shape=(N, N))
        out.sort_indices()
        return out

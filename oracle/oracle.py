"""Python front of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers share one interface over :class:`vbcsr_b200.workloads.BlockCSR`
inputs:

* ``Restated``  -- the plain-C restatement in oracle/vbcsr_oracle.c
  (oracle/_ref/libvbcsr_oracle.so);
* ``Reference`` -- the reference VBCSR C++ core itself, compiled from its own
  sources by oracle/build_ref.sh (oracle/_ref/libvbcsr_ref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline import this
module.  The shipped library never does.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
ORACLE_LIB = REF_DIR / "libvbcsr_oracle.so"
REFERENCE_LIB = REF_DIR / "libvbcsr_ref.so"

_vp = C.c_void_p


class _OrcMat(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("bsz", _vp),
        ("row_ptr", _vp),
        ("col_ind", _vp),
        ("vals", _vp),
        ("is_complex", C.c_int),
    ]


class _OrcResult(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("row_ptr", C.POINTER(C.c_int)),
        ("col_ind", C.POINTER(C.c_int)),
        ("vals", C.POINTER(C.c_double)),
        ("nnzb", C.c_int64),
        ("nnz", C.c_int64),
        ("stats", C.c_int64 * 4),
    ]


def build(force: bool = False) -> None:
    """Builds oracle/_ref (the C restatement always; the reference core when
    its sources are present -- oracle/build_ref.sh decides and skips it
    otherwise)."""
    import subprocess

    if not force and ORACLE_LIB.exists() and REFERENCE_LIB.exists():
        return
    subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True)


def reference_root() -> Path | None:
    """The reference checkout: $VBCSR_REFERENCE, else the one build_ref.sh
    compiled the reference core from; None when neither exists on this
    machine."""
    cand = os.environ.get("VBCSR_REFERENCE")
    if not cand and (REF_DIR / "reference_root").exists():
        cand = (REF_DIR / "reference_root").read_text().strip()
    if cand and (Path(cand) / "vbcsr" / "core" / "block_csr.hpp").exists():
        return Path(cand)
    return None


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class _Keep:
    """Keeps numpy buffers alive while C holds pointers to them."""

    def __init__(self, H, complex_=None):
        self.is_complex = int(np.iscomplexobj(H.values) if complex_ is None else complex_)
        self.bsz = _c(H.block_sizes, np.int32)
        self.rp = _c(H.row_ptr, np.int32)
        self.ci = _c(H.col_ind, np.int32)
        self.vals = _c(H.values, np.complex128 if self.is_complex else np.float64)
        self.mat = _OrcMat(
            len(self.bsz), self.bsz.ctypes.data, self.rp.ctypes.data, self.ci.ctypes.data,
            self.vals.ctypes.data, self.is_complex,
        )


def _result_to_blockcsr(res: _OrcResult, bsz, is_complex):
    from vbcsr_b200.workloads import BlockCSR

    n = res.n
    rp = np.ctypeslib.as_array(res.row_ptr, shape=(n + 1,)).copy()
    ci = np.ctypeslib.as_array(res.col_ind, shape=(max(res.nnzb, 1),))[: res.nnzb].copy()
    cw = 2 if is_complex else 1
    v = np.ctypeslib.as_array(res.vals, shape=(max(res.nnz * cw, 1),))[: res.nnz * cw].copy()
    if is_complex:
        v = v.view(np.complex128)
    return BlockCSR(np.asarray(bsz, np.int32).copy(), rp.astype(np.int32), ci.astype(np.int32), v)


class Restated:
    """The plain-C restatement."""

    def __init__(self, path: str | os.PathLike | None = None):
        p = Path(path) if path else ORACLE_LIB
        if not p.exists():
            build()
        self.lib = C.CDLL(str(p))
        L = self.lib
        L.orc_apply.argtypes = [C.POINTER(_OrcMat), C.c_int, _vp, _vp, C.c_int]
        L.orc_block_norms.argtypes = [C.POINTER(_OrcMat), _vp]
        L.orc_kpm_moments.argtypes = [C.POINTER(_OrcMat), C.c_int, _vp, C.c_int, C.c_int, _vp]
        L.orc_cheb_apply.argtypes = [C.POINTER(_OrcMat), C.c_int, _vp, _vp, _vp]
        L.orc_set_random.argtypes = [C.c_int, _vp, C.c_int, C.c_uint64, C.c_int, C.c_int, _vp]
        L.orc_spgemm.argtypes = [C.POINTER(_OrcMat), C.POINTER(_OrcMat), C.c_double, C.POINTER(_OrcResult)]
        L.orc_spgemm_hermitian.argtypes = [C.POINTER(_OrcMat), C.POINTER(_OrcMat), C.c_double,
                                           C.POINTER(_OrcResult)]
        L.orc_filter_blocks.argtypes = [C.POINTER(_OrcMat), C.c_double, C.POINTER(_OrcResult)]
        L.orc_axpby.argtypes = [C.POINTER(_OrcMat), C.c_double, C.c_double, C.POINTER(_OrcMat), C.c_double,
                                C.c_double, C.POINTER(_OrcResult)]
        L.orc_transpose.argtypes = [C.POINTER(_OrcMat), C.POINTER(_OrcResult)]
        for f in ("orc_rarh_upper", "orc_rhar_upper"):
            getattr(L, f).argtypes = [C.POINTER(_OrcMat), C.POINTER(_OrcMat), C.c_double, C.POINTER(_OrcResult)]
        L.orc_square_polynomial_upper.argtypes = [C.POINTER(_OrcMat)] + [C.c_double] * 7 + [C.POINTER(_OrcResult)]
        L.orc_result_free.argtypes = [C.POINTER(_OrcResult)]

    def apply(self, H, X, adjoint=False):
        k = _Keep(H)
        X = np.asarray(X)
        vec = X.ndim == 1
        X2 = _c(X.reshape(len(X), -1), np.complex128 if k.is_complex else np.float64)
        Y = np.zeros_like(X2)
        self.lib.orc_apply(C.byref(k.mat), X2.shape[1], X2.ctypes.data, Y.ctypes.data, int(adjoint))
        return Y[:, 0] if vec else Y

    def block_norms(self, H):
        k = _Keep(H)
        out = np.zeros(max(len(k.ci), 1))
        self.lib.orc_block_norms(C.byref(k.mat), out.ctypes.data)
        return out[: len(k.ci)]

    def kpm_moments(self, H, V0, M, two_moment=True):
        k = _Keep(H)
        V = _c(V0, np.float64)
        R = V.shape[1] if V.ndim == 2 else 1
        mu = np.zeros(M)
        self.lib.orc_kpm_moments(C.byref(k.mat), R, V.ctypes.data, M, int(two_moment), mu.ctypes.data)
        return mu

    def cheb_apply(self, H, coeffs, psi):
        k = _Keep(H, complex_=True)
        c = _c(coeffs, np.complex128)
        p = _c(psi, np.complex128)
        out = np.zeros_like(p)
        self.lib.orc_cheb_apply(C.byref(k.mat), len(c), c.ctypes.data, p.ctypes.data, out.ctypes.data)
        return out

    def set_random(self, block_sizes, k, seed, normalize=True, complex_=False):
        bsz = _c(block_sizes, np.int32)
        N = int(bsz.sum())
        out = np.zeros((N, k), np.complex128 if complex_ else np.float64)
        self.lib.orc_set_random(len(bsz), bsz.ctypes.data, k, C.c_uint64(seed), int(normalize), int(complex_),
                                out.ctypes.data)
        return out

    def _result(self, fn, *args, bsz, is_complex):
        res = _OrcResult()
        fn(*args, C.byref(res))
        try:
            out = _result_to_blockcsr(res, bsz, is_complex)
            stats = list(res.stats)
        finally:
            self.lib.orc_result_free(C.byref(res))
        return out, stats

    def spgemm(self, A, B, threshold):
        ka, kb = _Keep(A), _Keep(B)
        return self._result(self.lib.orc_spgemm, C.byref(ka.mat), C.byref(kb.mat), C.c_double(threshold),
                            bsz=A.block_sizes, is_complex=ka.is_complex)

    def spgemm_hermitian(self, A, B, threshold):
        """Upper block triangle of the thresholded product, mirrored and with
        Hermitized diagonal blocks (vbcsr_oracle.c orc_spgemm_hermitian)."""
        ka, kb = _Keep(A), _Keep(B)
        return self._result(self.lib.orc_spgemm_hermitian, C.byref(ka.mat), C.byref(kb.mat), C.c_double(threshold),
                            bsz=A.block_sizes, is_complex=ka.is_complex)

    def filter_blocks(self, A, threshold):
        ka = _Keep(A)
        return self._result(self.lib.orc_filter_blocks, C.byref(ka.mat), C.c_double(threshold),
                            bsz=A.block_sizes, is_complex=ka.is_complex)[0]

    def axpby(self, Y, alpha, X, beta):
        ky, kx = _Keep(Y), _Keep(X)
        a, b = complex(alpha), complex(beta)
        return self._result(self.lib.orc_axpby, C.byref(ky.mat), a.real, a.imag, C.byref(kx.mat), b.real, b.imag,
                            bsz=Y.block_sizes, is_complex=ky.is_complex)[0]

    def transpose(self, A):
        ka = _Keep(A)
        return self._result(self.lib.orc_transpose, C.byref(ka.mat), bsz=A.block_sizes,
                            is_complex=ka.is_complex)[0]

    def rarh_upper(self, A, B, threshold):
        """Upper block triangle of A B A^H (A, B Hermitian), the fused
        executor's gates and single drop (vbcsr_oracle.c orc_rarh_upper)."""
        ka, kb = _Keep(A), _Keep(B)
        return self._result(self.lib.orc_rarh_upper, C.byref(ka.mat), C.byref(kb.mat), C.c_double(threshold),
                            bsz=A.block_sizes, is_complex=ka.is_complex)[0]

    def rhar_upper(self, A, B, threshold):
        """Upper block triangle of A^H B A (vbcsr_oracle.c orc_rhar_upper)."""
        ka, kb = _Keep(A), _Keep(B)
        return self._result(self.lib.orc_rhar_upper, C.byref(ka.mat), C.byref(kb.mat), C.c_double(threshold),
                            bsz=A.block_sizes, is_complex=ka.is_complex)[0]

    def square_polynomial_upper(self, A, c2, c1, c0, threshold):
        """Upper block triangle of c2 A^2 + c1 A + c0 I (A Hermitian)
        (vbcsr_oracle.c orc_square_polynomial_upper)."""
        ka = _Keep(A)
        c2, c1, c0 = complex(c2), complex(c1), complex(c0)
        return self._result(self.lib.orc_square_polynomial_upper, C.byref(ka.mat), c2.real, c2.imag, c1.real,
                            c1.imag, c0.real, c0.imag, C.c_double(threshold), bsz=A.block_sizes,
                            is_complex=ka.is_complex)[0]


class Reference:
    """The reference VBCSR core (BlockSpMat) behind oracle/ref_harness.cpp."""

    def __init__(self, path: str | os.PathLike | None = None, threads: int | None = None):
        p = Path(path) if path else REFERENCE_LIB
        if not p.exists():
            raise FileNotFoundError(f"reference oracle not built: {p}")
        self.lib = C.CDLL(str(p))
        L = self.lib
        L.ref_mat_create.restype = _vp
        L.ref_mat_create.argtypes = [C.c_int, _vp, _vp, _vp, _vp, C.c_int]
        L.ref_mat_free.argtypes = [_vp]
        for f in ("ref_mat_nnzb", "ref_mat_nnz"):
            getattr(L, f).restype = C.c_longlong
            getattr(L, f).argtypes = [_vp]
        L.ref_mat_rows.argtypes = [_vp]
        L.ref_mat_kind.argtypes = [_vp]
        L.ref_mat_structure.argtypes = [_vp, _vp, _vp]
        L.ref_mat_values.argtypes = [_vp, _vp]
        for f in ("ref_mult", "ref_mult_adjoint"):
            getattr(L, f).argtypes = [_vp, _vp, _vp]
        for f in ("ref_mult_dense", "ref_mult_dense_adjoint"):
            getattr(L, f).argtypes = [_vp, C.c_int, _vp, _vp]
        L.ref_mult_repeat.argtypes = [_vp, _vp, _vp, C.c_int]
        L.ref_spmm.restype = _vp
        L.ref_spmm.argtypes = [_vp, _vp, C.c_double, C.c_int, C.c_int]
        L.ref_transpose.restype = _vp
        L.ref_transpose.argtypes = [_vp]
        L.ref_spmm_hermitian.restype = _vp
        L.ref_spmm_hermitian.argtypes = [_vp, _vp, C.c_double, C.c_int]
        for f in ("ref_rarh_upper", "ref_rhar_upper"):
            getattr(L, f).restype = _vp
            getattr(L, f).argtypes = [_vp, _vp, C.c_double]
        L.ref_square_polynomial_upper.restype = _vp
        L.ref_square_polynomial_upper.argtypes = [_vp] + [C.c_double] * 7
        L.ref_duplicate.restype = _vp
        L.ref_duplicate.argtypes = [_vp]
        L.ref_filter_blocks.argtypes = [_vp, C.c_double]
        L.ref_scale.argtypes = [_vp, C.c_double, C.c_double]
        L.ref_shift.argtypes = [_vp, C.c_double, C.c_double]
        L.ref_axpby.argtypes = [_vp, C.c_double, C.c_double, _vp, C.c_double, C.c_double]
        L.ref_block_density.restype = C.c_double
        L.ref_block_density.argtypes = [_vp]
        L.ref_block_norms.argtypes = [_vp, _vp]
        L.ref_set_random.argtypes = [_vp, C.c_int, C.c_ulonglong, C.c_int, _vp]
        L.ref_kpm_moments.argtypes = [_vp, C.c_int, C.c_int, _vp, _vp]
        L.ref_cheb_apply.argtypes = [_vp, C.c_int, _vp, _vp, _vp]
        L.ref_set_threads.argtypes = [C.c_int]
        if threads:
            L.ref_set_threads(int(threads))

    def threads(self) -> int:
        return int(self.lib.ref_get_threads())

    def set_threads(self, n: int) -> None:
        self.lib.ref_set_threads(int(n))

    # matrices are opaque handles wrapped in RefMatrix
    def matrix(self, H) -> "RefMatrix":
        k = _Keep(H)
        h = self.lib.ref_mat_create(len(k.bsz), k.bsz.ctypes.data, k.rp.ctypes.data, k.ci.ctypes.data,
                                    k.vals.ctypes.data, k.is_complex)
        return RefMatrix(self, h, k.is_complex, k.bsz)


class RefMatrix:
    def __init__(self, ref: Reference, h, is_complex, bsz):
        self.ref = ref
        self.lib = ref.lib
        self.h = _vp(h)
        self.is_complex = is_complex
        self.bsz = np.asarray(bsz, np.int32)
        self.N = int(self.bsz.sum())

    def __del__(self):
        try:
            if self.h and self.h.value:
                self.lib.ref_mat_free(self.h)
                self.h = _vp()
        except Exception:
            pass

    @property
    def dtype(self):
        return np.complex128 if self.is_complex else np.float64

    def _wrap(self, h):
        return RefMatrix(self.ref, h, self.is_complex, self.bsz)

    def to_blockcsr(self):
        from vbcsr_b200.workloads import BlockCSR

        n = int(self.lib.ref_mat_rows(self.h))
        nnzb = int(self.lib.ref_mat_nnzb(self.h))
        nnz = int(self.lib.ref_mat_nnz(self.h))
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(max(nnzb, 1), np.int32)
        self.lib.ref_mat_structure(self.h, rp.ctypes.data, ci.ctypes.data)
        v = np.zeros(max(nnz, 1), self.dtype)
        self.lib.ref_mat_values(self.h, v.ctypes.data)
        return BlockCSR(self.bsz.copy(), rp, ci[:nnzb], v[:nnz])

    def kind(self) -> str:
        return {0: "csr", 1: "bsr", 2: "vbcsr"}[int(self.lib.ref_mat_kind(self.h))]

    def mult(self, x, adjoint=False):
        x = _c(x, self.dtype)
        y = np.zeros_like(x)
        (self.lib.ref_mult_adjoint if adjoint else self.lib.ref_mult)(self.h, x.ctypes.data, y.ctypes.data)
        return y

    def mult_dense(self, X, adjoint=False):
        X = _c(X, self.dtype)
        Y = np.zeros_like(X)
        fn = self.lib.ref_mult_dense_adjoint if adjoint else self.lib.ref_mult_dense
        fn(self.h, X.shape[1], X.ctypes.data, Y.ctypes.data)
        return Y

    def mult_repeat(self, x, repeats):
        x = _c(x, np.float64)
        y = np.zeros_like(x)
        self.lib.ref_mult_repeat(self.h, x.ctypes.data, y.ctypes.data, int(repeats))
        return y

    def spmm(self, B: "RefMatrix", threshold, transA=False, transB=False) -> "RefMatrix":
        return self._wrap(self.lib.ref_spmm(self.h, B.h, float(threshold), int(transA), int(transB)))

    def rarh_upper(self, B: "RefMatrix", threshold) -> "RefMatrix":
        return self._wrap(self.lib.ref_rarh_upper(self.h, B.h, float(threshold)))

    def rhar_upper(self, B: "RefMatrix", threshold) -> "RefMatrix":
        return self._wrap(self.lib.ref_rhar_upper(self.h, B.h, float(threshold)))

    def square_polynomial_upper(self, c2, c1, c0, threshold) -> "RefMatrix":
        c2, c1, c0 = complex(c2), complex(c1), complex(c0)
        return self._wrap(self.lib.ref_square_polynomial_upper(self.h, c2.real, c2.imag, c1.real, c1.imag, c0.real,
                                                               c0.imag, float(threshold)))

    def spmm_hermitian(self, B: "RefMatrix", threshold, transA=False) -> "RefMatrix":
        return self._wrap(self.lib.ref_spmm_hermitian(self.h, B.h, float(threshold), int(transA)))

    def transpose(self):
        return self._wrap(self.lib.ref_transpose(self.h))

    def duplicate(self):
        return self._wrap(self.lib.ref_duplicate(self.h))

    def filter_blocks(self, thr):
        self.lib.ref_filter_blocks(self.h, float(thr))

    def scale(self, a):
        a = complex(a)
        self.lib.ref_scale(self.h, a.real, a.imag)

    def shift(self, a):
        a = complex(a)
        self.lib.ref_shift(self.h, a.real, a.imag)

    def axpby(self, alpha, X: "RefMatrix", beta):
        a, b = complex(alpha), complex(beta)
        self.lib.ref_axpby(self.h, a.real, a.imag, X.h, b.real, b.imag)

    def block_density(self):
        return float(self.lib.ref_block_density(self.h))

    def block_norms(self):
        nnzb = int(self.lib.ref_mat_nnzb(self.h))
        out = np.zeros(max(nnzb, 1))
        self.lib.ref_block_norms(self.h, out.ctypes.data)
        return out[:nnzb]

    def set_random(self, k, seed, normalize=True):
        out = np.zeros((self.N, k), self.dtype)
        self.lib.ref_set_random(self.h, k, C.c_ulonglong(seed), int(normalize), out.ctypes.data)
        return out

    def kpm_moments(self, V0, M):
        V = _c(V0, np.float64)
        mu = np.zeros(M)
        self.lib.ref_kpm_moments(self.h, V.shape[1], M, V.ctypes.data, mu.ctypes.data)
        return mu

    def cheb_apply(self, coeffs, psi):
        c = _c(coeffs, np.complex128)
        p = _c(psi, np.complex128)
        out = np.zeros_like(p)
        self.lib.ref_cheb_apply(self.h, len(c), c.ctypes.data, p.ctypes.data, out.ctypes.data)
        return out


def reference_available() -> bool:
    return REFERENCE_LIB.exists()

"""ctypes binding of the C ABI declared in include/vbcsr_b200.h.

This is the same binding any ctypes caller of the library would write.  Every call checks the status code and
raises RuntimeError with vbg_last_error() on failure.  Device buffers are
passed as raw pointers (ints); callers typically hold them in torch tensors.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvbcsr_b200.so"

VBG_F64 = 0
VBG_C128 = 1
VBG_PREC_F64 = 0
VBG_PREC_F32 = 1
KIND_NAMES = {0: "csr", 1: "bsr", 2: "vbcsr"}

_vp = C.c_void_p
_i = C.c_int
_i64 = C.c_int64
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pi64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)

_SIGNATURES = {
    "vbg_version": ([], _i),
    "vbg_last_error": ([], C.c_char_p),
    "vbg_device_count": ([], _i),
    "vbg_device_status": ([C.POINTER(C.c_uint), _i], _i),
    "vbg_set_option": ([C.c_char_p, C.c_longlong], _i),
    "vbg_get_option": ([C.c_char_p, C.POINTER(C.c_longlong)], _i),
    "vbg_memory_reserve": ([C.c_size_t], _i),
    "vbg_memory_trim": ([], _i),
    "vbg_apply_kernel": ([_vp, _i, _i, _pi], _i),
    "vbg_matrix_create": ([C.POINTER(_vp), _i, _i, _pi, _pi, _pi, _vp, _vp], _i),
    "vbg_matrix_destroy": ([_vp], _i),
    "vbg_matrix_duplicate": ([_vp, C.POINTER(_vp), _vp], _i),
    "vbg_matrix_info": ([_vp, _pi, _pi, _pi64, _pi64, _pi64, _pi], _i),
    "vbg_matrix_get_structure": ([_vp, _pi, _pi, _pi], _i),
    "vbg_matrix_get_values": ([_vp, _vp, _vp], _i),
    "vbg_matrix_set_values": ([_vp, _vp, _vp], _i),
    "vbg_matrix_set_values_device": ([_vp, _vp, _vp], _i),
    "vbg_matrix_device_values": ([_vp, C.POINTER(_vp), C.POINTER(_vp)], _i),
    "vbg_matrix_block_norms": ([_vp, _vp, _vp], _i),
    "vbg_spmv": ([_vp, _vp, _vp, _vp], _i),
    "vbg_spmv_adjoint": ([_vp, _vp, _vp, _vp], _i),
    "vbg_spmm": ([_vp, _i, _i, _vp, _vp, _vp], _i),
    "vbg_spmm_adjoint": ([_vp, _i, _i, _vp, _vp, _vp], _i),
    "vbg_spmv_host": ([_vp, _vp, _vp, _vp], _i),
    "vbg_spmm_host": ([_vp, _i, _vp, _vp, _vp], _i),
    "vbg_cheb_step": ([_vp, _i, _i, _d, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _vp], _i),
    "vbg_cheb_step_adjoint": ([_vp, _i, _i, _d, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _vp], _i),
    "vbg_cheb_step_noalloc": ([_vp, _i, _i, _d, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _vp], _i),
    "vbg_kpm_moments": ([_vp, _i, _i, _vp, _i, _i, _i, _i, _vp, _vp], _i),
    "vbg_kpm_moments_host": ([_vp, _i, _vp, _i, _i, _i, _vp, _vp], _i),
    "vbg_kpm_moments_batched": ([_vp, _i, _pi, _i, _i, _vp, _i, _i, _i, _i, _vp, _vp], _i),
    "vbg_mv_scale": ([_i, _i64, _i, _i, _d, _d, _vp, _vp], _i),
    "vbg_mv_axpby": ([_i, _i64, _i, _i, _d, _d, _vp, _d, _d, _vp, _vp], _i),
    "vbg_mv_bdot": ([_i, _i64, _i, _i, _vp, _vp, _vp, _vp], _i),
    "vbg_mv_pointwise": ([_i, _i64, _i, _i, _vp, _i, _vp, _vp], _i),
    "vbg_mv_set_random": ([_vp, _i, _i, C.c_uint64, _i, _vp, _vp], _i),
    "vbg_matrix_scale": ([_vp, _d, _d, _vp], _i),
    "vbg_matrix_shift": ([_vp, _d, _d, _vp], _i),
    "vbg_matrix_add_diagonal": ([_vp, _vp, _vp], _i),
    "vbg_matrix_axpby": ([_vp, _d, _d, _vp, _d, _d, _vp], _i),
    "vbg_matrix_filter_blocks": ([_vp, _d, _vp], _i),
    "vbg_matrix_transpose": ([_vp, C.POINTER(_vp), _vp], _i),
    "vbg_matrix_conjugate": ([_vp, _vp], _i),
    "vbg_spgemm": ([_vp, _vp, _d, C.POINTER(_vp), _pi64, _vp], _i),
    "vbg_spgemm_hermitian": ([_vp, _vp, _d, C.POINTER(_vp), _pi64, _vp], _i),
    "vbg_spgemm_ex": ([_vp, _vp, _d, _i, _i, C.POINTER(_vp), _pi64, _vp], _i),
    "vbg_matrix_trace": ([_vp, _vp, _vp], _i),
    "vbg_matrix_norm_fro": ([_vp, _vp, _vp], _i),
    "vbg_sddmm": ([_vp, _i, _i, _vp, _vp, _d, _d, _vp, _vp], _i),
    "vbg_cheb_series": ([_vp, _i, _i, _vp, _i, _vp, _d, _d, _vp, _i, _vp, _vp], _i),
    "vbg_apply_tile_rows": ([_vp, _i, _i, _pi], _i),
    "vbg_matrix_create_device": ([C.POINTER(_vp), _i, _i, _vp, C.c_int64, _vp, _vp, _vp, _vp], _i),
    "vbg_square_polynomial_upper": ([_vp, _d, _d, _d, _d, _d, _d, _d, C.POINTER(_vp), _vp], _i),
    "vbg_rarh_upper": ([_vp, _vp, _d, C.POINTER(_vp), _vp], _i),
    "vbg_rhar_upper": ([_vp, _vp, _d, C.POINTER(_vp), _vp], _i),
    "vbg_matrix_complete_hermitian": ([_vp, _vp], _i),
}

_lib = None


def exported_symbols() -> list[str]:
    """Names of the entry points this binding expects the library to export."""
    return sorted(_SIGNATURES)


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the CUDA library (once).  Raises if it is missing: there is no
    CPU fallback behind this API."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"vbcsr_b200 CUDA library not found at {p}; build it with `python -m vbcsr_b200._build`"
        )
    lib = C.CDLL(str(p))
    for name, (argtypes, restype) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = restype
    if path is None:
        _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = load().vbg_last_error()
        raise RuntimeError(f"{what or 'vbcsr_b200'} failed ({rc}): {msg.decode() if msg else ''}")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def device_count() -> int:
    return int(load().vbg_device_count())


def device_status(clear: bool = True) -> int:
    """Status bits of the current device's kernels (VBG_STATUS_*); 0 = ok."""
    st = C.c_uint(0)
    call("vbg_device_status", C.byref(st), int(clear))
    return int(st.value)


KERNEL_NAMES = {0: "vector", 1: "rows", 2: "pipe", 3: "tile", 4: "chain", 5: "scalar_rows"}


def apply_kernel(dm: "DeviceMatrix", ld: int, precision: int = 0) -> str:
    """Which forward apply kernel this matrix uses at leading dimension ld:
    'vector' or 'scalar_rows' (ld 1), 'rows', 'pipe', 'tile' or 'chain'."""
    out = C.c_int(-1)
    call("vbg_apply_kernel", dm.h, int(ld), int(precision), C.byref(out))
    return KERNEL_NAMES[out.value]


def apply_tile_rows(dm: "DeviceMatrix", ld: int, precision: int = 0) -> int:
    """Block rows per tile of the tiled kernel's plan at leading dimension
    ld (the autotuner's choice once made; 0 without a plan)."""
    out = C.c_int(0)
    call("vbg_apply_tile_rows", dm.h, int(ld), int(precision), C.byref(out))
    return int(out.value)


def set_option(name: str, value: int) -> None:
    call("vbg_set_option", name.encode(), int(value))


def get_option(name: str) -> int:
    out = C.c_longlong()
    call("vbg_get_option", name.encode(), C.byref(out))
    return int(out.value)


def memory_reserve(nbytes: int) -> None:
    """Map `nbytes` of device memory into the library's pool ahead of use."""
    call("vbg_memory_reserve", C.c_size_t(int(nbytes)))


def memory_trim() -> None:
    """Return the library pool's unused device memory to the driver."""
    call("vbg_memory_trim")


def _arr_i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _ptr(a: np.ndarray, typ=C.c_int):
    return a.ctypes.data_as(C.POINTER(typ))


class DeviceMatrix:
    """Owning Python handle of a vbg_matrix (thin; the product API is VBCSR)."""

    def __init__(self, handle: int, owner: bool = True):
        self.h = _vp(handle)
        self._owner = owner
        info = self.info()
        self.dtype_code = info["dtype"]
        self.n = info["n"]
        self.nnzb = info["nnzb"]
        self.nnz = info["nnz"]
        self.N = info["N"]
        self.kind = KIND_NAMES[info["kind"]]

    @classmethod
    def create(cls, block_sizes, row_ptr, col_ind, values=None, dtype=None, stream: int = 0):
        """dtype: float64 or complex128; by default that of `values`
        (complex values are never cast to real silently)."""
        bsz = _arr_i32(block_sizes)
        rp = _arr_i32(row_ptr)
        ci = _arr_i32(col_ind)
        if dtype is None:
            dtype = np.complex128 if values is not None and np.iscomplexobj(values) else np.float64
        elif np.dtype(dtype) != np.complex128 and values is not None and np.iscomplexobj(values):
            raise TypeError("complex values for a real matrix")
        code = VBG_C128 if np.dtype(dtype) == np.complex128 else VBG_F64
        vals = None
        if values is not None:
            vals = np.ascontiguousarray(values, dtype=np.complex128 if code == VBG_C128 else np.float64)
        out = _vp()
        call(
            "vbg_matrix_create",
            C.byref(out),
            code,
            len(bsz),
            _ptr(bsz),
            _ptr(rp),
            _ptr(ci),
            vals.ctypes.data_as(_vp) if vals is not None else None,
            _vp(stream),
        )
        return cls(out.value)

    def __del__(self):
        try:
            if self._owner and self.h and self.h.value:
                load().vbg_matrix_destroy(self.h)
                self.h = _vp()
        except Exception:
            pass

    def info(self) -> dict:
        dt, n, kind = C.c_int(), C.c_int(), C.c_int()
        nnzb, nnz, N = C.c_int64(), C.c_int64(), C.c_int64()
        call("vbg_matrix_info", self.h, C.byref(dt), C.byref(n), C.byref(nnzb), C.byref(nnz), C.byref(N), C.byref(kind))
        return dict(dtype=dt.value, n=n.value, nnzb=nnzb.value, nnz=nnz.value, N=N.value, kind=kind.value)

    @property
    def np_dtype(self):
        return np.complex128 if self.dtype_code == VBG_C128 else np.float64

    def structure(self):
        info = self.info()
        rp = np.zeros(info["n"] + 1, np.int32)
        ci = np.zeros(max(info["nnzb"], 1), np.int32)
        bs = np.zeros(max(info["n"], 1), np.int32)
        call("vbg_matrix_get_structure", self.h, _ptr(rp), _ptr(ci), _ptr(bs))
        return rp, ci[: info["nnzb"]], bs[: info["n"]]

    def values(self, stream: int = 0) -> np.ndarray:
        info = self.info()
        out = np.zeros(max(info["nnz"], 1), dtype=self.np_dtype)
        call("vbg_matrix_get_values", self.h, out.ctypes.data_as(_vp), _vp(stream))
        return out[: info["nnz"]]

    def set_values(self, values, stream: int = 0) -> None:
        v = np.ascontiguousarray(values, dtype=self.np_dtype)
        call("vbg_matrix_set_values", self.h, v.ctypes.data_as(_vp), _vp(stream))

    # ------------------------------------------------------------ algebra
    def to_blockcsr(self):
        from .workloads import BlockCSR

        rp, ci, bs = self.structure()
        return BlockCSR(bs, rp, ci, self.values())

    def duplicate(self, stream: int = 0) -> "DeviceMatrix":
        out = _vp()
        call("vbg_matrix_duplicate", self.h, C.byref(out), _vp(stream))
        return DeviceMatrix(out.value)

    def transpose(self, stream: int = 0) -> "DeviceMatrix":
        out = _vp()
        call("vbg_matrix_transpose", self.h, C.byref(out), _vp(stream))
        return DeviceMatrix(out.value)

    def spgemm(self, B: "DeviceMatrix", threshold: float, stream: int = 0):
        out = _vp()
        stats = (C.c_int64 * 4)()
        call("vbg_spgemm", self.h, B.h, float(threshold), C.byref(out), stats, _vp(stream))
        return DeviceMatrix(out.value), list(stats)

    def spgemm_hermitian(self, B: "DeviceMatrix", threshold: float, stream: int = 0):
        """C = self @ B for a product known to be Hermitian: the upper block
        triangle multiplied, the lower one mirrored (vbg_spgemm_hermitian).
        Returns (C, stats)."""
        out = _vp()
        stats = (C.c_int64 * 4)()
        call("vbg_spgemm_hermitian", self.h, B.h, float(threshold), C.byref(out), stats, _vp(stream))
        return DeviceMatrix(out.value), list(stats)

    def spgemm_ex(self, B: "DeviceMatrix", threshold: float, precision: int = VBG_PREC_F64, hermitian: bool = False,
                  stream: int = 0):
        """vbg_spgemm / vbg_spgemm_hermitian with the numeric phase in
        `precision` (VBG_PREC_F32: FP32 operands and accumulation).  Returns
        (C, stats)."""
        out = _vp()
        stats = (C.c_int64 * 4)()
        call("vbg_spgemm_ex", self.h, B.h, float(threshold), int(precision), int(bool(hermitian)), C.byref(out), stats,
             _vp(stream))
        return DeviceMatrix(out.value), list(stats)

    @classmethod
    def create_device(cls, block_sizes, row_ptr, col_ind, values=None, stream: int = 0) -> "DeviceMatrix":
        """From a structure in device memory: row_ptr / col_ind int32 CUDA
        tensors (columns ascending per row), values a float64 / complex128
        CUDA tensor in slot order (None: zeros); block_sizes on the host
        (vbg_matrix_create_device)."""
        import torch

        bsz = _arr_i32(block_sizes)
        for t in (row_ptr, col_ind):
            if t.dtype != torch.int32 or not t.is_cuda or not t.is_contiguous():
                raise TypeError("row_ptr and col_ind must be contiguous int32 CUDA tensors")
        code = VBG_F64
        vp = None
        if values is not None:
            if not values.is_cuda or not values.is_contiguous():
                raise TypeError("values must be a contiguous CUDA tensor")
            if values.dtype == torch.complex128:
                code = VBG_C128
            elif values.dtype != torch.float64:
                raise TypeError("values must be float64 or complex128")
            vp = _vp(values.data_ptr())
        out = _vp()
        call("vbg_matrix_create_device", C.byref(out), code, len(bsz), bsz.ctypes.data_as(_vp), int(col_ind.numel()),
             _vp(row_ptr.data_ptr()), _vp(col_ind.data_ptr()), vp, _vp(stream))
        return cls(out.value)

    def square_polynomial_upper(self, c2, c1, c0, threshold: float, stream: int = 0) -> "DeviceMatrix":
        """Upper block triangle of c2 A^2 + c1 A + c0 I for Hermitian A, one
        drop of the finished blocks (vbg_square_polynomial_upper)."""
        c2, c1, c0 = complex(c2), complex(c1), complex(c0)
        out = _vp()
        call("vbg_square_polynomial_upper", self.h, c2.real, c2.imag, c1.real, c1.imag, c0.real, c0.imag,
             float(threshold), C.byref(out), _vp(stream))
        return DeviceMatrix(out.value)

    def rarh_upper(self, B: "DeviceMatrix", threshold: float, stream: int = 0) -> "DeviceMatrix":
        """Upper block triangle of A B A^H, A and B Hermitian (vbg_rarh_upper)."""
        out = _vp()
        call("vbg_rarh_upper", self.h, B.h, float(threshold), C.byref(out), _vp(stream))
        return DeviceMatrix(out.value)

    def rhar_upper(self, B: "DeviceMatrix", threshold: float, stream: int = 0) -> "DeviceMatrix":
        """Upper block triangle of A^H B A, B Hermitian (vbg_rhar_upper)."""
        out = _vp()
        call("vbg_rhar_upper", self.h, B.h, float(threshold), C.byref(out), _vp(stream))
        return DeviceMatrix(out.value)

    def complete_hermitian(self, stream: int = 0) -> None:
        """Upper block triangle -> the full Hermitian matrix, in place."""
        call("vbg_matrix_complete_hermitian", self.h, _vp(stream))

    def trace_dev(self, out_ptr: int, stream: int = 0) -> None:
        """tr(A) (re, im) into the device doubles at out_ptr (vbg_matrix_trace)."""
        call("vbg_matrix_trace", self.h, _vp(out_ptr), _vp(stream))

    def norm_fro_dev(self, out_ptr: int, stream: int = 0) -> None:
        """||A||_F into the device double at out_ptr (vbg_matrix_norm_fro)."""
        call("vbg_matrix_norm_fro", self.h, _vp(out_ptr), _vp(stream))

    def filter_blocks(self, threshold: float, stream: int = 0) -> None:
        call("vbg_matrix_filter_blocks", self.h, float(threshold), _vp(stream))
        self._refresh()

    def axpby(self, alpha, X: "DeviceMatrix", beta, stream: int = 0) -> None:
        a, b = complex(alpha), complex(beta)
        call("vbg_matrix_axpby", self.h, a.real, a.imag, X.h, b.real, b.imag, _vp(stream))
        self._refresh()

    def scale(self, alpha, stream: int = 0) -> None:
        a = complex(alpha)
        call("vbg_matrix_scale", self.h, a.real, a.imag, _vp(stream))

    def shift(self, alpha, stream: int = 0) -> None:
        a = complex(alpha)
        call("vbg_matrix_shift", self.h, a.real, a.imag, _vp(stream))

    def conjugate(self, stream: int = 0) -> None:
        call("vbg_matrix_conjugate", self.h, _vp(stream))

    def _refresh(self) -> None:
        info = self.info()
        self.n, self.nnzb, self.nnz, self.N = info["n"], info["nnzb"], info["nnz"], info["N"]
        self.kind = KIND_NAMES[info["kind"]]

"""GPU-side helpers for the parity tests: every call goes through the C ABI
(vbcsr_b200._capi), torch only holds the device buffers."""
import ctypes as C

import numpy as np
import torch

from vbcsr_b200 import _capi

_vp = C.c_void_p


def ld_for(k, dtype):
    es = np.dtype(dtype).itemsize
    return 1 if k == 1 else ((k * es + 63) // 64) * 64 // es


def dmat(H):
    return _capi.DeviceMatrix.create(H.block_sizes, H.row_ptr, H.col_ind, H.values, dtype=H.values.dtype)


def to_dev_mv(X, ld, dtype):
    X = np.asarray(X)
    X2 = X.reshape(X.shape[0], -1)
    buf = torch.zeros((X2.shape[0], ld), dtype=torch.complex128 if np.dtype(dtype) == np.complex128 else torch.float64,
                      device="cuda")
    buf[:, : X2.shape[1]] = torch.from_numpy(np.ascontiguousarray(X2.astype(dtype))).cuda()
    return buf


def apply(dm, X, adjoint=False):
    X = np.asarray(X)
    dt = dm.np_dtype
    vec = X.ndim == 1
    k = 1 if vec else X.shape[1]
    ld = 1 if vec else ld_for(k, dt)
    xb = to_dev_mv(X, ld, dt)
    yb = torch.zeros_like(xb)
    if vec:
        _capi.call("vbg_spmv_adjoint" if adjoint else "vbg_spmv", dm.h, _vp(xb.data_ptr()), _vp(yb.data_ptr()), None)
    else:
        _capi.call("vbg_spmm_adjoint" if adjoint else "vbg_spmm", dm.h, k, ld, _vp(xb.data_ptr()),
                   _vp(yb.data_ptr()), None)
    torch.cuda.synchronize()
    y = yb.cpu().numpy()
    # pad lanes must stay zero
    if not vec and ld > k:
        assert np.all(y[:, k:] == 0)
    return y[:, 0] if vec else y[:, :k]


def kpm_moments(dm, V0, M, precision=0, two_moment=True, use_graph=False):
    R = V0.shape[1]
    ld = ld_for(R, np.float64) if R > 1 else 1
    vb = to_dev_mv(V0, ld, np.float64)
    mu = torch.zeros(M, dtype=torch.float64, device="cuda")
    _capi.call("vbg_kpm_moments", dm.h, R, ld, _vp(vb.data_ptr()), M, precision, int(two_moment), int(use_graph),
               _vp(mu.data_ptr()), None)
    torch.cuda.synchronize()
    return mu.cpu().numpy()

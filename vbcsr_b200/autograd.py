"""Differentiable sparse apply and Chebyshev expansions (torch.autograd).

The reference has no gradients; these Functions add them on top of the same
device kernels (C ABI):

* :func:`sparse_apply` — Y = A X (vector or multivector), differentiable in
  the block values of A and in X.  Backward: dX = A^H dY (vbg_spmm_adjoint),
  dA = dY X^H on A's pattern (vbg_sddmm).
* :func:`chebyshev_propagate` — psi = sum_n c_n T_n(H~) psi0 with
  H~ = (H - center) / scale, the Chebyshev propagation of
  examples/ex09_graphene_dynamics.py:570-601 (``propagate_chebyshev``), with
  c_n = (2 - delta_n0) (-i)^n J_n(scale dt) for exp(-i H dt).  Differentiable
  in the block values of H and in psi0.
* :func:`kpm_moments` — mu_n = sum_r <v_r, T_n(H~) v_r> (the plain recurrence
  of examples/ex08_graphene_dos.py:99-114), differentiable in H's values.

Backward of the Chebyshev sums: with t_0 = v, t_1 = H~ t_0,
t_{n+1} = 2 H~ t_n - t_{n-1} and sources s_n = dL/dt_n* (conj(c_n) g for
psi = sum c_n t_n with g = dL/dpsi*; g_mu[n] v for the moments), the
adjoint vectors run backwards,

    a_n = s_n + w_n H~^H a_{n+1} - a_{n+2},   w_0 = 1, w_n = 2 (n >= 1),

and dL/dH~* = sum_n w_n a_{n+1} t_n^H on H's pattern (dL/dH* = that / scale),
dL/dv* = a_0 (+ sum_n g_mu[n] t_n for the moments).  The forward keeps every
`checkpoint`-th pair (t_s, t_{s+1}); the backward recomputes each segment of
t's from its checkpoint, runs the adjoint recurrence through it and adds the
segment's outer products with one SDDMM over all its columns.

Values are passed as a device tensor in the library's value layout (slot
order, row-major blocks; complex128 for complex matrices).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi

_vp = C.c_void_p


def _ptr(t: torch.Tensor) -> _vp:
    return _vp(t.data_ptr())


def _stream() -> _vp:
    return _vp(torch.cuda.current_stream().cuda_stream)


def _mv_args(X: torch.Tensor):
    """(k, ld) of a device vector (N,) or row-major multivector (N, k)."""
    if X.dim() == 1:
        return 1, 1
    assert X.stride(1) == 1, "multivectors must be row-major"
    return X.shape[1], X.stride(0)


def _padded(X: torch.Tensor) -> torch.Tensor:
    """A row-major copy whose rows span a multiple of 16 bytes (the apply's
    multivector rule); vectors pass through."""
    if X.dim() == 1:
        return X.contiguous()
    es = X.element_size()
    k = X.shape[1]
    ld = ((k * es + 15) // 16) * 16 // es
    if X.is_contiguous() and ld == k:
        return X
    out = torch.zeros((X.shape[0], ld), dtype=X.dtype, device=X.device)
    out[:, :k] = X
    return out[:, :k]


def _set_values(op: "_capi.DeviceMatrix", values: torch.Tensor) -> None:
    _capi.call("vbg_matrix_set_values_device", op.h, _ptr(values.contiguous()), _stream())


def _apply(op, X: torch.Tensor, adjoint: bool = False) -> torch.Tensor:
    X = _padded(X)
    Y = torch.zeros_like(X) if X.dim() == 1 else torch.zeros(X.shape[0], X.stride(0), dtype=X.dtype,
                                                             device=X.device)[:, :X.shape[1]]
    k, ld = _mv_args(X)
    if X.dim() == 1:
        _capi.call("vbg_spmv_adjoint" if adjoint else "vbg_spmv", op.h, _ptr(X), _ptr(Y), _stream())
    else:
        _capi.call("vbg_spmm_adjoint" if adjoint else "vbg_spmm", op.h, k, ld, _ptr(X), _ptr(Y), _stream())
    return Y


def _sddmm(op, G: torch.Tensor, X: torch.Tensor, out: torch.Tensor, alpha: complex = 1.0) -> None:
    G = G.contiguous()
    X = X.contiguous()
    k, ld = _mv_args(G)
    a = complex(alpha)
    _capi.call("vbg_sddmm", op.h, k, ld, _ptr(G), _ptr(X), a.real, a.imag, _ptr(out), _stream())


class SparseApply(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, X, op):
        _set_values(op, values)
        Y = _apply(op, X)
        ctx.op = op
        ctx.save_for_backward(values, X)
        return Y

    @staticmethod
    def backward(ctx, gY):
        values, X = ctx.saved_tensors
        op = ctx.op
        _set_values(op, values)
        gV = gX = None
        if ctx.needs_input_grad[1]:
            gX = _apply(op, gY, adjoint=True)
        if ctx.needs_input_grad[0]:
            gV = torch.zeros_like(values)
            _sddmm(op, gY, X, gV)
        return gV, gX, None


def sparse_apply(values: torch.Tensor, X: torch.Tensor, op) -> torch.Tensor:
    """Y = A X with A = (op's pattern, `values`); differentiable in values and X."""
    return SparseApply.apply(values, X, op)


def _cheb_step(op, scale, center, X, Xprev, first: bool, acc=None, coef=0.0, dot_with=None, dots=None):
    """Y = H~ X (first) or 2 H~ X - Xprev; acc += coef * Y; dots as vbg_cheb_step."""
    k, ld = _mv_args(X)
    # the kernels write whole padded rows (pad lanes stay zero when X's are)
    Y = torch.empty_like(X) if X.dim() == 1 else torch.empty(X.shape[0], ld, dtype=X.dtype,
                                                             device=X.device)[:, :k]
    alpha = (1.0 if first else 2.0) / scale
    beta = -(1.0 if first else 2.0) * center / scale
    gamma = 0.0 if first else -1.0
    c = complex(coef)
    _capi.call("vbg_cheb_step", op.h, k, ld, alpha, beta, gamma, _ptr(X), _ptr(Xprev) if Xprev is not None else None,
               _ptr(Y), _ptr(dot_with) if dot_with is not None else None, _ptr(dots) if dots is not None else None,
               _ptr(acc) if acc is not None else None, c.real, c.imag, _stream())
    return Y


def _adj_step(op, scale, center, a1, a2, w, acc, scratch):
    """acc += w H~^H a1 - a2 in one fused adjoint apply (vbg_cheb_step_adjoint;
    scratch receives the added term)."""
    k, ld = _mv_args(a1)
    _capi.call("vbg_cheb_step_adjoint", op.h, k, ld, w / scale, -w * float(np.real(center)) / scale,
               0.0 if a2 is None else -1.0, _ptr(a1), _ptr(a2) if a2 is not None else None, _ptr(scratch), None,
               None, _ptr(acc), 1.0, 0.0, _stream())


def _cheb_forward(op, scale, center, v, coeffs, K, want_moments):
    """psi = sum_n coeffs[n] t_n (if coeffs is not None), moments
    mu_n = Re <v, t_n> (if want_moments), and the checkpoints."""
    M = len(coeffs) if coeffs is not None else want_moments
    dev = v.device
    v = _padded(v)
    if coeffs is not None and not want_moments:
        return _cheb_series(op, scale, center, v, coeffs, K)
    psi = None
    if coeffs is not None:
        psi = torch.zeros_like(v) if v.dim() == 1 else torch.zeros(v.shape[0], v.stride(0), dtype=v.dtype,
                                                                   device=dev)[:, :v.shape[1]]
        psi.add_(v, alpha=complex(coeffs[0]) if v.is_complex() else float(np.real(coeffs[0])))
    mu = torch.zeros(M, dtype=torch.float64, device=dev) if want_moments else None
    dots = torch.zeros(2, dtype=torch.float64, device=dev)
    if want_moments:
        mu[0] = torch.sum((v.conj() * v).real) if v.is_complex() else torch.sum(v * v)
    ckpt = {0: (v, None)}
    t_prev, t = None, v
    for n in range(1, M):
        coef = coeffs[n] if coeffs is not None else 0.0
        t_next = _cheb_step(op, scale, center, t, t_prev, n == 1, acc=psi, coef=coef,
                            dot_with=v if want_moments else None, dots=dots if want_moments else None)
        if want_moments:
            mu[n] = dots[0]
        t_prev, t = t, t_next
        if n % K == 0:
            ckpt[n] = (t, t_prev)
    return psi, mu, ckpt


def _cheb_series(op, scale, center, v, coeffs, K):
    """psi = sum_n coeffs[n] t_n and the checkpoints in one library call
    (vbg_cheb_series): the recurrence runs on the library's three working
    vectors, the pairs (t_n, t_{n-1}) of n = K, 2K, ... are copied into one
    preallocated block."""
    M = len(coeffs)
    k, ld = _mv_args(v)
    n_ck = (M - 1) // K
    if v.dim() == 1:
        psi = torch.empty_like(v)
        store = torch.empty((max(2 * n_ck, 1), v.shape[0]), dtype=v.dtype, device=v.device)
        views = [store[i] for i in range(2 * n_ck)]
    else:
        psi = torch.empty((v.shape[0], ld), dtype=v.dtype, device=v.device)[:, :k]
        store = torch.empty((max(2 * n_ck, 1), v.shape[0], ld), dtype=v.dtype, device=v.device)
        views = [store[i, :, :k] for i in range(2 * n_ck)]
    c = np.ascontiguousarray(np.stack([np.real(coeffs), np.imag(coeffs)], axis=1), dtype=np.float64)
    _capi.call("vbg_cheb_series", op.h, k, ld, _ptr(v), M, c.ctypes.data_as(_vp), float(scale), float(center),
               _ptr(psi), K, _ptr(store), _stream())
    ckpt = {0: (v, None)}
    for j in range(n_ck):
        ckpt[(j + 1) * K] = (views[2 * j], views[2 * j + 1])
    return psi, None, ckpt


def _cheb_backward(op, scale, center, v, M, K, ckpt, source):
    """Adjoint recurrence; returns (dL/dH~* on the pattern as a value array,
    a_0).  source(n) -> s_n (tensor shaped like v, or None)."""
    dH = torch.zeros(op.nnz, dtype=v.dtype if v.is_complex() else torch.float64, device=v.device)
    a1 = a2 = None  # a_{n+1}, a_{n+2}
    scratch = torch.empty_like(v) if v.dim() == 1 else torch.empty(v.shape[0], v.stride(0), dtype=v.dtype,
                                                                   device=v.device)[:, :v.shape[1]]
    seg_starts = list(range(0, M, K))
    for s0 in reversed(seg_starts):
        s1 = min(s0 + K, M)
        # recompute t_{s0} .. t_{s1 - 1}
        t, t_prev = ckpt[s0]
        ts = [t]
        for n in range(s0 + 1, s1):
            t_next = _cheb_step(op, scale, center, t, t_prev, n == 1)
            t_prev, t = t, t_next
            ts.append(t)
        us, tcols = [], []
        for n in range(s1 - 1, s0 - 1, -1):
            w = 1.0 if n == 0 else 2.0
            a = source(n)  # a fresh tensor (or None)
            if a is None:
                a = torch.zeros_like(v) if v.dim() == 1 else torch.zeros(v.shape[0], v.stride(0), dtype=v.dtype,
                                                                         device=v.device)[:, :v.shape[1]]
            elif v.dim() > 1 and a.stride(0) != v.stride(0):
                a = _padded(a)  # a padded copy
            if a1 is not None:
                # a_n = s_n + w H~^H a_{n+1} - a_{n+2}
                _adj_step(op, scale, center, a1, a2, w, a, scratch)
                us.append(a1 if n > 0 else a1 * 0.5)  # columns carry w / 2 (the SDDMM's alpha is 2)
                tcols.append(ts[n - s0])
            a2, a1 = a1, a
        if us:
            G = torch.stack(us, dim=-1) if v.dim() == 1 else torch.cat(us, dim=1)
            Xc = torch.stack(tcols, dim=-1) if v.dim() == 1 else torch.cat(tcols, dim=1)
            _sddmm(op, G, Xc, dH, alpha=2.0)
    return dH / scale, a1


class ChebyshevPropagation(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, psi0, op, coeffs, scale, center, checkpoint):
        _set_values(op, values)
        psi, _, ckpt = _cheb_forward(op, scale, center, psi0, coeffs, checkpoint, False)
        ctx.op, ctx.coeffs, ctx.scale, ctx.center, ctx.K = op, coeffs, scale, center, checkpoint
        ctx.ckpt = ckpt
        ctx.save_for_backward(values, psi0)
        return psi

    @staticmethod
    def backward(ctx, g):
        values, psi0 = ctx.saved_tensors
        op = ctx.op
        _set_values(op, values)
        coeffs = ctx.coeffs
        g = _padded(g)

        def source(n):
            return g * np.conj(coeffs[n])

        dH, a0 = _cheb_backward(op, ctx.scale, ctx.center, _padded(psi0), len(coeffs), ctx.K, ctx.ckpt, source)
        ctx.ckpt = None
        gV = dH if ctx.needs_input_grad[0] else None
        gpsi = a0 if ctx.needs_input_grad[1] else None
        return gV, gpsi, None, None, None, None, None


def chebyshev_coefficients(scale: float, dt: float, num_terms: int) -> np.ndarray:
    """c_n = (2 - delta_n0) (-i)^n J_n(scale dt): exp(-i H dt) on H / scale
    (examples/ex09_graphene_dynamics.py:102-133)."""
    from scipy.special import jv

    n = np.arange(num_terms)
    return np.where(n == 0, 1.0, 2.0) * ((-1j) ** n) * jv(n, scale * dt)


def chebyshev_propagate(values: torch.Tensor, psi0: torch.Tensor, op, dt: float, scale: float,
                        center: float = 0.0, num_terms: int = 256, checkpoint: int = 16) -> torch.Tensor:
    """psi(dt) = exp(-i H dt) psi0 by a `num_terms`-term Chebyshev expansion of
    H~ = (H - center) / scale (spectrum of H inside [center - scale,
    center + scale]); differentiable in values and psi0 (complex128)."""
    coeffs = chebyshev_coefficients(scale, dt, num_terms)
    psi = ChebyshevPropagation.apply(values, psi0, op, coeffs, float(scale), float(center), int(checkpoint))
    if center:
        psi = psi * np.exp(-1j * center * dt)
    return psi


class KPMMoments(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, V, op, M, scale, center, checkpoint):
        _set_values(op, values)
        _, mu, ckpt = _cheb_forward(op, scale, center, V, None, checkpoint, int(M))
        ctx.op, ctx.M, ctx.scale, ctx.center, ctx.K, ctx.ckpt = op, int(M), scale, center, checkpoint, ckpt
        ctx.save_for_backward(values, V)
        return mu

    @staticmethod
    def backward(ctx, gmu):
        values, V = ctx.saved_tensors
        op = ctx.op
        _set_values(op, values)
        Vp = _padded(V)
        gm = gmu.detach().cpu().numpy()

        def source(n):
            # mu_0 = <v, v> does not depend on H; mu_n = <v, t_n> for n >= 1
            return None if n == 0 or gm[n] == 0.0 else Vp * float(gm[n])

        dH, _ = _cheb_backward(op, ctx.scale, ctx.center, Vp, ctx.M, ctx.K, ctx.ckpt, source)
        ctx.ckpt = None
        return (dH if ctx.needs_input_grad[0] else None), None, None, None, None, None, None


def kpm_moments(values: torch.Tensor, V: torch.Tensor, op, num_moments: int, scale: float = 1.0,
                center: float = 0.0, checkpoint: int = 16) -> torch.Tensor:
    """Unnormalised moments mu_n = sum_r <v_r, T_n(H~) v_r> (plain
    recurrence) of a real symmetric H; differentiable in values."""
    return KPMMoments.apply(values, V, op, int(num_moments), float(scale), float(center), int(checkpoint))

"""Kernel polynomial method helpers (host side).

Mirrors the reference's scalar helpers -- ``jackson_kernel``,
``compute_kpm_coeffs`` (vbcsr/utils.py:5-68) and the DOS reconstruction on
Chebyshev nodes (examples/inp_nanocrystal_dos/kpm.py:132-145) -- and drives
the device moment loop (``vbg_kpm_moments``) for :func:`kpm_moments` and
:func:`compute_kpm_dos`.
"""
from __future__ import annotations

import numpy as np


def jackson_kernel(N: int) -> np.ndarray:
    """Jackson damping g_n, n = 0..N-1 (vbcsr/utils.py:5-17):
    g_n = [(N - n + 1) cos(pi n / (N + 1)) + sin(pi n / (N + 1)) cot(pi / (N + 1))] / (N + 1)."""
    if N <= 0:
        raise ValueError("num_moments must be positive")
    n = np.arange(N, dtype=np.float64)
    th = np.pi / (N + 1)
    return ((N - n + 1) * np.cos(th * n) + np.sin(th * n) / np.tan(th)) / (N + 1)


def compute_kpm_coeffs(n_kpm: int, func) -> np.ndarray:
    """Jackson-damped Chebyshev coefficients of a scalar function on [-1, 1]
    from 2 n_kpm samples on the Chebyshev grid (vbcsr/utils.py:35-68)."""
    k = np.arange(2 * n_kpm)
    x_k = np.cos(np.pi * k / n_kpm)
    coeffs = np.fft.fft(func(x_k)).real[:n_kpm] / n_kpm
    damped = coeffs * jackson_kernel(n_kpm)
    damped[0] /= 2.0
    return damped


def chebyshev_nodes(num_points: int) -> np.ndarray:
    """Ascending Gauss-Chebyshev nodes x_j = -cos(pi (j + 1/2) / P)."""
    theta = np.pi * (np.arange(num_points) + 0.5) / num_points
    return -np.cos(theta)


def dos_from_moments(mu: np.ndarray, num_points: int = 2000, kernel: bool = True, x: np.ndarray | None = None):
    """DOS rho(x) = [g_0 mu_0 + 2 sum_n g_n mu_n T_n(x)] / (pi sqrt(1 - x^2)) on
    Chebyshev nodes (or the given x), mu already normalised."""
    mu = np.asarray(mu, dtype=np.float64)
    M = len(mu)
    g = jackson_kernel(M) if kernel else np.ones(M)
    if x is None:
        x = chebyshev_nodes(num_points)
    t0 = np.ones_like(x)
    t1 = x.copy()
    rho = g[0] * mu[0] * t0
    if M > 1:
        rho = rho + 2.0 * g[1] * mu[1] * t1
    for n in range(2, M):
        t2 = 2.0 * x * t1 - t0
        rho += 2.0 * g[n] * mu[n] * t2
        t0, t1 = t1, t2
    rho /= np.pi * np.sqrt(np.maximum(1.0e-15, 1.0 - x * x))
    return x, rho


def batched_kpm_moments(hamiltonians, num_moments: int, num_random_vecs: int = 16, precision: str = "fp64",
                        seed: int = 0, two_moment: bool = True, use_graph: bool = True, vectors=None):
    """Unnormalised KPM moments of many independent real symmetric
    Hamiltonians (already rescaled into [-1, 1], BlockCSR) in one batched
    device recurrence: the matrices are stacked block-diagonally and every
    Chebyshev step is one apply over all of them (vbg_kpm_moments_batched).
    Random vectors: +-1, num_random_vecs per Hamiltonian from `seed`, unless
    `vectors` (list of N_i x R arrays) is given.  Returns (moments
    [count x num_moments], per-Hamiltonian N)."""
    import ctypes as C

    import torch

    from . import _capi
    from .workloads import block_diagonal

    H, seg = block_diagonal(list(hamiltonians))
    R = num_random_vecs if vectors is None else vectors[0].shape[1]
    if vectors is None:
        rng = np.random.default_rng(seed)
        V = np.where(rng.random((H.N, R)) < 0.5, -1.0, 1.0)
    else:
        V = np.concatenate(vectors, axis=0)
    dm = _capi.DeviceMatrix.create(H.block_sizes, H.row_ptr, H.col_ind, H.values)
    ld = ((R * 8 + 63) // 64) * 8
    V0 = torch.zeros((H.N, ld), dtype=torch.float64, device="cuda")
    V0[:, :R] = torch.from_numpy(V).cuda()
    mu = torch.zeros((len(seg) - 1, num_moments), dtype=torch.float64, device="cuda")
    segc = np.ascontiguousarray(seg, dtype=np.int32)
    prec = {"fp64": 0, "fp32": 1}[precision]
    _capi.call("vbg_kpm_moments_batched", dm.h, len(seg) - 1, segc.ctypes.data_as(C.POINTER(C.c_int)), R, ld,
               C.c_void_p(V0.data_ptr()), int(num_moments), prec, int(two_moment), int(use_graph),
               C.c_void_p(mu.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    sizes = [int(np.sum(h.block_sizes)) for h in hamiltonians]
    return mu.cpu().numpy(), np.asarray(sizes)

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

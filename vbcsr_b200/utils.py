"""Chebyshev / KPM helpers with the reference's names and meaning
(vbcsr/utils.py:5-126, examples/ex08_graphene_dos.py:66-156).

``kpm_apply`` and ``compute_kpm_dos`` keep the reference's recurrences; their
inner loop runs as one fused device step per Chebyshev term (vbg_cheb_step /
vbg_kpm_moments) instead of the reference's separate mult / axpby / axpy /
bdot passes with temporaries.
"""
from __future__ import annotations

import numpy as np

from .kpm import chebyshev_nodes, compute_kpm_coeffs, dos_from_moments, jackson_kernel  # noqa: F401
from .multivector import DistMultiVector


def fermi_dirac(E, beta, mu):
    """Fermi-Dirac occupation expit(-beta (E - mu)) (vbcsr/utils.py:20-26)."""
    from scipy.special import expit

    return expit(-beta * (E - mu))


def gaussian(E, mu):
    return np.exp(-(E - mu) ** 2)


def kpm_apply(matrix, vector, coeffs, scale, center):
    """y = sum_n c_n T_n((H - center) / scale) v  (vbcsr/utils.py:71-126).

    Recurrence: v0 = v, v1 = (H v0 - center v0) / scale,
    v_{n+1} = 2 (H v_n - center v_n) / scale - v_{n-1}; each step is one fused
    device pass that also accumulates y += c_n v_{n+1}, and the whole series
    runs inside one library call (vbg_cheb_series) on the library's own
    working vectors."""
    n_kpm = len(coeffs)
    if n_kpm == 0:
        res = vector.duplicate()
        res.set_constant(0.0)
        return res
    y = vector.duplicate()
    y.scale(coeffs[0])  # c_0 v; also the scalar-type check of the vector's scale
    if n_kpm == 1:
        return y
    matrix._core.cheb_series(vector._core, np.asarray(coeffs, dtype=np.complex128), float(scale), float(center),
                             y._core)
    return y


def kpm_moments(H_scaled, vectors: DistMultiVector, num_moments: int, precision: str = "fp64",
                two_moment: bool = True, use_graph: bool = True) -> np.ndarray:
    """Unnormalised moments mu_n = sum_r <r | T_n(H) | r> of an already
    rescaled real symmetric matrix, all recurrence work on the device.
    precision "fp64" (plain) or "fp32" (FP32 storage/arithmetic, FP64 sums)."""
    prec = {"fp64": 0, "fp32": 1}[precision]
    return np.asarray(H_scaled._core.kpm_moments(vectors._core, int(num_moments), prec, bool(two_moment),
                                                 bool(use_graph)))


def compute_kpm_dos(H, num_moments: int = 200, num_random_vecs: int = 10, E_bound: float | None = None,
                    num_points: int = 400, seed: int | None = None, precision: str = "fp64",
                    two_moment: bool = True, vectors=None):
    """DOS by KPM, the procedure of examples/ex08_graphene_dos.py:66-156:
    scale H by 1 / E_bound, moments mu_n = sum_r <r|T_n|r> / (R N) over random
    vectors, Jackson damping, reconstruction rho(E).  Returns
    (energies, dos, moments).  Vectors: +-1 (Rademacher) from `seed` unless
    given (numpy N x R or a DistMultiVector).  Energies on Chebyshev nodes of
    the scaled interval (interior points; ex08's linspace includes the +-1
    endpoints where rho diverges)."""
    if E_bound is None:
        raise ValueError("E_bound (half-width of the spectrum) is required")
    Hs = H.duplicate()
    Hs.scale(1.0 / E_bound)
    N = H.shape[0]
    if vectors is None:
        rng = np.random.default_rng(seed)
        vectors = np.where(rng.random((N, num_random_vecs)) < 0.5, -1.0, 1.0)
    if isinstance(vectors, np.ndarray):
        mv = H.create_multivector(vectors.shape[1])
        mv.from_numpy(vectors.astype(H.dtype))
        vectors = mv
    R = vectors.num_vectors
    mu = kpm_moments(Hs, vectors, num_moments, precision=precision, two_moment=two_moment) / (R * N)
    x, rho = dos_from_moments(mu, num_points)
    return x * E_bound, rho / E_bound, mu

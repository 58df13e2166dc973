"""Chebyshev time propagation psi(t) = exp(-i H t) psi0
(examples/ex09_graphene_dynamics.py:102-133 of the reference): coefficients
c_n = (2 - delta_n0) (-i)^n J_n(E_max dt) on H / E_max, evaluated by the
fused device recurrence of :func:`vbcsr_b200.utils.kpm_apply`."""
from __future__ import annotations

import numpy as np

from .utils import kpm_apply


def chebyshev_coefficients(E_max: float, dt: float, num_moments: int) -> np.ndarray:
    from scipy.special import jv

    n = np.arange(num_moments)
    return np.where(n == 0, 1.0, 2.0) * ((-1j) ** n) * jv(n, E_max * dt)


def propagate_chebyshev(H, psi, dt: float, num_moments: int = 50, E_max: float | None = None,
                        E_center: float = 0.0) -> np.ndarray:
    """psi(dt) for a complex Hermitian H (VBCSR, complex128); psi a numpy array
    or DistVector.  E_max: spectral half-width (required); a non-zero
    E_center multiplies the result by exp(-i E_center dt)."""
    if E_max is None:
        raise ValueError("E_max (spectral half-width) is required")
    coeffs = chebyshev_coefficients(E_max, dt, num_moments)
    if isinstance(psi, np.ndarray):
        v = H.create_vector()
        v.from_numpy(psi.astype(H.dtype))
    else:
        v = psi
    y = kpm_apply(H, v, coeffs, E_max, E_center)
    out = y.to_numpy().copy()
    if E_center:
        out *= np.exp(-1j * E_center * dt)
    return out

"""McWeeny purification P <- 3 P^2 - 2 P^3 with thresholded SpGEMM
(README.md:22-33 and examples/ex07_graphene_purification.py:136-173 of the
reference), every product, filter and reduction on the device.

Beside the reference's plain FP64 loop, a mixed-precision variant: the bulk
iterations multiply in FP32 (the operands' FP32 copies, FP32 accumulation;
vbg_spgemm_ex), while FP64 stays on the device for what decides the answer:
the trace of every iterate and the optional electron-count correction, the
idempotency residual ||P^2 - P||_F, and the last `polish` iterations, which
run in FP64 and remove the FP32 rounding the bulk iterations left behind
(McWeeny's map contracts errors quadratically near an idempotent matrix).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class PurifyResult:
    P: object
    nnzb: list = field(default_factory=list)      # stored blocks after each iteration
    residual: list = field(default_factory=list)  # ||P_k^2 - P_k||_F of the iterate entering step k
    trace: list = field(default_factory=list)     # tr(P) after each iteration (and any correction)
    precision: list = field(default_factory=list)  # "fp32" / "fp64" per iteration


def frobenius(M) -> float:
    """||M||_F, reduced in FP64 on the device."""
    return float(M._core.norm_fro_fp64())


def trace(M) -> float:
    """Re tr(M), reduced in FP64 on the device."""
    return float(np.real(M._core.trace_fp64()))


def mcweeny_purify(H, threshold: float = 1e-5, iterations: int = 10, alpha: float | None = None,
                   beta: float | None = None, filter_each: bool = True, track: bool = True,
                   hermitian: bool = False, precision: str = "fp64", polish: int = 2,
                   electrons: float | None = None) -> PurifyResult:
    """P0 = alpha H + beta I (defaults: the reference README's 0.1 / 0.5), then
    `iterations` steps of P2 = P.spmm(P, thr); P3 = P2.spmm(P, thr);
    P = 3 P2 - 2 P3; P.filter_blocks(thr).

    precision: "fp64" (the reference's loop) or "fp32" -- the first
      iterations - polish products in FP32, the last `polish` in FP64.
    electrons: if given, after every FP32 iteration the diagonal is shifted
      by (electrons - tr P) / N so that the trace keeps the electron count
      (computed in FP64 on the device).
    track: record the block count, tr(P) and ||P^2 - P||_F of each iterate
      (from the P^2 the step computes anyway), all reduced on the device.
    hermitian (H Hermitian): both products through spmm_hermitian -- P2 and
      P3 are polynomials in P, so Hermitian -- which multiplies the upper
      block triangle only and keeps every iterate exactly Hermitian."""
    if precision not in ("fp64", "fp32"):
        raise ValueError("precision must be 'fp64' or 'fp32'")
    P = H.copy()
    P.scale(0.1 if alpha is None else alpha)
    P.shift(0.5 if beta is None else beta)
    N = P.shape[0]
    out = PurifyResult(P=P)
    wrap = type(P)._wrap_core
    for it in range(iterations):
        fp32 = precision == "fp32" and it < iterations - polish
        prec = 1 if fp32 else 0
        P2 = wrap(P._core.spmm_ex(P._core, threshold, prec, hermitian), P.dtype, P.comm)
        if track:
            D = P2.duplicate()
            D.axpby(-1.0, P, 1.0)
            out.residual.append(frobenius(D))
            del D
        P3 = wrap(P2._core.spmm_ex(P._core, threshold, prec, hermitian), P.dtype, P.comm)
        P3.axpby(3.0, P2, -2.0)  # P3 <- 3 P2 - 2 P3
        P = P3
        if filter_each:
            P.filter_blocks(threshold)
        if fp32 and electrons is not None:
            P.shift((float(electrons) - trace(P)) / N)
        if track:
            out.nnzb.append(P.local_block_nnz)
            out.trace.append(trace(P))
            out.precision.append("fp32" if fp32 else "fp64")
    out.P = P
    return out

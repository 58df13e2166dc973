"""McWeeny purification P <- 3 P^2 - 2 P^3 with thresholded SpGEMM
(README.md:22-33 and examples/ex07_graphene_purification.py:136-173 of the
reference), every product and filter on the device."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class PurifyResult:
    P: object
    nnzb: list = field(default_factory=list)      # stored blocks after each iteration
    residual: list = field(default_factory=list)  # ||P_k^2 - P_k||_F of the iterate entering step k
    trace: list = field(default_factory=list)     # tr(P) after each iteration


def frobenius(M) -> float:
    v = M.get_values()
    return float(np.sqrt(np.sum(np.abs(v) ** 2)))


def trace(M) -> float:
    v = M.get_values()
    rp, ci = M.row_ptr, M.col_ind
    bsz = np.asarray(M.graph.block_sizes)
    tr = 0.0
    off = 0
    for i in range(len(bsz)):
        for s in range(rp[i], rp[i + 1]):
            j = ci[s]
            r, c = bsz[i], bsz[j]
            if j == i:
                tr += float(np.real(np.trace(v[off:off + r * c].reshape(r, c))))
            off += r * c
    return tr


def mcweeny_purify(H, threshold: float = 1e-5, iterations: int = 10, alpha: float | None = None,
                   beta: float | None = None, filter_each: bool = True, track: bool = True,
                   hermitian: bool = False) -> PurifyResult:
    """P0 = alpha H + beta I (defaults: the reference README's 0.1 / 0.5), then
    `iterations` steps of P2 = P.spmm(P, thr); P3 = P2.spmm(P, thr);
    P = 3 P2 - 2 P3; P.filter_blocks(thr).  With `track`, records the block
    count, tr(P) and the idempotency residual ||P^2 - P||_F of each iterate
    (from the P^2 the step computes anyway).  `hermitian` (H Hermitian):
    both products through spmm_hermitian -- P2 and P3 are polynomials in P,
    so Hermitian -- which multiplies the upper block triangle only and keeps
    every iterate exactly Hermitian."""
    P = H.copy()
    P.scale(0.1 if alpha is None else alpha)
    P.shift(0.5 if beta is None else beta)
    out = PurifyResult(P=P)
    for _ in range(iterations):
        mul = P.spmm_hermitian if hermitian else P.spmm
        P2 = mul(P, threshold=threshold)
        if track:
            D = P2.duplicate()
            D.axpby(-1.0, P, 1.0)
            out.residual.append(frobenius(D))
        P3 = (P2.spmm_hermitian if hermitian else P2.spmm)(P, threshold=threshold)
        P = 3.0 * P2 - 2.0 * P3
        if filter_each:
            P.filter_blocks(threshold)
        if track:
            out.nnzb.append(P.local_block_nnz)
            out.trace.append(trace(P))
    out.P = P
    return out

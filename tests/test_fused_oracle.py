"""The oracle's restatement of the reference's fused triple products
(square_polynomial_upper, rarh_upper, rhar_upper; vbcsr/core/block_csr.hpp
:1803-1853) pinned against the reference core itself, on CPU: the patterns
must be identical except for blocks whose norm lies within 1e-10 relative of
the threshold, the values equal to 1e-12 of the largest."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W


def blocks(H):
    off = H.slot_offsets()
    rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
    return {(int(i), int(j)): H.values[off[s]:off[s + 1]] for s, (i, j) in enumerate(zip(rows, H.col_ind))}


def assert_same_product(got, want, thr, tol=1e-12, band=1e-10):
    gb, wb = blocks(got), blocks(want)
    for key in set(gb) ^ set(wb):
        v = gb.get(key, wb.get(key))
        nrm = float(np.sqrt(np.sum(np.abs(v) ** 2)))
        assert thr > 0 and abs(nrm - thr) <= band * thr, (key, nrm, thr)
    common = set(gb) & set(wb)
    if not common:
        return
    scale = max(np.abs(v).max() for v in wb.values())
    err = max(np.abs(gb[k] - wb[k]).max() for k in common)
    assert err <= tol * scale, err / scale


def hermitian_cases():
    H, _ = W.tmd_lattice(5, seed=21)
    yield "tmd", H
    Hc, _ = W.tmd_lattice(4, seed=22, bond_phase=True)
    yield "tmd_complex", Hc
    yield "banded", W.banded_decaying(80, neighbours=5, band=6, decay=1.5, seed=23)


def perturbed(H, seed):
    """H's pattern, values no longer Hermitian."""
    from vbcsr_b200.workloads import BlockCSR

    rng = np.random.default_rng(seed)
    v = H.values * (1.0 + 0.3 * rng.normal(size=H.values.shape))
    return BlockCSR(H.block_sizes.copy(), H.row_ptr.copy(), H.col_ind.copy(), v)


def scaled_square(oracle, H):
    """B = H H / max|.| (Hermitian, denser, same block sizes)."""
    from vbcsr_b200.workloads import BlockCSR

    S, _ = oracle.spgemm(H, H, 0.0)
    return BlockCSR(S.block_sizes, S.row_ptr, S.col_ind, S.values / np.abs(S.values).max())


THRESHOLDS = [0.0, 1e-3, 1e-2, 3e-2, 1e-1]


@pytest.mark.parametrize("rel_thr", THRESHOLDS)
def test_square_polynomial_oracle_vs_reference(oracle, reference, rel_thr):
    for name, H in hermitian_cases():
        thr = rel_thr * np.abs(H.values).max()
        cplx = np.iscomplexobj(H.values)
        c2, c1, c0 = (0.375 + 0.1j, -1.25, 1.875 - 0.2j) if cplx else (0.375, -1.25, 1.875)
        got = oracle.square_polynomial_upper(H, c2, c1, c0, thr)
        want = reference.matrix(H).square_polynomial_upper(c2, c1, c0, thr).to_blockcsr()
        assert_same_product(got, want, thr)


@pytest.mark.parametrize("rel_thr", THRESHOLDS)
def test_rarh_oracle_vs_reference(oracle, reference, rel_thr):
    for name, H in hermitian_cases():
        B = scaled_square(oracle, H)
        thr = rel_thr * np.abs(H.values).max()
        got = oracle.rarh_upper(H, B, thr)
        want = reference.matrix(H).rarh_upper(reference.matrix(B), thr).to_blockcsr()
        assert_same_product(got, want, thr)


@pytest.mark.parametrize("rel_thr", THRESHOLDS)
def test_rhar_oracle_vs_reference(oracle, reference, rel_thr):
    for name, H in hermitian_cases():
        A = perturbed(H, 5)
        B = scaled_square(oracle, H)
        thr = rel_thr * np.abs(H.values).max()
        got = oracle.rhar_upper(A, B, thr)
        want = reference.matrix(A).rhar_upper(reference.matrix(B), thr).to_blockcsr()
        assert_same_product(got, want, thr)


def test_fused_products_reduce_to_dense(oracle):
    """At threshold 0 nothing is skipped: the products equal the dense
    upper triangles of c2 H^2 + c1 H + c0 I, H B H^H and A^H B A."""
    H, _ = W.tmd_lattice(3, seed=24, bond_phase=True)
    A = perturbed(H, 6)
    B = scaled_square(oracle, H)
    so = H.scalar_offsets()
    Hd, Ad, Bd = H.to_dense(), A.to_dense(), B.to_dense()

    def upper(D):
        U = D.copy()
        for i in range(H.n):
            U[so[i]:so[i + 1], :so[i]] = 0.0
        return U

    sp = oracle.square_polynomial_upper(H, 0.5, -1.0, 2.0, 0.0).to_dense()
    assert np.abs(sp - upper(0.5 * Hd @ Hd - Hd + 2.0 * np.eye(H.N))).max() < 1e-12
    assert np.abs(oracle.rarh_upper(H, B, 0.0).to_dense() - upper(Hd @ Bd @ Hd.conj().T)).max() < 1e-12
    assert np.abs(oracle.rhar_upper(A, B, 0.0).to_dense() - upper(Ad.conj().T @ Bd @ Ad)).max() < 1e-12

"""The fused triple products on the GPU (vbg_square_polynomial_upper,
vbg_rarh_upper, vbg_rhar_upper) against the oracle's restatement and, where
it is built, the reference core itself: patterns identical except for blocks
whose norm lies within 1e-10 relative of the threshold, values to 1e-12 of
the largest; thresholds from 0 to 10 % of the largest entry, real and
complex, the completed Hermitian matrix against the dense product."""
import numpy as np
import pytest

from .test_fused_oracle import THRESHOLDS, assert_same_product, hermitian_cases, perturbed, scaled_square

pytestmark = pytest.mark.gpu


def _dmat(H):
    from . import _gpu

    return _gpu.dmat(H)


@pytest.mark.parametrize("rel_thr", THRESHOLDS)
def test_square_polynomial_gpu(oracle, dev, rel_thr):
    for name, H in hermitian_cases():
        thr = rel_thr * np.abs(H.values).max()
        cplx = np.iscomplexobj(H.values)
        c2, c1, c0 = (0.375 + 0.1j, -1.25, 1.875 - 0.2j) if cplx else (0.375, -1.25, 1.875)
        got = _dmat(H).square_polynomial_upper(c2, c1, c0, thr).to_blockcsr()
        want = oracle.square_polynomial_upper(H, c2, c1, c0, thr)
        assert_same_product(got, want, thr)


@pytest.mark.parametrize("rel_thr", THRESHOLDS)
def test_rarh_gpu(oracle, dev, rel_thr):
    for name, H in hermitian_cases():
        B = scaled_square(oracle, H)
        thr = rel_thr * np.abs(H.values).max()
        got = _dmat(H).rarh_upper(_dmat(B), thr).to_blockcsr()
        assert_same_product(got, oracle.rarh_upper(H, B, thr), thr)


@pytest.mark.parametrize("rel_thr", THRESHOLDS)
def test_rhar_gpu(oracle, dev, rel_thr):
    for name, H in hermitian_cases():
        A = perturbed(H, 5)
        B = scaled_square(oracle, H)
        thr = rel_thr * np.abs(H.values).max()
        got = _dmat(A).rhar_upper(_dmat(B), thr).to_blockcsr()
        assert_same_product(got, oracle.rhar_upper(A, B, thr), thr)


def test_fused_against_reference(oracle, reference, dev):
    """A larger banded case (300 block rows) against the reference core."""
    from vbcsr_b200 import workloads as W

    H = W.banded_decaying(300, neighbours=6, band=10, decay=2.0, seed=31)
    B = scaled_square(oracle, H)
    A = perturbed(H, 7)
    for rel in (0.0, 1e-3, 3e-2):
        thr = rel * np.abs(H.values).max()
        rh, rb, ra = reference.matrix(H), reference.matrix(B), reference.matrix(A)
        assert_same_product(_dmat(H).square_polynomial_upper(0.375, -1.25, 1.875, thr).to_blockcsr(),
                            rh.square_polynomial_upper(0.375, -1.25, 1.875, thr).to_blockcsr(), thr)
        assert_same_product(_dmat(H).rarh_upper(_dmat(B), thr).to_blockcsr(),
                            rh.rarh_upper(rb, thr).to_blockcsr(), thr)
        assert_same_product(_dmat(A).rhar_upper(_dmat(B), thr).to_blockcsr(),
                            ra.rhar_upper(rb, thr).to_blockcsr(), thr)


def test_completed_products_dense(oracle, dev):
    """Threshold 0, completed to the full Hermitian matrix: equal to the
    dense c2 H^2 + c1 H + c0 I, H B H^H and A^H B A."""
    from vbcsr_b200 import workloads as W

    H, _ = W.tmd_lattice(3, seed=24, bond_phase=True)
    A = perturbed(H, 6)
    B = scaled_square(oracle, H)
    Hd, Ad, Bd = H.to_dense(), A.to_dense(), B.to_dense()
    P = _dmat(H).square_polynomial_upper(0.5, -1.0, 2.0, 0.0)
    P.complete_hermitian()
    R = _dmat(H).rarh_upper(_dmat(B), 0.0)
    R.complete_hermitian()
    S = _dmat(A).rhar_upper(_dmat(B), 0.0)
    S.complete_hermitian()
    assert np.abs(P.to_blockcsr().to_dense() - (0.5 * Hd @ Hd - Hd + 2.0 * np.eye(H.N))).max() < 1e-12
    assert np.abs(R.to_blockcsr().to_dense() - Hd @ Bd @ Hd.conj().T).max() < 1e-12
    assert np.abs(S.to_blockcsr().to_dense() - Ad.conj().T @ Bd @ Ad).max() < 1e-12


def test_fused_through_python_api(oracle, dev):
    """The same products through VBCSR (the host core's methods), then
    completed: upper triangles equal the oracle's, completion Hermitian."""
    from vbcsr_b200 import VBCSR
    from vbcsr_b200.workloads import BlockCSR

    for name, H in hermitian_cases():
        B = scaled_square(oracle, H)
        thr = 1e-2 * np.abs(H.values).max()
        dt = H.values.dtype
        vH = VBCSR.from_block_csr(H.block_sizes, H.row_ptr, H.col_ind, H.values, dtype=dt)
        vB = VBCSR.from_block_csr(B.block_sizes, B.row_ptr, B.col_ind, B.values, dtype=dt)

        def bcsr(M):
            return BlockCSR(H.block_sizes, M.row_ptr, M.col_ind, M.get_values())

        P = vH.square_polynomial_upper(0.375, -1.25, 1.875, thr)
        assert_same_product(bcsr(P), oracle.square_polynomial_upper(H, 0.375, -1.25, 1.875, thr), thr)
        R = vH.rarh_upper(vB, thr)
        assert_same_product(bcsr(R), oracle.rarh_upper(H, B, thr), thr)
        F = R.complete_hermitian()
        D = F.to_dense()
        assert np.abs(D - D.conj().T).max() == 0.0
        R.complete_hermitian_inplace()
        assert np.array_equal(R.to_dense(), D)

"""The Python surface of the drop-in on the GPU: the calls a user of the
reference's package makes (vbcsr/matrix.py:505-617,732-744 mult / @ /
_matvec / _matmat / _rmatvec and the SciPy LinearOperator adapter;
vbcsr/vector.py and vbcsr/multivector.py dot / bdot / axpby / scale /
pointwise_mult / set_random; vbcsr/utils.py kpm_apply and the KPM DOS of
examples/ex08_graphene_dos.py:66-156; the Chebyshev propagation of
examples/ex09_graphene_dynamics.py:570-601), each run through this
repository's API on the vbcsr_core host core and compared with the C oracle,
the golden fixtures generated from the reference, or plain numpy on the same
inputs.  Tolerance: 1e-12 relative for FP64 / complex128 values."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W

from .conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12
GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def _vbcsr(H):
    from vbcsr_b200 import VBCSR

    return VBCSR.from_block_csr(H.block_sizes, H.row_ptr, H.col_ind, H.values, dtype=H.values.dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.complex128])
def test_matmul_vector_and_multivector(oracle, dtype):
    H = W.random_pattern(60, 1, 7, 5, seed=31, dtype=dtype)
    A = _vbcsr(H)
    rng = np.random.default_rng(3)
    x = rng.normal(size=H.N).astype(dtype)
    X = rng.normal(size=(H.N, 5)).astype(dtype)
    if dtype == np.complex128:
        x = x + 1j * rng.normal(size=H.N)
        X = X + 1j * rng.normal(size=(H.N, 5))
    from vbcsr_b200 import DistMultiVector, DistVector

    # `A @ ndarray` returns a DistVector / DistMultiVector, as the reference's
    # __matmul__ -> mult does (vbcsr/matrix.py:505-541,732-744)
    y = A @ x
    assert isinstance(y, DistVector) and y.shape == (H.N,)
    assert rel_err(y.to_numpy(), oracle.apply(H, x)) < TOL
    Y = A @ X
    assert isinstance(Y, DistMultiVector) and Y.shape == (H.N, 5)
    assert rel_err(Y.to_numpy(), oracle.apply(H, X)) < TOL
    # the LinearOperator hooks
    assert rel_err(A._matvec(x), oracle.apply(H, x)) < TOL
    assert rel_err(A._matmat(X), oracle.apply(H, X)) < TOL
    assert rel_err(A._rmatvec(x), oracle.apply(H, x, adjoint=True)) < TOL
    assert rel_err(A._rmatmat(X), oracle.apply(H, X, adjoint=True)) < TOL
    # mult into a DistVector / DistMultiVector, and the dense equivalent
    v = A.create_vector()
    v.from_numpy(x)
    w = A.mult(v)
    assert rel_err(w.to_numpy(), H.to_dense() @ x) < TOL
    mv = A.create_multivector(5)
    mv.from_numpy(X)
    out = A.mult(mv)
    assert rel_err(out.to_numpy(), H.to_dense() @ X) < TOL
    # a later host write through the numpy view must reach the device copy
    v.to_numpy()[:] = 2.0 * x
    assert rel_err((A @ v).to_numpy(), 2.0 * (H.to_dense() @ x)) < TOL


def test_linear_operator_cg():
    """SciPy's conjugate gradients through the LinearOperator adapter
    (vbcsr/matrix.py:583-617) on a symmetric positive definite VBCSR matrix."""
    import scipy.sparse.linalg as sla

    H = W.random_symmetric_blocks(120, seed=32)
    W.add_diagonal(H, np.full(H.N, 4.0 * W.gershgorin_bound(H)))
    A = _vbcsr(H)
    assert isinstance(A, sla.LinearOperator)
    b = np.random.default_rng(4).normal(size=H.N)
    x, info = sla.cg(A, b, rtol=1e-12, maxiter=500)
    assert info == 0
    assert np.linalg.norm(H.to_dense() @ x - b) <= 1e-10 * np.linalg.norm(b)
    x_ref = np.linalg.solve(H.to_dense(), b)
    assert rel_err(x, x_ref) < 1e-9


@pytest.mark.parametrize("dtype", [np.float64, np.complex128])
def test_multivector_ops(dtype):
    """DistMultiVector bdot / axpby / axpy / scale / pointwise_mult(_vec) /
    set_constant (vbcsr/core/dist_multivector.hpp:179-314) and DistVector dot
    / axpby / pointwise_mult (dist_vector.hpp:113) against numpy."""
    H = W.random_pattern(40, 2, 6, 4, seed=33, dtype=dtype)
    A = _vbcsr(H)
    rng = np.random.default_rng(5)

    def draw(shape):
        z = rng.normal(size=shape)
        if dtype == np.complex128:
            z = z + 1j * rng.normal(size=shape)
        return z.astype(dtype)

    k = 3
    Xn, Yn, Pn = draw((H.N, k)), draw((H.N, k)), draw((H.N, k))
    X, Y = A.create_multivector(k), A.create_multivector(k)
    X.from_numpy(Xn)
    Y.from_numpy(Yn)
    got = np.asarray(X.bdot(Y))
    want = np.einsum("ij,ij->j", Xn.conj(), Yn)
    assert rel_err(got, want) < TOL
    a, b = (0.7 - 0.2j, 1.3 + 0.4j) if dtype == np.complex128 else (0.7, 1.3)
    Y.axpby(a, X, b)
    Yn = a * Xn + b * Yn
    assert rel_err(Y.to_numpy(), Yn) < TOL
    Y.axpy(a, X)
    Yn = Yn + a * Xn
    assert rel_err(Y.to_numpy(), Yn) < TOL
    Y.scale(b)
    Yn = b * Yn
    assert rel_err(Y.to_numpy(), Yn) < TOL
    P = A.create_multivector(k)
    P.from_numpy(Pn)
    Y.pointwise_mult(P)
    Yn = Yn * Pn
    assert rel_err(Y.to_numpy(), Yn) < TOL
    d = draw(H.N)
    dv = A.create_vector()
    dv.from_numpy(d)
    Y.pointwise_mult(dv)
    Yn = Yn * d[:, None]
    assert rel_err(Y.to_numpy(), Yn) < TOL
    # a device result read back through the view, then an op on the device again
    assert rel_err(np.asarray(Y.bdot(X)), np.einsum("ij,ij->j", Yn.conj(), Xn)) < TOL
    Y.set_constant(2.5)
    assert np.all(Y.to_numpy() == dtype(2.5))
    # DistVector
    xn, yn = draw(H.N), draw(H.N)
    x, y = A.create_vector(), A.create_vector()
    x.from_numpy(xn)
    y.from_numpy(yn)
    assert abs(x.dot(y) - np.vdot(xn, yn)) <= TOL * np.abs(xn).dot(np.abs(yn))
    y.axpby(a, x, b)
    yn = a * xn + b * yn
    assert rel_err(y.to_numpy(), yn) < TOL
    y.pointwise_mult(x)
    yn = yn * xn
    assert rel_err(y.to_numpy(), yn) < TOL
    y.scale(a)
    assert rel_err(y.to_numpy(), a * yn) < TOL


def test_set_random_golden():
    """The device counter-hash fill (vbg_mv_set_random) against the reference
    core's set_random on the same block sizes (random_vectors.hpp:52-160):
    Rademacher values bit-identical, random phases to 1e-15."""
    from vbcsr_b200 import VBCSR

    d = np.load(GOLDEN / "set_random.npz")
    bsz = d["bsz"]
    n = len(bsz)
    rp = np.arange(n + 1, dtype=np.int32)
    ci = np.arange(n, dtype=np.int32)
    vals = np.concatenate([np.eye(b).ravel() for b in bsz])
    A = VBCSR.from_block_csr(bsz, rp, ci, vals)
    mv = A.create_multivector(3)
    mv.set_random(77, True)
    assert np.array_equal(mv.to_numpy(), d["real"])
    mv2 = A.create_multivector(2)
    mv2.set_random(5, normalize=False)
    assert np.array_equal(mv2.to_numpy(), d["real_raw"])
    Z = VBCSR.from_block_csr(bsz, rp, ci, vals.astype(np.complex128), dtype=np.complex128)
    mz = Z.create_multivector(3)
    mz.set_random(77, True)
    assert np.abs(mz.to_numpy() - d["cplx"]).max() < 1e-15
    # DistVector.set_random draws column 0 of the same stream
    v = A.create_vector()
    v.set_random(77, True)
    assert np.array_equal(v.to_numpy(), d["real"][:, 0])


def test_compute_kpm_dos_matches_oracle(oracle):
    """utils.compute_kpm_dos (ex08's procedure) against the oracle's moments
    of the same scaled matrix and vectors, and against the DOS rebuilt from
    those moments."""
    from vbcsr_b200 import kpm, utils

    H, _ = W.tmd_lattice(10, seed=34)
    A = _vbcsr(H)
    g = W.gershgorin_bound(H) / 0.95
    V = np.where(np.random.default_rng(6).random((H.N, 8)) < 0.5, -1.0, 1.0)
    x, rho, mu = utils.compute_kpm_dos(A, num_moments=96, E_bound=g, num_points=300, vectors=V)
    Hs = W.BlockCSR(H.block_sizes, H.row_ptr, H.col_ind, H.values / g)
    mu_ref = oracle.kpm_moments(Hs, V, 96, True) / (8 * H.N)
    assert np.abs(mu - mu_ref).max() / abs(mu_ref[0]) < TOL
    xr, rr = kpm.dos_from_moments(mu_ref, 300)
    assert rel_err(x, xr * g) < TOL and rel_err(rho, rr / g) < 1e-10
    # the plain ex08 recurrence gives the same moments
    _, _, mu_plain = utils.compute_kpm_dos(A, num_moments=96, E_bound=g, num_points=300, vectors=V,
                                           two_moment=False)
    assert np.abs(mu_plain - mu_ref).max() / abs(mu_ref[0]) < 1e-11


def test_kpm_apply_and_propagation_match_oracle(oracle):
    """utils.kpm_apply (vbcsr/utils.py:71-126) with complex coefficients on a
    complex Hermitian lattice, and propagation.propagate_chebyshev, against
    the oracle's Chebyshev sum; and the propagated state against a dense
    matrix exponential."""
    from scipy.linalg import expm

    from vbcsr_b200 import propagation, utils

    d = np.load(GOLDEN / "cheb_apply_cplx.npz")
    H = W.BlockCSR(d["A_bsz"], d["A_rp"], d["A_ci"], d["A_val"])
    A = _vbcsr(H)
    v = A.create_vector()
    v.from_numpy(d["psi"])
    y = utils.kpm_apply(A, v, d["coeffs"], 1.0, 0.0)
    assert rel_err(y.to_numpy(), d["out"]) < TOL  # the reference core's own result
    Hl, _ = W.tmd_lattice(4, seed=35, bond_phase=True, dtype=np.complex128)
    Al = _vbcsr(Hl)
    Emax = W.gershgorin_bound(Hl) * 1.01
    psi = np.random.default_rng(8).normal(size=Hl.N) + 0j
    psi /= np.linalg.norm(psi)
    dt = 2.0
    out = propagation.propagate_chebyshev(Al, psi, dt, num_moments=64, E_max=Emax)
    coeffs = propagation.chebyshev_coefficients(Emax, dt, 64)
    Hs = W.BlockCSR(Hl.block_sizes, Hl.row_ptr, Hl.col_ind, Hl.values / Emax)
    assert rel_err(out, oracle.cheb_apply(Hs, coeffs, psi)) < TOL
    exact = expm(-1j * dt * Hl.to_dense()) @ psi
    assert np.abs(out - exact).max() < 1e-10

"""Pins the CPU oracle (the plain-C restatement) to golden vectors produced by
the REFERENCE implementation itself (tests/golden/make_golden.py), and checks
this package's host-side constructors against the reference's random stream.
CPU only."""
from pathlib import Path

import numpy as np
import pytest

from vbcsr_b200 import workloads as W

GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    return np.load(GOLD / f"{name}.npz")


def bcsr(d, p="A"):
    return W.BlockCSR(d[f"{p}_bsz"], d[f"{p}_rp"], d[f"{p}_ci"], d[f"{p}_val"])


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", ["apply_vbcsr", "apply_cplx", "apply_csr"])
def test_apply_golden(oracle, name):
    d = load(name)
    H = bcsr(d)
    assert rel(oracle.apply(H, d["x"]), d["y"]) < 1e-13
    assert rel(oracle.apply(H, d["x"], True), d["ya"]) < 1e-13
    assert rel(oracle.apply(H, d["X"]), d["Y"]) < 1e-13
    assert rel(oracle.apply(H, d["X"], True), d["Ya"]) < 1e-13
    assert rel(oracle.block_norms(H), d["norms"]) < 1e-15


def test_spmm_threshold_golden(oracle):
    d = load("spmm_threshold")
    A = bcsr(d)
    for k in range(4):
        thr = float(d[f"thr{k}"])
        C, _ = oracle.spgemm(A, A, thr)
        assert np.array_equal(C.row_ptr, d[f"C{k}_rp"]) and np.array_equal(C.col_ind, d[f"C{k}_ci"]), thr
        assert rel(C.values, d[f"C{k}_val"]) < 1e-14
    T = oracle.transpose(A)
    assert np.array_equal(T.col_ind, d["T_ci"]) and np.array_equal(T.values, d["T_val"])
    F = oracle.filter_blocks(A, float(d["F_thr"]))
    assert np.array_equal(F.col_ind, d["F_ci"]) and np.array_equal(F.values, d["F_val"])


def test_ring_golden(oracle):
    d = load("ring")
    A = bcsr(d)
    C0, _ = oracle.spgemm(A, A, 0.0)
    C6, _ = oracle.spgemm(A, A, 0.6)
    assert np.array_equal(C0.col_ind, d["C0_ci"]) and np.allclose(C0.values, d["C0_val"])
    assert np.array_equal(C6.col_ind, d["C6_ci"]) and np.allclose(C6.values, d["C6_val"])
    # reference tests/test_spmm.py: A^2 1 = 2.25 everywhere; with thr 0.6 -> 2.0
    one = np.ones(A.N)
    assert np.allclose(oracle.apply(C0, one), 2.25) and np.allclose(oracle.apply(C6, one), 2.0)


def test_set_random_golden(oracle):
    d = load("set_random")
    assert np.array_equal(oracle.set_random(d["bsz"], 3, 77, True), d["real"])
    assert np.array_equal(oracle.set_random(d["bsz"], 2, 5, False), d["real_raw"])
    assert np.abs(oracle.set_random(d["bsz"], 3, 77, True, complex_=True) - d["cplx"]).max() < 1e-15


def test_kpm_golden(oracle):
    d = load("kpm_tmd5")
    H = bcsr(d)
    for two in (False, True):
        mu = oracle.kpm_moments(H, d["V"], 40, two)
        assert np.abs(mu - d["mu"]).max() / abs(d["mu"][0]) < 1e-12


def test_cheb_apply_golden(oracle):
    d = load("cheb_apply_cplx")
    out = oracle.cheb_apply(bcsr(d), d["coeffs"], d["psi"])
    assert rel(out, d["out"]) < 1e-12


def test_create_random_matches_reference_stream():
    from vbcsr_b200 import VBCSR

    d = load("create_random")
    for k in range(3):
        nb, lo, hi, dens, seed, cplx = d[f"m{k}_args"]
        M = VBCSR.create_random(int(nb), int(lo), int(hi), float(dens),
                                dtype=np.complex128 if cplx else np.float64, seed=int(seed))
        assert np.array_equal(M.row_ptr, d[f"m{k}_rp"])
        assert np.array_equal(M.col_ind, d[f"m{k}_ci"])
        assert np.array_equal(np.asarray(M.graph.block_sizes), d[f"m{k}_bsz"])
        assert np.array_equal(M.get_values(), d[f"m{k}_val"])


def test_restated_against_reference_core(oracle, reference):
    """Where the reference core is built: random cases beyond the fixtures."""
    rng = np.random.default_rng(5)
    for seed in range(3):
        H = W.random_pattern(40, 1, 8, 5, seed=200 + seed)
        R = reference.matrix(H)
        X = rng.normal(size=(H.N, 3))
        assert rel(oracle.apply(H, X), R.mult_dense(X)) < 1e-13
        P = W.random_symmetric_blocks(40, seed=210 + seed)
        P.values *= 0.2
        Rp = reference.matrix(P)
        for thr in (0.0, 0.01, 0.1):
            C, _ = oracle.spgemm(P, P, thr)
            Cr = Rp.spmm(Rp, thr).to_blockcsr()
            assert np.array_equal(C.col_ind, Cr.col_ind) and np.array_equal(C.row_ptr, Cr.row_ptr)


def test_spmm_hermitian_golden(oracle):
    """The reference core's spmm_hermitian (upper block triangle, mirror,
    Hermitized diagonal) on a real symmetric and a complex Hermitian operand:
    the restated pattern is identical, values to 1e-14, the result exactly
    Hermitian."""
    d = load("spmm_hermitian")
    for tag in ("R", "Z"):
        A = bcsr(d, tag)
        for k in range(3):
            C, _ = oracle.spgemm_hermitian(A, A, float(d[f"{tag}thr{k}"]))
            assert np.array_equal(C.row_ptr, d[f"{tag}C{k}_rp"]) and np.array_equal(C.col_ind, d[f"{tag}C{k}_ci"])
            assert rel(C.values, d[f"{tag}C{k}_val"]) < 1e-14
            D = C.to_dense()
            assert np.array_equal(D, D.conj().T)


def test_spmm_hermitian_edge_rows_against_reference_core(oracle, reference):
    """Where the reference core is built: spmm_hermitian on a symmetric
    pattern with empty block rows and rows without a diagonal block, at
    thresholds that keep all, some and none of the blocks."""
    from .test_spgemm_gpu import _sym_drop

    A = _sym_drop(W.banded_decaying(120, neighbours=5, band=8, seed=4),
                  lambda i, j: i % 13 != 5 and not (i % 4 == 0 and i == j))
    R = reference.matrix(A)
    for thr in (0.0, 1e-3, 1e6):
        C, _ = oracle.spgemm_hermitian(A, A, thr)
        Cr = R.spmm_hermitian(R, thr).to_blockcsr()
        assert np.array_equal(C.row_ptr, Cr.row_ptr) and np.array_equal(C.col_ind, Cr.col_ind), thr
        if Cr.nnzb:
            assert rel(C.values, Cr.values) < 1e-13

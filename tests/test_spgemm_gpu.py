"""Thresholded SpGEMM, filter, union axpby and transpose on the GPU against the
CPU oracle (and the reference core where built).

Bar: the symbolic pattern is bit-exact; the final (filtered) pattern is
identical except for blocks whose Frobenius norm lies within 1e-10 relative
of the threshold; FP64 values match to 1e-12 relative."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W

pytestmark = pytest.mark.gpu
BAND = 1e-10
TOL = 1e-12


def block_dict(H):
    off = H.slot_offsets()
    d = {}
    for i in range(H.n):
        for s in range(H.row_ptr[i], H.row_ptr[i + 1]):
            d[(i, int(H.col_ind[s]))] = H.values[off[s]:off[s + 1]]
    return d


def assert_same_result(G, O, thr):
    """G: GPU result, O: oracle result (BlockCSR)."""
    gd, od = block_dict(G), block_dict(O)
    scale = max((np.abs(v).max() for v in od.values() if len(v)), default=1.0)
    for key in set(gd) ^ set(od):
        v = gd.get(key, od.get(key))
        nrm = np.sqrt(np.sum(np.abs(v) ** 2))
        assert thr > 0 and abs(nrm - thr) <= BAND * thr, f"block {key} differs (norm {nrm}, thr {thr})"
    for key in set(gd) & set(od):
        assert np.abs(gd[key] - od[key]).max() <= TOL * scale, key


def _operands():
    P = W.random_symmetric_blocks(150, seed=9)
    P.values *= 0.1
    B = W.banded_decaying(300, neighbours=6, band=12, seed=4)
    Z = W.random_pattern(60, 2, 6, 4, seed=3, dtype=np.complex128)
    Q = W.random_pattern(50, 1, 11, 5, seed=8)  # block sizes up to 11
    return {"sym": P, "banded": B, "cplx": Z, "wide": Q}


@pytest.fixture(scope="module")
def ops():
    return _operands()


@pytest.mark.parametrize("name", ["sym", "banded", "cplx", "wide"])
@pytest.mark.parametrize("thr", [0.0, 1e-5, 1e-2, 0.05, 0.3])
def test_spgemm_vs_oracle(ops, oracle, dev, name, thr):
    from . import _gpu

    A = ops[name]
    dA = _gpu.dmat(A)
    C, stats = dA.spgemm(dA, thr)
    O, ostats = oracle.spgemm(A, A, thr)
    assert stats[0] == ostats[0], "symbolic block count"
    assert_same_result(C.to_blockcsr(), O, thr)


def test_symbolic_pattern_bit_exact(ops, oracle, dev):
    """thr > 0 with the filter undone: compare the symbolic stage alone by
    choosing a threshold no block norm reaches from below the band."""
    from . import _gpu

    A = ops["banded"]
    dA = _gpu.dmat(A)
    for thr in (1e-6, 1e-3, 1e-1):
        C, stats = dA.spgemm(dA, thr)
        _, ostats = oracle.spgemm(A, A, thr)
        assert stats[0] == ostats[0]


def test_spgemm_vs_reference_core(ops, reference, dev):
    from . import _gpu

    A = ops["sym"]
    R = reference.matrix(A)
    dA = _gpu.dmat(A)
    for thr in (0.0, 0.02, 0.2):
        C, _ = dA.spgemm(dA, thr)
        assert_same_result(C.to_blockcsr(), R.spmm(R, thr).to_blockcsr(), thr)


def test_ring_known_answers(oracle, dev):
    """tests/test_spmm.py:93-200 of the reference: the directed ring 4x(2x2)
    with I on the diagonal and 0.5 I on (i, i+1): A^2 1 = 2.25, with
    threshold 0.6 the distance-2 blocks (norm 0.354) vanish and A^2 1 = 2.0;
    A I = A."""
    from . import _gpu

    A = W.ring_blocks(4, 2)
    dA = _gpu.dmat(A)
    one = np.ones(A.N)
    C, _ = dA.spgemm(dA, 0.0)
    assert np.allclose(_gpu.apply(C, one), 2.25)
    C6, _ = dA.spgemm(dA, 0.6)
    assert C6.nnzb == 8
    assert np.allclose(_gpu.apply(C6, one), 2.0)
    I = W.BlockCSR(A.block_sizes, np.arange(5, dtype=np.int32), np.arange(4, dtype=np.int32),
                   np.tile(np.eye(2).ravel(), 4))
    CI, _ = dA.spgemm(_gpu.dmat(I), 0.0)
    assert np.allclose(_gpu.apply(CI, one), _gpu.apply(dA, one))


def test_asymmetric_row_eps(oracle, dev):
    """Row-dependent numeric skip threshold / nnzblk(A row)
    (vbcsr/core/test/test_asymmetric_filter.cpp pattern): rows with different
    block counts drop different pairs; result must equal the oracle."""
    from . import _gpu

    rng = np.random.default_rng(7)
    n = 6
    bsz = np.full(n, 2)
    rows = [0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 3, 4, 5]
    cols = [0, 1, 2, 3, 1, 0, 2, 3, 3, 0, 5, 4, 5]
    key = sorted(zip(rows, cols))
    r = np.array([k[0] for k in key])
    c = np.array([k[1] for k in key])
    vals = rng.uniform(0.2, 1.0, size=(len(key), 2, 2))
    A = W._assemble(n, bsz.astype(np.int64), r, c, [(np.arange(len(key)), vals)])
    dA = _gpu.dmat(A)
    for thr in (0.3, 0.9, 1.5):
        C, st = dA.spgemm(dA, thr)
        O, ost = oracle.spgemm(A, A, thr)
        assert st[0] == ost[0] and st[2] == ost[2]
        assert_same_result(C.to_blockcsr(), O, thr)


def test_filter_blocks(ops, oracle, dev):
    from . import _gpu

    A = ops["banded"]
    for thr in (0.0, 0.05, 0.5, 1.0, 100.0):
        d = _gpu.dmat(A)
        d.filter_blocks(thr)
        assert_same_result(d.to_blockcsr(), oracle.filter_blocks(A, thr), thr)


def test_filter_keeps_diagonal_ring(dev):
    """vbcsr/core/test/test_spmm.cpp filtered-structure test: on the ring,
    filter_blocks(1.0) keeps only the diagonal blocks (norm sqrt(2) vs 0.71)."""
    from . import _gpu

    d = _gpu.dmat(W.ring_blocks(4, 2))
    d.filter_blocks(1.0)
    rp, ci, _ = d.structure()
    assert list(ci) == [0, 1, 2, 3] and list(rp) == [0, 1, 2, 3, 4]


@pytest.mark.parametrize("alpha,beta", [(3.0, -2.0), (0.0, 2.0), (1.5, 0.0), (-1.0, 1.0)])
def test_axpby_union(ops, oracle, dev, alpha, beta):
    from . import _gpu

    A = ops["sym"]
    C, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
    Cb = C.to_blockcsr()
    dY = _gpu.dmat(Cb)
    dX = _gpu.dmat(A)
    dY.axpby(alpha, dX, beta)  # Y = alpha A + beta C
    G = dY.to_blockcsr()
    if alpha == 0.0:
        ref = Cb
        ref = W.BlockCSR(Cb.block_sizes, Cb.row_ptr, Cb.col_ind, beta * Cb.values)
    elif beta == 0.0:
        ref = W.BlockCSR(A.block_sizes, A.row_ptr, A.col_ind, alpha * A.values)
    else:
        ref = oracle.axpby(Cb, alpha, A, beta)
    assert np.array_equal(G.row_ptr, ref.row_ptr) and np.array_equal(G.col_ind, ref.col_ind)
    assert np.abs(G.values - ref.values).max() <= TOL * np.abs(ref.values).max()


@pytest.mark.parametrize("alpha,beta", [(1.0 + 0.5j, -0.25 + 2.0j), (0.0, 1.0 - 1.0j), (2.0j, 0.0)])
def test_axpby_union_complex(ops, oracle, dev, alpha, beta):
    """Complex coefficients on complex blocks: union pattern (Z Z thresholded
    against Z), X's pattern (beta = 0), Y's pattern (alpha = 0)."""
    from . import _gpu

    Z = ops["cplx"]
    C, _ = _gpu.dmat(Z).spgemm(_gpu.dmat(Z), 0.5)
    Cb = C.to_blockcsr()
    dY = _gpu.dmat(Cb)
    dY.axpby(alpha, _gpu.dmat(Z), beta)
    G = dY.to_blockcsr()
    if alpha == 0.0:
        ref = W.BlockCSR(Cb.block_sizes, Cb.row_ptr, Cb.col_ind, beta * Cb.values)
    elif beta == 0.0:
        ref = W.BlockCSR(Z.block_sizes, Z.row_ptr, Z.col_ind, alpha * Z.values)
    else:
        ref = oracle.axpby(Cb, alpha, Z, beta)
    assert np.array_equal(G.row_ptr, ref.row_ptr) and np.array_equal(G.col_ind, ref.col_ind)
    assert np.abs(G.values - ref.values).max() <= TOL * np.abs(ref.values).max()


@pytest.mark.parametrize("name,alpha,beta", [("sym", 3.0, -2.0), ("cplx", 1.0 - 2.0j, 0.5j), ("wide", -1.0, 0.0)])
def test_axpby_same_pattern(ops, oracle, dev, name, alpha, beta):
    """Y and X on one pattern: updated in place, pattern unchanged."""
    from . import _gpu

    A = ops[name]
    rng = np.random.default_rng(2)
    Xv = W.BlockCSR(A.block_sizes, A.row_ptr, A.col_ind, A.values * rng.uniform(0.5, 1.5, A.values.shape))
    dY = _gpu.dmat(A)
    dY.axpby(alpha, _gpu.dmat(Xv), beta)
    G = dY.to_blockcsr()
    ref = oracle.axpby(A, alpha, Xv, beta)
    assert np.array_equal(G.row_ptr, ref.row_ptr) and np.array_equal(G.col_ind, ref.col_ind)
    assert np.abs(G.values - ref.values).max() <= TOL * np.abs(ref.values).max()


@pytest.mark.parametrize("name", ["sym", "cplx", "wide"])
def test_device_built_structure_roundtrip(ops, oracle, dev, name):
    """A SpGEMM result (its pattern built on the device, host copy read back
    on first use) through every host-side consumer: apply and adjoint apply
    (k = 1, 8), duplicate, transpose, filter, axpby against itself-shaped
    and differently-shaped operands."""
    from . import _gpu

    A = ops[name]
    C, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
    O = oracle.spgemm(A, A, 0.05)[0]
    G = C.to_blockcsr()
    assert_same_result(G, O, 0.05)
    rng = np.random.default_rng(4)
    dense = G.to_dense()
    for k in (1, 8):
        X = rng.standard_normal((G.N, k) if k > 1 else G.N).astype(A.values.dtype)
        for adj in (False, True):
            C2, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
            Y = _gpu.apply(C2, X, adjoint=adj)
            ref = (dense.conj().T if adj else dense) @ X
            assert np.abs(Y - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    C3, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
    D = C3.duplicate().to_blockcsr()
    assert np.array_equal(D.row_ptr, G.row_ptr) and np.array_equal(D.values, G.values)
    C4, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
    T = C4.transpose().to_blockcsr()
    OT = oracle.transpose(G)
    assert np.array_equal(T.row_ptr, OT.row_ptr) and np.array_equal(T.col_ind, OT.col_ind)
    assert np.array_equal(T.values, OT.values)
    # axpby of two device-built operands: same pattern (in place) and union
    C5, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
    C6, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
    C5.axpby(2.0, C6, -1.0)
    S = C5.to_blockcsr()
    assert np.array_equal(S.col_ind, G.col_ind)
    assert np.abs(S.values - G.values).max() <= TOL * np.abs(G.values).max()
    C7, _ = _gpu.dmat(A).spgemm(_gpu.dmat(A), 0.05)
    C7.filter_blocks(0.2)
    C7.axpby(1.0, C6, 1.0)
    U = C7.to_blockcsr()
    ref = oracle.axpby(oracle.filter_blocks(G, 0.2), 1.0, G, 1.0)
    assert np.array_equal(U.row_ptr, ref.row_ptr) and np.array_equal(U.col_ind, ref.col_ind)
    assert np.abs(U.values - ref.values).max() <= TOL * np.abs(ref.values).max()


def test_memory_trim_and_reserve_keep_results(ops, dev):
    """Products before and after returning the cached memory to the driver
    (and after mapping pool memory ahead) are identical: buffers are reused
    only once nothing can still use them."""
    from vbcsr_b200 import _capi

    from . import _gpu

    A = ops["banded"]
    first = [_gpu.dmat(A).spgemm(_gpu.dmat(A), thr)[0].to_blockcsr() for thr in (0.0, 1e-3)]
    _capi.memory_trim()
    _capi.memory_reserve(64 << 20)
    again = [_gpu.dmat(A).spgemm(_gpu.dmat(A), thr)[0].to_blockcsr() for thr in (0.0, 1e-3)]
    for F, G in zip(first, again):
        assert np.array_equal(F.row_ptr, G.row_ptr) and np.array_equal(F.col_ind, G.col_ind)
        assert np.array_equal(F.values, G.values)
    _capi.memory_trim()


@pytest.mark.parametrize("name", ["sym", "cplx", "wide"])
def test_transpose(ops, oracle, dev, name):
    from . import _gpu

    A = ops[name]
    T = _gpu.dmat(A).transpose().to_blockcsr()
    O = oracle.transpose(A)
    assert np.array_equal(T.row_ptr, O.row_ptr) and np.array_equal(T.col_ind, O.col_ind)
    assert np.array_equal(T.values, O.values)


def test_mcweeny_iterations_match_oracle(oracle, dev):
    """Three McWeeny steps P <- 3 P^2 - 2 P^3 with threshold on a banded,
    decaying matrix scaled into McWeeny's basin: nnzb per iteration and
    values follow the oracle."""
    from . import _gpu

    H = W.banded_decaying(200, neighbours=6, band=10, seed=12)
    g = W.gershgorin_bound(H)
    P = W.BlockCSR(H.block_sizes, H.row_ptr, H.col_ind, -0.45 / g * H.values)
    so = P.scalar_offsets()
    W.add_diagonal(P, np.full(P.N, 0.5))
    thr = 1e-5
    dP = _gpu.dmat(P)
    Po = P
    for _ in range(3):
        dP2, _ = dP.spgemm(dP, thr)
        dP3, _ = dP2.spgemm(dP, thr)
        dP2.axpby(-2.0, dP3, 3.0)
        dP = dP2
        P2, _ = oracle.spgemm(Po, Po, thr)
        P3, _ = oracle.spgemm(P2, Po, thr)
        Po = oracle.axpby(P2, -2.0, P3, 3.0)
        G = dP.to_blockcsr()
        assert np.array_equal(G.col_ind, Po.col_ind)
        assert np.abs(G.values - Po.values).max() < 1e-11


@pytest.mark.parametrize("name", ["sym", "banded", "herm"])
@pytest.mark.parametrize("thr", [0.0, 1e-3, 0.05])
def test_spgemm_hermitian_vs_oracle(ops, oracle, dev, name, thr):
    """Upper block triangle multiplied, lower triangle mirrored, diagonal
    blocks Hermitized: the pattern equals the oracle's (threshold band
    aside), values 1e-12, the result exactly Hermitian, and about half the
    block products of the full product."""
    from . import _gpu

    A = ops[name] if name != "herm" else W.tmd_lattice(5, seed=3, bond_phase=True, dtype=np.complex128)[0]
    dA = _gpu.dmat(A)
    C, stats = dA.spgemm_hermitian(dA, thr)
    O, ostats = oracle.spgemm_hermitian(A, A, thr)
    assert stats[0] == ostats[0] and stats[2] == ostats[2]
    G = C.to_blockcsr()
    assert_same_result(G, O, thr)
    D = G.to_dense()
    assert np.array_equal(D, D.conj().T)
    _, full = dA.spgemm(dA, thr)
    assert stats[2] <= full[2]
    if thr == 0.0:  # at larger thresholds the surviving products can all be on the diagonal
        assert stats[2] <= 0.6 * full[2] + 8


def test_spgemm_hermitian_vs_reference_core(ops, reference, dev):
    from . import _gpu

    for name in ("sym", "banded"):
        A = ops[name]
        R = reference.matrix(A)
        dA = _gpu.dmat(A)
        for thr in (0.0, 0.02):
            C, _ = dA.spgemm_hermitian(dA, thr)
            assert_same_result(C.to_blockcsr(), R.spmm_hermitian(R, thr).to_blockcsr(), thr)


def test_spmm_hermitian_api(dev):
    """VBCSR.spmm_hermitian (the reference's Python method) on a symmetric
    matrix: equal to spmm to rounding, and exactly symmetric."""
    import scipy.sparse as sp

    from vbcsr_b200 import VBCSR

    rng = np.random.default_rng(3)
    n, b = 40, 3
    mask = rng.random((n, n)) < 0.15
    mask = mask | mask.T | np.eye(n, dtype=bool)
    D = np.kron(mask, np.ones((b, b))) * rng.normal(size=(n * b, n * b))
    D = D + D.T
    M = VBCSR.from_scipy(sp.bsr_matrix(D, blocksize=(b, b)))
    H = M.spmm_hermitian(M, 0.0).to_dense()
    F = M.spmm(M, 0.0).to_dense()
    assert np.array_equal(H, H.T)
    assert np.abs(H - F).max() <= 1e-12 * np.abs(F).max()
    assert np.abs(H - D @ D).max() <= 1e-12 * np.abs(D @ D).max()


def _serial_full(VBCSR, nb, bs, rng, hermitian):
    """Dense block pattern (every block present), complex values; Hermitian
    when asked (diagonal blocks Hermitian, (j, i) = (i, j)^H), else each block
    drawn on its own (the reference's tests/test_spmm_hermitian.py inputs)."""
    M = VBCSR.create_serial(nb, [bs] * nb, [list(range(nb)) for _ in range(nb)], dtype=np.complex128)

    def draw():
        return rng.standard_normal((bs, bs)) + 1j * rng.standard_normal((bs, bs))

    for i in range(nb):
        for j in range(i, nb):
            blk = draw()
            if hermitian and i == j:
                blk = 0.5 * (blk + blk.conj().T)
            M.add_block(i, j, blk)
            if i != j:
                M.add_block(j, i, blk.conj().T if hermitian else draw())
    M.assemble()
    return M


def test_spmm_hermitian_congruence_transA(dev):
    """Z^H (S Z) with S Hermitian and Z general, through transA (the
    reference's congruence case), and X X for Hermitian X: equal to the full
    product to 1e-12 and exactly Hermitian."""
    from vbcsr_b200 import VBCSR

    rng = np.random.default_rng(7)
    S = _serial_full(VBCSR, 6, 3, rng, True)
    Z = _serial_full(VBCSR, 6, 3, rng, False)
    SZ = S.spmm(Z, 0.0)
    full = Z.spmm(SZ, 0.0, True).to_dense()
    half = Z.spmm_hermitian(SZ, 0.0, True).to_dense()
    assert np.abs(full - half).max() < 1e-12 * np.abs(full).max()
    assert np.array_equal(half, half.conj().T)
    X = _serial_full(VBCSR, 5, 4, np.random.default_rng(11), True)
    full = X.spmm(X, 0.0).to_dense()
    half = X.spmm_hermitian(X, 0.0).to_dense()
    assert np.abs(full - half).max() < 1e-12 * np.abs(full).max()
    assert np.array_equal(half, half.conj().T)


def test_mcweeny_hermitian_iterations_match_oracle(oracle, dev):
    """Three McWeeny steps with both products Hermitian: nnzb and values
    follow the oracle's Hermitian product, and stay near the full-product
    iterates; the purification API's hermitian switch gives the same P."""
    import scipy.sparse as sp

    from vbcsr_b200 import VBCSR
    from vbcsr_b200.purification import mcweeny_purify

    from . import _gpu

    H = W.banded_decaying(200, neighbours=6, band=10, seed=12)
    g = W.gershgorin_bound(H)
    P = W.BlockCSR(H.block_sizes, H.row_ptr, H.col_ind, -0.45 / g * H.values)
    W.add_diagonal(P, np.full(P.N, 0.5))
    thr = 1e-5
    dP, Po, Pf = _gpu.dmat(P), P, P
    for _ in range(3):
        dP2, _ = dP.spgemm_hermitian(dP, thr)
        dP3, _ = dP2.spgemm_hermitian(dP, thr)
        dP2.axpby(-2.0, dP3, 3.0)
        dP = dP2
        P2, _ = oracle.spgemm_hermitian(Po, Po, thr)
        P3, _ = oracle.spgemm_hermitian(P2, Po, thr)
        Po = oracle.axpby(P2, -2.0, P3, 3.0)
        F2, _ = oracle.spgemm(Pf, Pf, thr)
        F3, _ = oracle.spgemm(F2, Pf, thr)
        Pf = oracle.axpby(F2, -2.0, F3, 3.0)
        G = dP.to_blockcsr()
        assert np.array_equal(G.col_ind, Po.col_ind)
        assert np.abs(G.values - Po.values).max() < 1e-11
        D = G.to_dense()
        assert np.array_equal(D, D.T)
        assert np.abs(D - Pf.to_dense()).max() < 10 * thr  # dropped blocks differ, each below thr
    A = VBCSR.from_scipy(sp.bsr_matrix(H.to_dense()))
    r_full = mcweeny_purify(A, threshold=0.0, iterations=3, alpha=-0.45 / g, beta=0.5)
    r_herm = mcweeny_purify(A, threshold=0.0, iterations=3, alpha=-0.45 / g, beta=0.5, hermitian=True)
    Dh, Df = r_herm.P.to_dense(), r_full.P.to_dense()
    assert np.array_equal(Dh, Dh.T)
    assert np.abs(Dh - Df).max() < 1e-12 * np.abs(Df).max()


def test_spgemm_hermitian_golden(dev):
    """The reference core's spmm_hermitian outputs (committed fixture): the
    GPU pattern equals it (threshold band aside) and values match to 1e-12."""
    from pathlib import Path

    from . import _gpu

    d = np.load(Path(__file__).parent / "golden" / "spmm_hermitian.npz")
    for tag in ("R", "Z"):
        A = W.BlockCSR(d[f"{tag}_bsz"], d[f"{tag}_rp"], d[f"{tag}_ci"], d[f"{tag}_val"])
        dA = _gpu.dmat(A)
        for k in range(3):
            thr = float(d[f"{tag}thr{k}"])
            C, _ = dA.spgemm_hermitian(dA, thr)
            ref = W.BlockCSR(A.block_sizes, d[f"{tag}C{k}_rp"], d[f"{tag}C{k}_ci"], d[f"{tag}C{k}_val"])
            assert_same_result(C.to_blockcsr(), ref, thr)


def _sym_drop(H, keep):
    """H restricted to the blocks (i, j) with keep(i, j) and keep(j, i): the
    pattern stays symmetric (H real symmetric or Hermitian stays so)."""
    off = H.slot_offsets()
    rp, ci, vals = [0], [], []
    for i in range(H.n):
        for s in range(H.row_ptr[i], H.row_ptr[i + 1]):
            j = int(H.col_ind[s])
            if keep(i, j) and keep(j, i):
                ci.append(j)
                vals.append(H.values[off[s]:off[s + 1]])
        rp.append(len(ci))
    return W.BlockCSR(H.block_sizes, np.array(rp, np.int32), np.array(ci, np.int32),
                      np.concatenate(vals) if vals else np.zeros(0, H.values.dtype))


@pytest.mark.parametrize("thr", [0.0, 1e-3, 1e6])
def test_spgemm_hermitian_edge_rows(ops, oracle, dev, thr):
    """Empty block rows, rows without a diagonal block (so C rows whose
    diagonal block exists only through the product or not at all) and a
    threshold that empties the result: pattern and values as the oracle's,
    exactly Hermitian."""
    from . import _gpu

    A = _sym_drop(ops["banded"], lambda i, j: i % 13 != 5 and not (i % 4 == 0 and i == j))
    dA = _gpu.dmat(A)
    C, st = dA.spgemm_hermitian(dA, thr)
    O, ost = oracle.spgemm_hermitian(A, A, thr)
    assert st[0] == ost[0] and st[1] == ost[1]
    G = C.to_blockcsr()
    assert_same_result(G, O, thr)
    if G.nnzb:
        D = G.to_dense()
        assert np.array_equal(D, D.conj().T)

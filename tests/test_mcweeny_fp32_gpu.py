"""Mixed-precision McWeeny purification on the GPU: FP32 products
(vbg_spgemm_ex, FP32 operands and accumulation) with FP64 trace, residual,
electron-count correction and final polishing iterations, checked against the
C oracle (FP64) and against the plain FP64 loop.

Tolerances, stated: an FP32 product matches the oracle's FP64 product to
2e-6 of its largest value, and its pattern is the oracle's except for blocks
whose norm lies within 1e-5 relative of the threshold (FP32 rounding moves
block norms by about 1e-7 relative); the FP64 device reductions (trace,
Frobenius norm) match numpy to 1e-13; purified with two FP64 polishing
iterations on a gapped Hamiltonian (where McWeeny converges and the FP64
steps contract the eigenvalue error FP32 left; the occupied subspace keeps
a rotation of about 2e-8, measured with numpy's FP32 products on the same
matrix), P matches the all-FP64 run to 2e-7 relative (Frobenius), is
idempotent to the FP64 run's level and its trace is the electron count."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _p0(n=300, seed=12):
    H = W.banded_decaying(n, neighbours=6, band=10, seed=seed)
    g = W.gershgorin_bound(H)
    P = W.BlockCSR(H.block_sizes, H.row_ptr, H.col_ind, -0.45 / g * H.values)
    W.add_diagonal(P, np.full(P.N, 0.5))
    return H, g, P


def _gapped(n, seed):
    """A banded, decaying Hamiltonian (scaled to norm 0.3) plus a staggered
    on-site term +-1 per block row: a gap of about 1.4 around zero, so the
    density matrix has tr = the scalar rows on the -1 sites."""
    H = W.banded_decaying(n, neighbours=6, band=10, seed=seed)
    H.values *= 0.3 / W.gershgorin_bound(H)
    so = H.scalar_offsets()
    d = np.concatenate([np.full(H.block_sizes[i], -1.0 if i % 2 else 1.0) for i in range(H.n)])
    W.add_diagonal(H, d)
    occupied = int(sum(H.block_sizes[i] for i in range(H.n) if i % 2))
    assert so[-1] == H.N
    return H, W.gershgorin_bound(H), occupied


def _blocks(H):
    off = H.slot_offsets()
    rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
    return {(int(i), int(j)): H.values[off[s]:off[s + 1]] for s, (i, j) in enumerate(zip(rows, H.col_ind))}


@pytest.mark.parametrize("thr", [0.0, 1e-4])
@pytest.mark.parametrize("hermitian", [False, True])
def test_fp32_product_vs_oracle(oracle, dev, thr, hermitian):
    from vbcsr_b200 import _capi

    from . import _gpu

    _, _, P = _p0()
    dP = _gpu.dmat(P)
    C, stats = dP.spgemm_ex(dP, thr, precision=_capi.VBG_PREC_F32, hermitian=hermitian)
    O, _ = (oracle.spgemm_hermitian if hermitian else oracle.spgemm)(P, P, thr)
    gd, od = _blocks(C.to_blockcsr()), _blocks(O)
    for key in set(gd) ^ set(od):
        v = gd.get(key, od.get(key))
        nrm = np.sqrt(np.sum(np.abs(v) ** 2))
        assert thr > 0 and abs(nrm - thr) <= 1e-5 * thr, key
    scale = max(np.abs(v).max() for v in od.values())
    err = max(np.abs(gd[k] - od[k]).max() for k in set(gd) & set(od))
    assert err <= 2e-6 * scale
    assert err > 0.0  # the arithmetic really was FP32
    # the FP64 product through the same entry point is the oracle's to 1e-12
    C64, _ = dP.spgemm_ex(dP, thr, precision=_capi.VBG_PREC_F64, hermitian=hermitian)
    g64 = _blocks(C64.to_blockcsr())
    assert max(np.abs(g64[k] - od[k]).max() for k in set(g64) & set(od)) <= 1e-12 * scale


def test_device_trace_and_norm(dev):
    import torch

    from . import _gpu

    for dtype in (np.float64, np.complex128):
        H = W.random_pattern(120, 1, 6, 4, seed=5, dtype=dtype)
        dm = _gpu.dmat(H)
        out = torch.zeros(2, dtype=torch.float64, device="cuda")
        dm.trace_dev(out.data_ptr())
        torch.cuda.synchronize()
        tr = np.trace(H.to_dense())
        got = out.cpu().numpy()
        assert abs(got[0] - tr.real) <= 1e-13 * np.abs(H.values).sum()
        assert abs(got[1] - tr.imag) <= 1e-13 * np.abs(H.values).sum()
        dm.norm_fro_dev(out.data_ptr())
        torch.cuda.synchronize()
        assert abs(out.cpu().numpy()[0] - np.linalg.norm(H.values)) <= 1e-13 * np.linalg.norm(H.values)


def test_mcweeny_fp32_with_fp64_polish(dev):
    """12 iterations without filtering on a gapped Hamiltonian: 10 FP32 + 2
    FP64 against 12 FP64.  The polished P matches, is idempotent to the FP64
    run's level, and its trace (FP64 device reduction) is the electron
    count."""
    from vbcsr_b200 import VBCSR
    from vbcsr_b200.purification import mcweeny_purify

    H, g, occ = _gapped(240, seed=13)
    A = VBCSR.from_block_csr(H.block_sizes, H.row_ptr, H.col_ind, H.values)
    r64 = mcweeny_purify(A, threshold=0.0, iterations=12, alpha=-0.45 / g, beta=0.5)
    r32 = mcweeny_purify(A, threshold=0.0, iterations=12, alpha=-0.45 / g, beta=0.5, precision="fp32", polish=2)
    assert r32.precision == ["fp32"] * 10 + ["fp64"] * 2
    P64, P32 = r64.P.to_dense(), r32.P.to_dense()
    assert np.linalg.norm(P32 - P64) <= 2e-7 * np.linalg.norm(P64)
    # FP32 products really ran: the iterates differ before the polish
    assert r32.residual[5] != r64.residual[5]
    res32 = np.linalg.norm(P32 @ P32 - P32)
    res64 = np.linalg.norm(P64 @ P64 - P64)
    assert res32 <= max(10 * res64, 1e-10 * np.linalg.norm(P64))
    assert abs(r32.trace[-1] - np.trace(P32)) <= 1e-12 * abs(np.trace(P32))
    assert abs(r32.trace[-1] - occ) <= 1e-8 * occ


def test_mcweeny_fp32_electron_count(dev):
    """With the electron-count correction the FP32 iterations keep tr(P) at
    the requested count (FP64 reduction and shift on the device)."""
    from vbcsr_b200 import VBCSR
    from vbcsr_b200.purification import mcweeny_purify

    H, g, ne = _gapped(200, seed=14)
    A = VBCSR.from_block_csr(H.block_sizes, H.row_ptr, H.col_ind, H.values)
    r = mcweeny_purify(A, threshold=0.0, iterations=8, alpha=-0.45 / g, beta=0.5, precision="fp32", polish=0,
                       electrons=ne)
    assert all(abs(t - ne) <= 1e-9 * ne for t in r.trace)
    assert abs(np.trace(r.P.to_dense()) - ne) <= 1e-9 * ne

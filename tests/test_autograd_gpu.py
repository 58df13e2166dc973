"""Gradients: the SDDMM kernel against a dense outer product, and the
autograd Functions (sparse apply, Chebyshev propagation, KPM moments)
against central finite differences (h = 1e-6) on random stored entries and,
for the propagation, against a dense torch matrix_exp reference.
Tolerances: SDDMM 1e-12 relative; gradients 1e-6 relative (finite
differences), 1e-9 relative (dense reference)."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dense_index(H):
    """(row, col) of every stored scalar in slot order (row-major blocks)."""
    so = np.concatenate([[0], np.cumsum(H.block_sizes)])
    rows, cols = [], []
    for i in range(len(H.block_sizes)):
        r = H.block_sizes[i]
        for s in range(H.row_ptr[i], H.row_ptr[i + 1]):
            j = H.col_ind[s]
            c = H.block_sizes[j]
            rr, cc = np.meshgrid(np.arange(r) + so[i], np.arange(c) + so[j], indexing="ij")
            rows.append(rr.ravel())
            cols.append(cc.ravel())
    return np.concatenate(rows), np.concatenate(cols)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("k", [1, 5, 16, 40])  # 40: past the shared-memory staging (32 columns)
@pytest.mark.parametrize("wide", [False, True])  # wide: blocks over 8 rows / columns, read from global memory
def test_sddmm_vs_dense(dev, cplx, k, wide):
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    dt = np.complex128 if cplx else np.float64
    H = W.random_pattern(40, 1, 12 if wide else 6, 5, seed=31, dtype=dt)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(k)
    G = rng.normal(size=(H.N, k))
    X = rng.normal(size=(H.N, k))
    if cplx:
        G = G + 1j * rng.normal(size=(H.N, k))
        X = X + 1j * rng.normal(size=(H.N, k))
    out0 = rng.normal(size=H.nnz) + (1j * rng.normal(size=H.nnz) if cplx else 0)
    tdt = torch.complex128 if cplx else torch.float64
    g = torch.from_numpy(np.ascontiguousarray(G.astype(dt))).cuda()
    x = torch.from_numpy(np.ascontiguousarray(X.astype(dt))).cuda()
    out = torch.from_numpy(np.ascontiguousarray(out0.astype(dt))).cuda()
    alpha = (0.7 - 0.2j) if cplx else 0.7
    from vbcsr_b200.autograd import _sddmm

    _sddmm(dm, g if k > 1 else g[:, 0], x if k > 1 else x[:, 0], out, alpha)
    torch.cuda.synchronize()
    r, c = _dense_index(H)
    full = G @ X.conj().T
    ref = out0 + alpha * full[r, c]
    got = out.cpu().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12
    assert got.dtype == np.dtype(dt) and tdt is not None


def _fd_check(loss_fn, values, grad, idx, h=1e-6, tol=1e-6):
    """Central differences on entries idx (real and, if complex, imaginary
    parts) against the autograd gradient (PyTorch convention: d/dRe + i d/dIm)."""
    import torch

    scale = max(float(grad.abs().max()), 1e-300)
    with torch.no_grad():
        for i in idx:
            parts = [1.0, 1j] if values.is_complex() else [1.0]
            for p in parts:
                v1 = values.clone()
                v2 = values.clone()
                v1[i] += h * p
                v2[i] -= h * p
                fd = (loss_fn(v1) - loss_fn(v2)) / (2 * h)
                an = grad[i].real if p == 1.0 else grad[i].imag
                assert abs(fd - float(an)) <= tol * scale, (i, p, fd, float(an))


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("k", [1, 8])
def test_sparse_apply_gradients(dev, cplx, k):
    import torch

    from vbcsr_b200.autograd import sparse_apply

    from . import _gpu

    dt = np.complex128 if cplx else np.float64
    tdt = torch.complex128 if cplx else torch.float64
    H = W.random_pattern(30, 2, 6, 4, seed=41, dtype=dt)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(5)
    vals = torch.from_numpy(H.values.astype(dt)).cuda().requires_grad_(True)
    Xn = rng.normal(size=(H.N, k)) + (1j * rng.normal(size=(H.N, k)) if cplx else 0)
    X = torch.from_numpy(np.ascontiguousarray(Xn.astype(dt) if k > 1 else Xn[:, 0].astype(dt))).cuda()
    X.requires_grad_(True)
    wts = torch.from_numpy(rng.uniform(size=X.shape)).cuda()

    def loss_of(v, x=None):
        Y = sparse_apply(v, X if x is None else x, dm)
        return (wts * (Y.conj() * Y).real).sum() if cplx else (wts * Y * Y).sum()

    L = loss_of(vals)
    L.backward()
    gV = vals.grad.detach().clone()
    gX = X.grad.detach().clone()
    idx = rng.choice(H.nnz, size=32, replace=False)
    _fd_check(lambda v: float(loss_of(v)), vals.detach(), gV, idx)
    xf = X.detach().reshape(-1)
    gxf = gX.reshape(-1)
    idx = rng.choice(xf.numel(), size=16, replace=False)
    _fd_check(lambda x: float(loss_of(vals.detach(), x.reshape(X.shape))), xf, gxf, idx)


def _wavepacket(H, L, rng, sigma=2.0):
    """Gaussian wavepacket over the lattice cells with a random momentum,
    normalised (complex)."""
    ncell = L * L
    ix, iy = np.meshgrid(np.arange(L), np.arange(L), indexing="xy")
    x, y = ix.ravel().astype(float), iy.ravel().astype(float)
    k = rng.uniform(-1, 1, size=2)
    env = np.exp(-((x - L / 2) ** 2 + (y - L / 2) ** 2) / (2 * sigma ** 2)) * np.exp(1j * (k[0] * x + k[1] * y))
    so = np.concatenate([[0], np.cumsum(H.block_sizes)])
    psi = np.zeros(H.N, np.complex128)
    for c in range(ncell):
        for site in range(3):
            b = 3 * c + site
            psi[so[b]:so[b + 1]] = env[c] * (rng.normal(size=so[b + 1] - so[b]) + 1j * rng.normal(size=so[b + 1] - so[b]))
    return psi / np.linalg.norm(psi)


def test_propagation_gradient(dev):
    """exp(-i H t) psi0 by 256 Chebyshev terms (checkpoints every 16 vectors);
    loss = sum_i o_i |psi_i|^2.  Gradient in H's values and psi0 against a
    dense torch matrix_exp reference, and against finite differences."""
    import torch

    from vbcsr_b200.autograd import chebyshev_coefficients, chebyshev_propagate

    from . import _gpu

    L = 10  # the propagation workload's 10 x 10 supercell
    H, _ = W.tmd_lattice(L, seed=7, bond_phase=True)
    assert np.iscomplexobj(H.values)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(11)
    t = 20.0
    assert abs(chebyshev_coefficients(1.0, t, 256)[-1]) < 1e-12
    psi0n = _wavepacket(H, L, rng)
    obs = torch.from_numpy(rng.uniform(size=H.N)).cuda()
    vals = torch.from_numpy(H.values.copy()).cuda().requires_grad_(True)
    psi0 = torch.from_numpy(psi0n).cuda().requires_grad_(True)

    def loss_of(v, p0=None):
        psi = chebyshev_propagate(v, psi0 if p0 is None else p0, dm, t, scale=1.0, num_terms=256, checkpoint=16)
        return (obs * (psi.conj() * psi).real).sum()

    loss = loss_of(vals)
    loss.backward()
    gV = vals.grad.detach().clone()
    gP = psi0.grad.detach().clone()

    # dense reference (FP64, torch autograd through matrix_exp)
    r, c = _dense_index(H)
    rr = torch.from_numpy(r).cuda()
    cc = torch.from_numpy(c).cuda()
    vref = torch.from_numpy(H.values.copy()).cuda().requires_grad_(True)
    pref = torch.from_numpy(psi0n).cuda().requires_grad_(True)
    Hd = torch.zeros((H.N, H.N), dtype=torch.complex128, device="cuda").index_put((rr, cc), vref, accumulate=True)
    U = torch.linalg.matrix_exp(-1j * t * Hd)
    psi_ref = U @ pref
    loss_ref = (obs * (psi_ref.conj() * psi_ref).real).sum()
    loss_ref.backward()
    assert abs(float(loss.detach()) - float(loss_ref.detach())) < 1e-10 * abs(float(loss_ref.detach()))
    assert float((gV - vref.grad).abs().max() / vref.grad.abs().max()) < 1e-9
    assert float((gP - pref.grad).abs().max() / pref.grad.abs().max()) < 1e-9

    idx = rng.choice(H.nnz, size=32, replace=False)
    _fd_check(lambda v: float(loss_of(v)), vals.detach(), gV, idx)


def test_kpm_moments_gradient(dev):
    import torch

    from vbcsr_b200.autograd import kpm_moments

    from . import _gpu

    H, _ = W.tmd_lattice(5, seed=8)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(3)
    V = torch.from_numpy(np.where(rng.random((H.N, 4)) < 0.5, -1.0, 1.0)).cuda()
    w = torch.from_numpy(rng.normal(size=40)).cuda()
    vals = torch.from_numpy(H.values.copy()).cuda().requires_grad_(True)

    def loss_of(v):
        return (w * kpm_moments(v, V, dm, 40, checkpoint=16)).sum()

    L = loss_of(vals)
    L.backward()
    idx = rng.choice(H.nnz, size=32, replace=False)
    _fd_check(lambda v: float(loss_of(v)), vals.detach(), vals.grad.detach().clone(), idx)

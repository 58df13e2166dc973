"""vbg_cheb_series (the whole Chebyshev series in one library call) against
the same series stepped term by term through vbg_cheb_step: psi and every
checkpoint pair (t_n, t_{n-1}), n = K, 2K, ...  Both run the same fused
apply kernel; the first apply of a matrix may run on a kernel the tuner
later drops, so the two are held to 1e-13 relative (of the largest entry)
rather than to the bit.  Hamiltonians: the TMD-like lattice (6 x 6 cells,
real, and complex with bond phases; spectrum inside [-0.95, 0.95])."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _stepped(op, scale, center, v, coeffs, K):
    """The series with one vbg_cheb_step per term (the reference's loop)."""
    import torch

    from vbcsr_b200.autograd import _cheb_step

    psi = torch.zeros_like(v) if v.dim() == 1 else torch.zeros(v.shape[0], v.stride(0), dtype=v.dtype,
                                                               device=v.device)[:, :v.shape[1]]
    psi.add_(v, alpha=complex(coeffs[0]) if v.is_complex() else float(np.real(coeffs[0])))
    ckpt = {0: (v, None)}
    t_prev, t = None, v
    for n in range(1, len(coeffs)):
        t_next = _cheb_step(op, scale, center, t, t_prev, n == 1, acc=psi, coef=coeffs[n])
        t_prev, t = t, t_next
        if n % K == 0:
            ckpt[n] = (t, t_prev)
    return psi, ckpt


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("k", [0, 3, 8])
@pytest.mark.parametrize("M,K", [(1, 16), (7, 16), (64, 16), (50, 7), (9, 1), (10, 2), (17, 16)])
def test_series_matches_steps(dev, cplx, k, M, K):
    import torch

    from vbcsr_b200.autograd import _cheb_series, _padded

    from . import _gpu

    H, _ = W.tmd_lattice(6, seed=5, bond_phase=cplx)
    assert np.iscomplexobj(H.values) == cplx
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(M * 100 + K + k)
    dt = torch.complex128 if cplx else torch.float64
    shape = (H.N,) if k == 0 else (H.N, k)
    vn = rng.standard_normal(shape) + (1j * rng.standard_normal(shape) if cplx else 0)
    v = _padded(torch.from_numpy(vn).to(dt).cuda())
    coeffs = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    scale, center = 1.1, 0.05
    psi, _, ck = _cheb_series(dm, scale, center, v, coeffs, K)
    psi_ref, ck_ref = _stepped(dm, scale, center, v, coeffs, K)
    torch.cuda.synchronize()
    tol = 1e-13

    def close(a, b):
        assert a.shape == b.shape
        d = float((a - b).abs().max())
        assert d <= tol * max(float(b.abs().max()), 1e-300), d

    close(psi, psi_ref)
    assert sorted(ck) == sorted(ck_ref) == [0] + list(range(K, M, K))
    for n in ck:
        if n == 0:
            continue
        close(ck[n][0], ck_ref[n][0])
        close(ck[n][1], ck_ref[n][1])


def test_series_argument_errors(dev):
    import ctypes as C

    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H, _ = W.tmd_lattice(4, seed=1)
    dm = _gpu.dmat(H)
    v = torch.ones(H.N, dtype=torch.float64, device="cuda")
    psi = torch.empty_like(v)
    c = np.ones((4, 2))
    cp = c.ctypes.data_as(C.c_void_p)
    with pytest.raises(RuntimeError):  # K > 0, M > K and no checkpoint buffer
        _capi.call("vbg_cheb_series", dm.h, 1, 1, C.c_void_p(v.data_ptr()), 4, cp, 1.0, 0.0,
                   C.c_void_p(psi.data_ptr()), 2, None, None)
    with pytest.raises(RuntimeError):  # scale 0
        _capi.call("vbg_cheb_series", dm.h, 1, 1, C.c_void_p(v.data_ptr()), 4, cp, 0.0, 0.0,
                   C.c_void_p(psi.data_ptr()), 0, None, None)
    with pytest.raises(RuntimeError):  # ld < k
        _capi.call("vbg_cheb_series", dm.h, 2, 1, C.c_void_p(v.data_ptr()), 4, cp, 1.0, 0.0,
                   C.c_void_p(psi.data_ptr()), 0, None, None)

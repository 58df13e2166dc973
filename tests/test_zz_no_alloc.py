"""vbg_cheb_step_noalloc: the fused Chebyshev step for callers that cannot let
the library allocate device memory (callers that own all device memory through
their own pool, or that must not synchronise the device inside the call).  It
reduces its dot products through a fixed array inside the library instead of
scratch allocated on first use.

Checked through the C ABI against vbg_cheb_step on the same inputs, twice in a
row (the array keeps the previous call's contents), for multivectors and a
plain vector, at the 1e-12 relative tolerance of the other parity tests.  This
file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from vbcsr_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _run(capi, dm, entry, k, ld, X, P, D, A0, with_dotw):
    import torch

    vp = C.c_void_p
    Y = torch.zeros_like(X)
    acc = A0.clone()
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    capi.call(entry, dm.h, k, ld, 1.7, -0.3, -1.0, vp(X.data_ptr()), vp(P.data_ptr()), vp(Y.data_ptr()),
              vp(D.data_ptr()) if with_dotw else None, vp(dots.data_ptr()), vp(acc.data_ptr()), 0.25, 0.0, None)
    torch.cuda.synchronize()
    return Y.cpu().numpy(), acc.cpu().numpy(), dots.cpu().numpy()


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("case", ["tmd_k16", "sym_k64_dotw", "sym_vector"])
def test_noalloc_matches_cheb_step(case):
    from vbcsr_b200 import _capi

    from . import _gpu

    if case == "tmd_k16":
        H, _ = W.tmd_lattice(12, seed=21)
        k, with_dotw = 16, False
    elif case == "sym_k64_dotw":
        H = W.random_symmetric_blocks(400, seed=22)
        k, with_dotw = 64, True
    else:
        H = W.random_symmetric_blocks(300, seed=23)
        k, with_dotw = 1, False
    dm = _gpu.dmat(H)
    ld = _gpu.ld_for(k, np.float64)
    rng = np.random.default_rng(7)
    X, P, D, A0 = (_gpu.to_dev_mv(rng.normal(size=(H.N, k)), ld, np.float64) for _ in range(4))
    ref = _run(_capi, dm, "vbg_cheb_step", k, ld, X, P, D, A0, with_dotw)
    for _ in range(2):  # two calls in a row share the static scratch
        got = _run(_capi, dm, "vbg_cheb_step_noalloc", k, ld, X, P, D, A0, with_dotw)
        assert _rel(got[0], ref[0]) < TOL
        assert _rel(got[1], ref[1]) < TOL
        assert _rel(got[2], ref[2]) < TOL
    # and the dots agree with their definition, not just with each other
    Y = got[0][:, :k]
    Dh = (D.cpu().numpy() if with_dotw else X.cpu().numpy())[:, :k]
    assert abs(got[2][0] - np.sum(Dh * Y)) <= TOL * np.sum(np.abs(Dh * Y))
    assert abs(got[2][1] - np.sum(Y * Y)) <= TOL * np.sum(Y * Y)


@pytest.mark.parametrize("k", [16, 64])
def test_noalloc_first_call_on_fresh_matrix(k):
    """The call a no-allocation caller makes first: on a freshly uploaded
    matrix, before any other apply has built the library's derived layouts.
    Free device memory is the same before and after the call, and the
    results agree with a later vbg_cheb_step on the same inputs (which does
    build the layouts and may pick another kernel)."""
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H, _ = W.tmd_lattice(16, seed=25)
    ld = _gpu.ld_for(k, np.float64)
    rng = np.random.default_rng(9)
    X, P, D, A0 = (_gpu.to_dev_mv(rng.normal(size=(H.N, k)), ld, np.float64) for _ in range(4))
    # a first call on another fresh matrix loads the kernels this path runs
    # (lazy module loading allocates on first launch) and looks up the array
    Hw, _ = W.tmd_lattice(6, seed=26)
    warm = [_gpu.to_dev_mv(rng.normal(size=(Hw.N, k)), ld, np.float64) for _ in range(4)]
    _run(_capi, _gpu.dmat(Hw), "vbg_cheb_step_noalloc", k, ld, *warm, False)
    dm = _gpu.dmat(H)
    Y = torch.zeros_like(X)
    acc = A0.clone()
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    vp = C.c_void_p
    for _ in range(2):
        acc.copy_(A0)
        torch.cuda.synchronize()
        _capi.call("vbg_cheb_step_noalloc", dm.h, k, ld, 1.7, -0.3, -1.0, vp(X.data_ptr()), vp(P.data_ptr()),
                   vp(Y.data_ptr()), None, vp(dots.data_ptr()), vp(acc.data_ptr()), 0.25, 0.0, None)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
    got = (Y.cpu().numpy(), acc.cpu().numpy(), dots.cpu().numpy())
    ref = _run(_capi, dm, "vbg_cheb_step", k, ld, X, P, D, A0, False)
    for g, r in zip(got, ref):
        assert _rel(g, r) < TOL


def test_noalloc_requires_dots():
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H = W.random_symmetric_blocks(50, seed=24)
    dm = _gpu.dmat(H)
    X = torch.zeros((H.N, 8), dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(X)
    vp = C.c_void_p
    with pytest.raises(RuntimeError, match="dots is required"):
        _capi.call("vbg_cheb_step_noalloc", dm.h, 3, 8, 1.0, 0.0, 0.0, vp(X.data_ptr()), None, vp(Y.data_ptr()),
                   None, None, None, 0.0, 0.0, None)

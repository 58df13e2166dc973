"""The apply autotuner: the first forward multivector apply on a matrix times
the kernels that can run it and keeps the fastest.  Checked: the tuned
choice is reported and kept, the trials leave the accumulator alone (it is
updated exactly once), results match the oracle at 1e-12, and the KPM
recurrence tunes before its graph capture."""
import ctypes as C

import numpy as np
import pytest

from vbcsr_b200 import workloads as W

from .conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def autotune_on():
    from vbcsr_b200 import _capi

    _capi.set_option("apply.chain", 2)
    _capi.set_option("apply.autotune", 1)
    yield
    _capi.set_option("apply.autotune", 1)


@pytest.mark.parametrize("k", [16, 64])
def test_tuned_cheb_step(oracle, dev, k):
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H, _ = W.tmd_lattice(20, seed=70 + k)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(k)
    X, P, A0 = (rng.normal(size=(H.N, k)) for _ in range(3))
    xb, pb, ab = (_gpu.to_dev_mv(Z, k, np.float64) for Z in (X, P, A0))
    yb = torch.zeros_like(xb)
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    vp = C.c_void_p
    _capi.call("vbg_cheb_step", dm.h, k, k, 2.0, 0.0, -1.0, vp(xb.data_ptr()), vp(pb.data_ptr()), vp(yb.data_ptr()),
               None, vp(dots.data_ptr()), vp(ab.data_ptr()), 0.5, 0.0, None)
    torch.cuda.synchronize()
    choice = _capi.apply_kernel(dm, k)
    assert choice in ("chain", "tile", "pipe")
    # the tiled kernel was timed at tile heights 16, 12 and 8: the kept plan
    # has at most the chosen height's block rows
    rows = _capi.apply_tile_rows(dm, k)
    assert rows in (4, 6, 8, 10, 12, 16)
    Y = 2.0 * oracle.apply(H, X) - P
    assert rel_err(yb.cpu().numpy(), Y) < 1e-12
    assert rel_err(ab.cpu().numpy(), A0 + 0.5 * Y) < 1e-12  # accumulated once, not per trial
    d = dots.cpu().numpy()
    assert abs(d[1] - np.sum(Y * Y)) / np.sum(Y * Y) < 1e-12
    # the choice is kept
    _capi.call("vbg_spmm", dm.h, k, k, vp(xb.data_ptr()), vp(yb.data_ptr()), None)
    torch.cuda.synchronize()
    assert _capi.apply_kernel(dm, k) == choice
    assert rel_err(yb.cpu().numpy(), oracle.apply(H, X)) < 1e-12


def test_tuned_kpm_graph(oracle, dev):
    from vbcsr_b200 import _capi

    from . import _gpu

    H, _ = W.tmd_lattice(14, seed=77)
    dm = _gpu.dmat(H)
    V = np.where(np.random.default_rng(3).random((H.N, 64)) < 0.5, -1.0, 1.0)
    ref = oracle.kpm_moments(H, V, 40, True)
    for _ in range(2):
        mu = _gpu.kpm_moments(dm, V, 40, precision=0, use_graph=True)
        assert np.abs(mu - ref).max() / abs(ref[0]) < 1e-12
    assert _capi.apply_kernel(dm, 64) in ("chain", "tile", "pipe")
    mu32 = _gpu.kpm_moments(dm, V, 40, precision=1, use_graph=True)
    assert np.abs(mu32 - ref).max() / abs(ref[0]) < 1e-5
    assert _capi.apply_kernel(dm, 64, precision=1) in ("chain", "tile", "pipe")


def test_autotune_off_uses_default_order(dev):
    from vbcsr_b200 import _capi

    from . import _gpu

    _capi.set_option("apply.autotune", 0)
    H, _ = W.tmd_lattice(12, seed=78)
    dm = _gpu.dmat(H)
    assert _capi.apply_kernel(dm, 64) == "tile"
    assert _capi.apply_kernel(dm, 64, precision=1) == "chain"
    assert _capi.get_option("apply.autotune") == 0

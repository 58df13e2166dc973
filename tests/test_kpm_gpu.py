"""Fused Chebyshev step and the KPM moment loop on the GPU against the CPU
oracle (FP64: 1e-12 relative to mu_0) and the FP32-bulk path's DOS error."""
import ctypes as C

import numpy as np
import pytest

from vbcsr_b200 import workloads as W
from vbcsr_b200 import kpm as K

from .conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lattice():
    H, g = W.tmd_lattice(10, seed=5)
    V = np.where(np.random.default_rng(9).random((H.N, 8)) < 0.5, -1.0, 1.0)
    return H, V


@pytest.mark.parametrize("two_moment", [True, False])
@pytest.mark.parametrize("M", [1, 2, 3, 4, 7, 64])
def test_moments_fp64(lattice, oracle, dev, two_moment, M):
    from . import _gpu

    H, V = lattice
    dm = _gpu.dmat(H)
    mu = _gpu.kpm_moments(dm, V, M, 0, two_moment)
    ref = oracle.kpm_moments(H, V, M, two_moment)
    assert np.abs(mu - ref).max() / abs(ref[0]) < 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_moments_64_vectors(oracle, dev, precision):
    """64 random vectors: the pipelined multivector kernel (FP64 and FP32)."""
    from . import _gpu

    H, _ = W.tmd_lattice(12, seed=7)
    V = np.where(np.random.default_rng(11).random((H.N, 64)) < 0.5, -1.0, 1.0)
    dm = _gpu.dmat(H)
    mu = _gpu.kpm_moments(dm, V, 48, precision, True, use_graph=True)
    ref = oracle.kpm_moments(H, V, 48, True)
    assert np.abs(mu - ref).max() / abs(ref[0]) < (1e-12 if precision == 0 else 1e-5)


def test_moments_single_vector(lattice, oracle, dev):
    from . import _gpu

    H, V = lattice
    dm = _gpu.dmat(H)
    mu = _gpu.kpm_moments(dm, V[:, :1], 32)
    ref = oracle.kpm_moments(H, V[:, :1], 32, True)
    assert np.abs(mu - ref).max() / abs(ref[0]) < 1e-12


def test_moments_graph_replay(lattice, oracle, dev):
    from . import _gpu

    H, V = lattice
    dm = _gpu.dmat(H)
    a = _gpu.kpm_moments(dm, V, 40, use_graph=True)
    b = _gpu.kpm_moments(dm, V, 40, use_graph=True)  # replay
    ref = oracle.kpm_moments(H, V, 40, True)
    assert np.array_equal(a, b)
    assert np.abs(a - ref).max() / abs(ref[0]) < 1e-12


def test_moments_against_reference(lattice, reference, dev):
    from . import _gpu

    H, V = lattice
    dm = _gpu.dmat(H)
    mu = _gpu.kpm_moments(dm, V, 48, 0, False)
    ref = reference.matrix(H).kpm_moments(V, 48)
    assert np.abs(mu - ref).max() / abs(ref[0]) < 1e-12


def test_fp32_bulk_dos_error(dev):
    """FP32 storage/arithmetic with FP64 moment sums: DOS within 1e-5 (relative
    to the DOS maximum) of the FP64 GPU result on the same vectors."""
    from . import _gpu

    H, _ = W.tmd_lattice(24, seed=6)
    V = np.where(np.random.default_rng(10).random((H.N, 16)) < 0.5, -1.0, 1.0)
    dm = _gpu.dmat(H)
    M = 256
    mu64 = _gpu.kpm_moments(dm, V, M, 0)
    mu32 = _gpu.kpm_moments(dm, V, M, 1)
    x, d64 = K.dos_from_moments(mu64 / (16 * H.N), 400)
    _, d32 = K.dos_from_moments(mu32 / (16 * H.N), 400)
    err = np.abs(d32 - d64).max() / np.abs(d64).max()
    assert err < 1e-5, err


def test_fp32_bulk_dos_error_full_config(dev):
    """The KPM workload at its own size: TMD 200 x 200 (N = 440,000), 64
    Rademacher vectors, 1024 moments, Jackson kernel, DOS on 2000 Chebyshev
    nodes: the FP32-bulk DOS within 1e-5 (relative to the DOS maximum) of the
    FP64 GPU DOS on the same vectors, and the FP64 moments' first entry the
    exact value mu_0 = R N."""
    from . import _gpu

    H, _ = W.tmd_lattice(200, seed=2)
    R, M = 64, 1024
    V = np.where(np.random.default_rng(11).random((H.N, R)) < 0.5, -1.0, 1.0)
    dm = _gpu.dmat(H)
    mu64 = _gpu.kpm_moments(dm, V, M, 0, use_graph=True)
    mu32 = _gpu.kpm_moments(dm, V, M, 1, use_graph=True)
    assert abs(mu64[0] - R * H.N) <= 1e-9 * R * H.N
    _, d64 = K.dos_from_moments(mu64 / (R * H.N), 2000)
    _, d32 = K.dos_from_moments(mu32 / (R * H.N), 2000)
    err = np.abs(d32 - d64).max() / np.abs(d64).max()
    assert err < 1e-5, err


@pytest.mark.parametrize("k", [6, 64, 128])
def test_cheb_step_epilogue(oracle, dev, k):
    """Y = alpha A X + beta X + gamma Xprev with dots and an accumulator
    (k = 64, 128: the pipelined kernel; one and two warp-width chunks)."""
    import torch

    from vbcsr_b200 import _capi
    from . import _gpu

    H = W.random_symmetric_blocks(150, seed=51)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(8)
    ld = _gpu.ld_for(k, np.float64)
    X, P, D, A0 = (rng.normal(size=(H.N, k)) for _ in range(4))
    xb, pb, db, ab = (_gpu.to_dev_mv(Z, ld, np.float64) for Z in (X, P, D, A0))
    yb = torch.zeros_like(xb)
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    vp = C.c_void_p
    _capi.call("vbg_cheb_step", dm.h, k, ld, 1.7, -0.3, -1.0, vp(xb.data_ptr()), vp(pb.data_ptr()),
               vp(yb.data_ptr()), vp(db.data_ptr()), vp(dots.data_ptr()), vp(ab.data_ptr()), 0.25, 0.0, None)
    torch.cuda.synchronize()
    Y = 1.7 * oracle.apply(H, X) - 0.3 * X - 1.0 * P
    assert rel_err(yb.cpu().numpy()[:, :k], Y) < 1e-12
    d = dots.cpu().numpy()
    assert abs(d[0] - np.sum(D * Y)) / abs(np.sum(np.abs(D * Y))) < 1e-12
    assert abs(d[1] - np.sum(Y * Y)) / np.sum(Y * Y) < 1e-12
    assert rel_err(ab.cpu().numpy()[:, :k], A0 + 0.25 * Y) < 1e-12


def test_device_status_clean(dev):
    """No pipelined apply in this module gave up waiting for staged data."""
    from vbcsr_b200 import _capi

    assert _capi.device_status(clear=True) == 0


def test_sharded_moments_single_process_device(oracle, dev):
    """The sharding helper's default (device) moment function, one process."""
    from vbcsr_b200 import distributed as D

    H, _ = W.tmd_lattice(6, seed=12)
    mu = D.kpm_moments_sharded(H, 32, 8, seed=4)
    ref = oracle.kpm_moments(H, D.rademacher_columns(H.N, 0, 8, 4), 32, True)
    assert np.abs(mu - ref).max() / abs(ref[0]) < 1e-12

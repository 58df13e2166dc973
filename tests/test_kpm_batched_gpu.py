"""Batched KPM: many Hamiltonians of uneven size in one device recurrence
(vbg_kpm_moments_batched) against the per-matrix FP64 moment loop on the same
vectors (1e-12 relative to mu_0) and the oracle, and the FP32 bulk batch's
DOS error (<= 1e-5)."""
import numpy as np
import pytest

from vbcsr_b200 import kpm as K
from vbcsr_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _batch(seed=4):
    return [W.tmd_lattice(L, seed=seed + L, disorder=1.0)[0] for L in (3, 7, 5, 4, 6)]


@pytest.mark.parametrize("R", [16, 64])
@pytest.mark.parametrize("two_moment", [True, False])
def test_batched_matches_single(dev, oracle, R, two_moment):
    from . import _gpu

    Hs = _batch()
    rng = np.random.default_rng(R)
    vecs = [np.where(rng.random((h.N, R)) < 0.5, -1.0, 1.0) for h in Hs]
    M = 40
    mu, sizes = K.batched_kpm_moments(Hs, M, precision="fp64", two_moment=two_moment, vectors=vecs)
    assert mu.shape == (len(Hs), M)
    for i, h in enumerate(Hs):
        ref = _gpu.kpm_moments(_gpu.dmat(h), vecs[i], M, 0, two_moment)
        assert np.abs(mu[i] - ref).max() / abs(ref[0]) < 1e-12, i
        assert sizes[i] == h.N
    o = oracle.kpm_moments(Hs[1], vecs[1], M, two_moment)
    assert np.abs(mu[1] - o).max() / abs(o[0]) < 1e-12


def test_batched_fp32_dos_error(dev):
    Hs = _batch(seed=9)
    M = 128
    mu64, sizes = K.batched_kpm_moments(Hs, M, num_random_vecs=16, precision="fp64", seed=3)
    mu32, _ = K.batched_kpm_moments(Hs, M, num_random_vecs=16, precision="fp32", seed=3)
    for i in range(len(Hs)):
        _, d64 = K.dos_from_moments(mu64[i] / (16 * sizes[i]), 300)
        _, d32 = K.dos_from_moments(mu32[i] / (16 * sizes[i]), 300)
        assert np.abs(d32 - d64).max() / np.abs(d64).max() < 1e-5


def test_batched_graph_replay_and_layout_change(dev):
    Hs = _batch(seed=11)
    a, _ = K.batched_kpm_moments(Hs, 24, seed=1, use_graph=True)
    b, _ = K.batched_kpm_moments(Hs, 24, seed=1, use_graph=True)
    assert np.array_equal(a, b)
    c, _ = K.batched_kpm_moments(Hs[:3], 24, seed=1, use_graph=True)
    assert c.shape == (3, 24)


def test_device_status_clean(dev):
    from vbcsr_b200 import _capi

    assert _capi.device_status(clear=True) == 0

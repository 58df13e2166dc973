"""The row-tiled multivector apply against the oracle -- both variants: the
chained tiles (apply_chain_kernel, X rows cached across the tiles of a
persistent CTA; library option "apply.chain" = 1) and the unchained tiles
(apply_tile_kernel, "apply.chain" = 0) -- and the kernel choice between them and
the pipelined apply.

Bar: FP64 and complex results 1e-12 relative; FP32 KPM moments within 1e-5 of
mu_0 of the FP64 ones; per-row dots of the batched recurrence 1e-12."""
import ctypes as C

import numpy as np
import pytest

from vbcsr_b200 import workloads as W

from .conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["chain", "tile"], autouse=True)
def tiles(request):
    """Runs each test with the chained tiles and again with the unchained
    ones; the option is process-wide and restored afterwards."""
    from vbcsr_b200 import _capi

    _capi.set_option("apply.chain", 1 if request.param == "chain" else 0)
    yield request.param
    _capi.set_option("apply.chain", 2)


@pytest.fixture(scope="module")
def lattice():
    # 11 x 11 cells: 363 block rows, the last tile shorter than the others
    H, _ = W.tmd_lattice(11, seed=21)
    return H


def test_kernel_choice(lattice, dev, tiles):
    """Lattice at warp-wide rows: tiled; far-apart neighbours: pipelined;
    narrower rows: pipelined; real vectors: a warp per block row until the
    autotuner decides, complex vectors: the scalar-row kernel."""
    from vbcsr_b200 import _capi

    from . import _gpu

    dm = _gpu.dmat(lattice)
    assert _capi.apply_kernel(dm, 64) == tiles
    assert _capi.apply_kernel(dm, 64, precision=1) == tiles
    assert _capi.apply_kernel(dm, 16) == tiles
    assert _capi.apply_kernel(dm, 128) == "pipe"
    assert _capi.apply_kernel(dm, 1) == "vector"
    Z, _ = W.tmd_lattice(7, seed=3, bond_phase=True, dtype=np.complex128)
    assert _capi.apply_kernel(_gpu.dmat(Z), 32) == tiles
    # complex vectors before the autotuner has run: the scalar-row kernel
    assert _capi.apply_kernel(_gpu.dmat(Z), 1) == "scalar_rows"
    far = W.random_pattern(3000, 4, 8, 12, seed=5)
    assert _capi.apply_kernel(_gpu.dmat(far), 64) == "pipe"


@pytest.mark.parametrize("with_dots", [True, False])
def test_tile_cheb_step(lattice, oracle, dev, with_dots, tiles):
    """Y = alpha A X + beta X + gamma Xprev, dots and accumulator, k = 64."""
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H = lattice
    dm = _gpu.dmat(H)
    assert _capi.apply_kernel(dm, 64) == tiles
    rng = np.random.default_rng(31)
    k = ld = 64
    X, P, D, A0 = (rng.normal(size=(H.N, k)) for _ in range(4))
    xb, pb, db, ab = (_gpu.to_dev_mv(Z, ld, np.float64) for Z in (X, P, D, A0))
    yb = torch.zeros_like(xb)
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    vp = C.c_void_p
    _capi.call("vbg_cheb_step", dm.h, k, ld, 1.7, -0.3, -1.0, vp(xb.data_ptr()), vp(pb.data_ptr()),
               vp(yb.data_ptr()), vp(db.data_ptr()) if with_dots else None,
               vp(dots.data_ptr()) if with_dots else None, vp(ab.data_ptr()), 0.25, 0.0, None)
    torch.cuda.synchronize()
    Y = 1.7 * oracle.apply(H, X) - 0.3 * X - 1.0 * P
    assert rel_err(yb.cpu().numpy(), Y) < 1e-12
    assert rel_err(ab.cpu().numpy(), A0 + 0.25 * Y) < 1e-12
    if with_dots:
        d = dots.cpu().numpy()
        assert abs(d[0] - np.sum(D * Y)) / np.sum(np.abs(D * Y)) < 1e-12
        assert abs(d[1] - np.sum(Y * Y)) / np.sum(Y * Y) < 1e-12
    assert _capi.device_status(clear=True) == 0


def test_tile_plain_apply_repeated(lattice, oracle, dev):
    """Y = A X through vbg_spmm, twice on the same plan (the second apply
    reuses it), and A (A X)."""
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H = lattice
    dm = _gpu.dmat(H)
    X = np.random.default_rng(2).normal(size=(H.N, 64))
    Y1 = _gpu.apply(dm, X)
    Y2 = _gpu.apply(dm, Y1)
    assert rel_err(Y1, oracle.apply(H, X)) < 1e-12
    assert rel_err(Y2, oracle.apply(H, oracle.apply(H, X))) < 1e-12
    assert _capi.device_status(clear=True) == 0
    torch.cuda.synchronize()


def _drop_blocks(H, keep):
    """H with only the slots s where keep(i, j) holds (i the block row, j the
    block column)."""
    off = H.slot_offsets()
    rp, ci, vals = [0], [], []
    for i in range(H.n):
        for s in range(H.row_ptr[i], H.row_ptr[i + 1]):
            j = int(H.col_ind[s])
            if keep(i, j):
                ci.append(j)
                vals.append(H.values[off[s]:off[s + 1]])
        rp.append(len(ci))
    return W.BlockCSR(H.block_sizes, np.array(rp, np.int32), np.array(ci, np.int32),
                      np.concatenate(vals) if vals else np.zeros(0, H.values.dtype))


def test_tile_edge_rows(oracle, dev, tiles):
    """Banded matrix (block sizes 4..8, n not a multiple of the tile height)
    with empty block rows and rows without a diagonal block: the tile's own
    X rows are staged even when no block reads them (beta X term)."""
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    B = W.banded_decaying(605, neighbours=4, band=6, seed=17)
    H = _drop_blocks(B, lambda i, j: i % 11 != 0 and not (i % 7 == 0 and i == j))
    dm = _gpu.dmat(H)
    assert _capi.apply_kernel(dm, 64) == tiles
    rng = np.random.default_rng(5)
    X, P = rng.normal(size=(H.N, 64)), rng.normal(size=(H.N, 64))
    xb, pb = _gpu.to_dev_mv(X, 64, np.float64), _gpu.to_dev_mv(P, 64, np.float64)
    yb = torch.zeros_like(xb)
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    vp = C.c_void_p
    _capi.call("vbg_cheb_step", dm.h, 64, 64, 2.0, 0.5, -1.0, vp(xb.data_ptr()), vp(pb.data_ptr()),
               vp(yb.data_ptr()), None, vp(dots.data_ptr()), None, 0.0, 0.0, None)
    torch.cuda.synchronize()
    Y = 2.0 * oracle.apply(H, X) + 0.5 * X - P
    assert rel_err(yb.cpu().numpy(), Y) < 1e-12
    d = dots.cpu().numpy()
    assert abs(d[0] - np.sum(X * Y)) / np.sum(np.abs(X * Y)) < 1e-12
    assert abs(d[1] - np.sum(Y * Y)) / np.sum(Y * Y) < 1e-12
    assert _capi.device_status(clear=True) == 0


def test_tile_complex_apply(oracle, dev, tiles):
    """Complex lattice with Peierls-like bond phases, k = 32 (one 16-byte
    complex per lane)."""
    from vbcsr_b200 import _capi

    from . import _gpu

    Z, _ = W.tmd_lattice(7, seed=3, bond_phase=True, dtype=np.complex128)
    dm = _gpu.dmat(Z)
    assert _capi.apply_kernel(dm, 32) == tiles
    rng = np.random.default_rng(4)
    X = rng.normal(size=(Z.N, 32)) + 1j * rng.normal(size=(Z.N, 32))
    assert rel_err(_gpu.apply(dm, X), oracle.apply(Z, X)) < 1e-12


def test_tile_kpm_fp64_and_fp32(lattice, oracle, dev):
    """KPM moments with 64 vectors: FP64 on the tiled kernel equal the oracle's
    to 1e-12 of mu_0 (graph replay included); FP32 within 1e-5."""
    from . import _gpu

    H = lattice
    dm = _gpu.dmat(H)
    V = np.where(np.random.default_rng(6).random((H.N, 64)) < 0.5, -1.0, 1.0)
    M = 48
    ref = oracle.kpm_moments(H, V, M, True)
    mu = _gpu.kpm_moments(dm, V, M, precision=0, use_graph=True)
    assert np.abs(mu - ref).max() / abs(ref[0]) < 1e-12
    mu2 = _gpu.kpm_moments(dm, V, M, precision=0, use_graph=True)  # replay
    assert np.abs(mu2 - ref).max() / abs(ref[0]) < 1e-12
    mu32 = _gpu.kpm_moments(dm, V, M, precision=1)
    assert np.abs(mu32 - ref).max() / abs(ref[0]) < 1e-5


def test_tile_batched_row_dots(oracle, dev):
    """Batched recurrence (per-row dots) over two lattices with 64 vectors each."""
    from vbcsr_b200 import kpm as K

    Hs = [W.tmd_lattice(L, seed=40 + L)[0] for L in (6, 9)]
    rng = np.random.default_rng(12)
    Vs = [np.where(rng.random((H.N, 64)) < 0.5, -1.0, 1.0) for H in Hs]
    mu, _ = K.batched_kpm_moments(Hs, 24, num_random_vecs=64, precision="fp64", vectors=Vs)
    for i, H in enumerate(Hs):
        ref = oracle.kpm_moments(H, Vs[i], 24, True)
        assert np.abs(mu[i] - ref).max() / abs(ref[0]) < 1e-12


def test_tile_fp32_32_columns(lattice, oracle, dev, tiles):
    """FP32 at 32 columns runs the tiled kernel with one scalar per lane: KPM
    moments of 32 vectors within 1e-5 of mu_0 of the oracle's FP64 ones; the
    batched FP32 recurrence at 16 vectors per Hamiltonian (padded with zero
    columns to 32) likewise, per Hamiltonian."""
    from vbcsr_b200 import _capi
    from vbcsr_b200 import kpm as K

    from . import _gpu

    H = lattice
    dm = _gpu.dmat(H)
    assert _capi.apply_kernel(dm, 32, precision=1) == tiles
    rng = np.random.default_rng(8)
    V = np.where(rng.random((H.N, 32)) < 0.5, -1.0, 1.0)
    ref = oracle.kpm_moments(H, V, 48, True)
    mu32 = _gpu.kpm_moments(dm, V, 48, precision=1)
    assert np.abs(mu32 - ref).max() / abs(ref[0]) < 1e-5
    Hs = [W.tmd_lattice(L, seed=50 + L)[0] for L in (5, 8)]
    B, _ = W.block_diagonal(Hs)
    assert _capi.apply_kernel(_gpu.dmat(B), 32, precision=1) == tiles
    Vs = [np.where(rng.random((h.N, 16)) < 0.5, -1.0, 1.0) for h in Hs]
    mu, _ = K.batched_kpm_moments(Hs, 24, num_random_vecs=16, precision="fp32", vectors=Vs)
    for i, h in enumerate(Hs):
        ref = oracle.kpm_moments(h, Vs[i], 24, True)
        assert np.abs(mu[i] - ref).max() / abs(ref[0]) < 1e-5
    assert _capi.device_status(clear=True) == 0


@pytest.mark.parametrize("L", [30, 47])
def test_tile_larger_lattice(oracle, dev, tiles, L):
    """Lattices whose tiles run in chains of many tiles per CTA (X rows
    reused from the cache across tiles): the fused step with dots against
    the oracle, FP64 at 64 columns.  L = 47 gives lattice rows that no tile
    height divides."""
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H, _ = W.tmd_lattice(L, seed=60 + L)
    dm = _gpu.dmat(H)
    assert _capi.apply_kernel(dm, 64) == tiles
    rng = np.random.default_rng(L)
    X, P = rng.normal(size=(H.N, 64)), rng.normal(size=(H.N, 64))
    xb, pb = _gpu.to_dev_mv(X, 64, np.float64), _gpu.to_dev_mv(P, 64, np.float64)
    yb = torch.zeros_like(xb)
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    vp = C.c_void_p
    for _ in range(2):  # the second call reuses the plan
        _capi.call("vbg_cheb_step", dm.h, 64, 64, 2.0, 0.0, -1.0, vp(xb.data_ptr()), vp(pb.data_ptr()),
                   vp(yb.data_ptr()), None, vp(dots.data_ptr()), None, 0.0, 0.0, None)
        torch.cuda.synchronize()
        Y = 2.0 * oracle.apply(H, X) - P
        assert rel_err(yb.cpu().numpy(), Y) < 1e-12
        d = dots.cpu().numpy()
        assert abs(d[0] - np.sum(X * Y)) / np.sum(np.abs(X * Y)) < 1e-12
        assert abs(d[1] - np.sum(Y * Y)) / np.sum(Y * Y) < 1e-12
    assert _capi.device_status(clear=True) == 0


@pytest.mark.parametrize("dtype", ["fp64", "fp32"])
def test_tile_16_columns(lattice, oracle, dev, tiles, dtype):
    """16 columns run on the tiled kernels with two lane groups (each half
    of the warp takes every other X row of a block row): FP64 cheb step with
    dots against the oracle at 1e-12; FP32 KPM moments of 16 vectors within
    1e-5 of mu_0."""
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    H = lattice
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(16)
    if dtype == "fp64":
        assert _capi.apply_kernel(dm, 16) == tiles
        X, P = rng.normal(size=(H.N, 16)), rng.normal(size=(H.N, 16))
        xb, pb = _gpu.to_dev_mv(X, 16, np.float64), _gpu.to_dev_mv(P, 16, np.float64)
        yb = torch.zeros_like(xb)
        dots = torch.zeros(2, dtype=torch.float64, device="cuda")
        vp = C.c_void_p
        _capi.call("vbg_cheb_step", dm.h, 16, 16, 2.0, 0.25, -1.0, vp(xb.data_ptr()), vp(pb.data_ptr()),
                   vp(yb.data_ptr()), None, vp(dots.data_ptr()), None, 0.0, 0.0, None)
        torch.cuda.synchronize()
        Y = 2.0 * oracle.apply(H, X) + 0.25 * X - P
        assert rel_err(yb.cpu().numpy(), Y) < 1e-12
        d = dots.cpu().numpy()
        assert abs(d[0] - np.sum(X * Y)) / np.sum(np.abs(X * Y)) < 1e-12
        assert abs(d[1] - np.sum(Y * Y)) / np.sum(Y * Y) < 1e-12
    else:
        assert _capi.apply_kernel(dm, 16, precision=1) == tiles
        V = np.where(rng.random((H.N, 16)) < 0.5, -1.0, 1.0)
        ref = oracle.kpm_moments(H, V, 40, True)
        mu32 = _gpu.kpm_moments(dm, V, 40, precision=1)
        assert np.abs(mu32 - ref).max() / abs(ref[0]) < 1e-5
    assert _capi.device_status(clear=True) == 0

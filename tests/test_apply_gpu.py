"""SpMV / SpMM and their adjoints on the GPU (through the C ABI) against the
CPU oracle, and against the reference core where it is built.
Tolerance: FP64 values to 1e-12 relative (max-norm)."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W

from .conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _cases():
    return {
        "vbcsr_sym": W.random_symmetric_blocks(300, seed=11),
        "vbcsr_wide": W.random_pattern(60, 1, 12, 5, seed=12),  # block sizes up to 12 (> 8 path)
        "csr": W.random_pattern(200, 1, 1, 6, seed=13),
        "bsr": W.random_pattern(80, 3, 3, 5, seed=14),
        "cplx": W.random_pattern(70, 2, 7, 4, seed=15, dtype=np.complex128),
        "single": W.random_pattern(1, 5, 5, 1, seed=16),
    }


@pytest.fixture(scope="module")
def cases():
    return _cases()


@pytest.mark.parametrize("name", list(_cases().keys()))
@pytest.mark.parametrize("adjoint", [False, True])
def test_spmv(cases, oracle, dev, name, adjoint):
    from . import _gpu

    H = cases[name]
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(1)
    x = rng.normal(size=H.N)
    if np.iscomplexobj(H.values):
        x = x + 1j * rng.normal(size=H.N)
    y = _gpu.apply(dm, x, adjoint)
    assert rel_err(y, oracle.apply(H, x, adjoint)) < TOL


@pytest.mark.parametrize("name", ["vbcsr_sym", "vbcsr_wide", "csr", "cplx"])
@pytest.mark.parametrize("k", [1, 3, 8, 16, 32, 64, 100, 128])
@pytest.mark.parametrize("adjoint", [False, True])
def test_spmm(cases, oracle, dev, name, k, adjoint):
    from . import _gpu

    H = cases[name]
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(k)
    X = rng.normal(size=(H.N, k))
    if np.iscomplexobj(H.values):
        X = X + 1j * rng.normal(size=(H.N, k))
    Y = _gpu.apply(dm, X, adjoint)
    assert rel_err(Y, oracle.apply(H, X, adjoint)) < TOL


def test_empty_rows_and_kinds(oracle, dev):
    from . import _gpu

    H = W.random_pattern(40, 2, 6, 3, seed=21)
    # drop every block of rows 5..9 (empty rows)
    keep_rows = np.ones(H.n, bool)
    keep_rows[5:10] = False
    rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
    off = H.slot_offsets()
    sel = keep_rows[rows]
    rp = np.zeros(H.n + 1, np.int32)
    np.add.at(rp, rows[sel] + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    vals = np.concatenate([H.values[off[s]:off[s + 1]] for s in np.nonzero(sel)[0]])
    E = W.BlockCSR(H.block_sizes, rp, H.col_ind[sel], vals)
    dm = _gpu.dmat(E)
    x = np.random.default_rng(3).normal(size=E.N)
    y = _gpu.apply(dm, x)
    assert rel_err(y, oracle.apply(E, x)) < TOL
    so = E.scalar_offsets()
    assert np.all(y[so[5]:so[10]] == 0)
    assert _gpu.dmat(W.random_pattern(10, 1, 1, 2, seed=1)).kind == "csr"
    assert _gpu.dmat(W.random_pattern(10, 4, 4, 2, seed=1)).kind == "bsr"
    assert dm.kind == "vbcsr"


def test_against_reference_core(reference, oracle, dev):
    from . import _gpu

    H = W.random_symmetric_blocks(400, seed=31)
    R = reference.matrix(H)
    dm = _gpu.dmat(H)
    x = np.random.default_rng(4).normal(size=H.N)
    assert rel_err(_gpu.apply(dm, x), R.mult(x)) < TOL
    X = np.random.default_rng(5).normal(size=(H.N, 16))
    assert rel_err(_gpu.apply(dm, X), R.mult_dense(X)) < TOL
    assert rel_err(_gpu.apply(dm, X, True), R.mult_dense(X, True)) < TOL


def test_host_buffer_entry_points(oracle, dev):
    import ctypes as C

    from vbcsr_b200 import _capi
    from . import _gpu

    H = W.random_symmetric_blocks(100, seed=41)
    dm = _gpu.dmat(H)
    x = np.random.default_rng(6).normal(size=H.N)
    y = np.zeros_like(x)
    _capi.call("vbg_spmv_host", dm.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), None)
    assert rel_err(y, oracle.apply(H, x)) < TOL
    X = np.random.default_rng(7).normal(size=(H.N, 5))
    Y = np.zeros_like(X)
    _capi.call("vbg_spmm_host", dm.h, 5, X.ctypes.data_as(C.c_void_p), Y.ctypes.data_as(C.c_void_p), None)
    assert rel_err(Y, oracle.apply(H, X)) < TOL


# (apply.vec_kernel, apply.vec_lanes): the autotuner; a warp per block row;
# scalar rows at 1, 2, 4, 8 threads per row
VEC_MODES = [(0, 0), (1, 0)] + [(2, s) for s in (1, 2, 4, 8)]


def _vec_mode(kernel, lanes):
    from vbcsr_b200 import _capi

    assert _capi.get_option("apply.vec_kernel") == 0 and _capi.get_option("apply.vec_lanes") == 0
    _capi.set_option("apply.vec_kernel", kernel)
    _capi.set_option("apply.vec_lanes", lanes)


def _vec_reset():
    from vbcsr_b200 import _capi

    _capi.set_option("apply.vec_kernel", 0)
    _capi.set_option("apply.vec_lanes", 0)


@pytest.mark.parametrize("adjoint", [False, True])
@pytest.mark.parametrize("mode", VEC_MODES)
@pytest.mark.parametrize("name", ["vbcsr_sym", "vbcsr_wide", "csr", "bsr", "cplx", "single", "empty_rows"])
def test_spmv_vec_kernels(cases, oracle, dev, name, mode, adjoint):
    """The vector apply and its adjoint on every vector kernel
    ("apply.vec_kernel": the scalar-row kernel, over the column view for the
    adjoint, or a warp per block row) and threads-per-row setting
    ("apply.vec_lanes"); blocks over 8 x 8 always take a warp per block
    row."""
    from vbcsr_b200 import _capi
    from . import _gpu

    if name == "empty_rows":
        H = W.random_pattern(40, 2, 6, 3, seed=21)
        rows = np.repeat(np.arange(H.n), np.diff(H.row_ptr))
        off = H.slot_offsets()
        sel = (rows < 5) | (rows >= 12)
        rp = np.concatenate([[0], np.cumsum(np.bincount(rows[sel], minlength=H.n))]).astype(np.int32)
        vals = np.concatenate([H.values[off[s]:off[s + 1]] for s in np.nonzero(sel)[0]])
        H = W.BlockCSR(H.block_sizes, rp, H.col_ind[sel], vals)
    else:
        H = cases[name]
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(mode[0] * 10 + mode[1])
    x = rng.normal(size=H.N)
    if np.iscomplexobj(H.values):
        x = x + 1j * rng.normal(size=H.N)
    _vec_mode(*mode)
    try:
        y = _gpu.apply(dm, x, adjoint)
        kern = _capi.apply_kernel(dm, 1)
    finally:
        _vec_reset()
    assert rel_err(y, oracle.apply(H, x, adjoint)) < TOL
    small = H.block_sizes.max() <= 8
    want = {1: "vector", 2: "scalar_rows"}.get(mode[0])
    if adjoint:
        pass
    elif not small:
        assert kern == "vector"
    elif want:
        assert kern == want
    else:
        assert kern in ("vector", "scalar_rows")
    if name == "empty_rows" and not adjoint:
        so = H.scalar_offsets()
        assert np.all(y[so[5]:so[12]] == 0)


@pytest.mark.parametrize("mode", VEC_MODES)
@pytest.mark.parametrize("cplx", [False, True])
def test_cheb_step_vec_kernels(oracle, dev, mode, cplx):
    """The fused vector step Y = a H X + b X + g Xprev with acc += c Y and the
    dots (Re <X, Y>, <Y, Y>) on every vector kernel, against numpy on the
    oracle's H X; then again after new values."""
    import ctypes as C

    import torch

    from vbcsr_b200 import _capi
    from . import _gpu

    H = W.random_pattern(500, 2, 8, 9, seed=17, dtype=np.complex128 if cplx else np.float64)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(3)
    dt = torch.complex128 if cplx else torch.float64

    def vec():
        v = rng.normal(size=H.N)
        return v + 1j * rng.normal(size=H.N) if cplx else v

    vp = C.c_void_p
    _vec_mode(*mode)
    try:
        for rep in range(2):
            if rep:
                H.values[:] = H.values * 0.5 + 0.25
                dm.set_values(H.values)
            x, xp, acc0 = vec(), vec(), vec()
            al, be, ga, c = 0.7, -0.3, -1.0, (0.25 - 0.5j) if cplx else 0.25
            X, Xp, A = (torch.from_numpy(v).to(dt).cuda() for v in (x, xp, acc0))
            Y = torch.zeros_like(X)
            dots = torch.zeros(2, dtype=torch.float64, device="cuda")
            _capi.call("vbg_cheb_step", dm.h, 1, 1, al, be, ga, vp(X.data_ptr()), vp(Xp.data_ptr()),
                       vp(Y.data_ptr()), None, vp(dots.data_ptr()), vp(A.data_ptr()), complex(c).real,
                       complex(c).imag, None)
            torch.cuda.synchronize()
            y = al * oracle.apply(H, x) + be * x + ga * xp
            assert rel_err(Y.cpu().numpy(), y) < TOL
            assert rel_err(A.cpu().numpy(), acc0 + c * y) < TOL
            d = dots.cpu().numpy()
            assert abs(d[0] - np.vdot(x, y).real) < 1e-11 * abs(np.vdot(y, y).real)
            assert abs(d[1] - np.vdot(y, y).real) < 1e-11 * abs(np.vdot(y, y).real)
    finally:
        _vec_reset()


@pytest.mark.parametrize("mode", [(0, 0), (1, 0), (2, 4)])
@pytest.mark.parametrize("k", [1, 3, 8])
@pytest.mark.parametrize("cplx", [False, True])
def test_cheb_step_adjoint(oracle, dev, k, cplx, mode):
    """vbg_cheb_step_adjoint: Y = a A^H X + b X + g Xprev, acc += c Y and the
    dots, against numpy on the oracle's adjoint apply (vectors and padded
    multivectors)."""
    import ctypes as C

    import torch

    from vbcsr_b200 import _capi
    from . import _gpu

    H = W.random_pattern(300, 2, 8, 7, seed=29, dtype=np.complex128 if cplx else np.float64)
    dm = _gpu.dmat(H)
    rng = np.random.default_rng(k)
    dt = np.complex128 if cplx else np.float64

    def mv():
        v = rng.normal(size=(H.N, k))
        return (v + 1j * rng.normal(size=(H.N, k))) if cplx else v

    x, xp, acc0 = mv(), mv(), mv()
    ld = _gpu.ld_for(k, dt) if k > 1 else 1
    X, Xp, A = (_gpu.to_dev_mv(v, ld, dt) for v in (x, xp, acc0))
    Y = torch.zeros_like(X)
    dots = torch.zeros(2, dtype=torch.float64, device="cuda")
    al, be, ga, c = 0.5, 0.2, -1.0, (1.5 + 0.5j) if cplx else 1.5
    vp = C.c_void_p
    _vec_mode(*mode)
    try:
        _capi.call("vbg_cheb_step_adjoint", dm.h, k, ld, al, be, ga, vp(X.data_ptr()), vp(Xp.data_ptr()),
                   vp(Y.data_ptr()), None, vp(dots.data_ptr()), vp(A.data_ptr()), complex(c).real, complex(c).imag,
                   None)
        torch.cuda.synchronize()
    finally:
        _vec_reset()
    xin = x[:, 0] if k == 1 else x
    y = al * oracle.apply(H, xin, True) + be * xin + ga * (xp[:, 0] if k == 1 else xp)
    y = y.reshape(H.N, k)
    Yh = Y.cpu().numpy()[:, :k]
    assert rel_err(Yh, y) < TOL
    assert rel_err(A.cpu().numpy()[:, :k], acc0 + c * y) < TOL
    d = dots.cpu().numpy()
    assert abs(d[0] - np.vdot(x, y).real) < 1e-11 * np.vdot(y, y).real
    assert abs(d[1] - np.vdot(y, y).real) < 1e-11 * np.vdot(y, y).real
    if ld > k:
        assert np.all(Yh.shape[1] == k) and np.all(Y.cpu().numpy()[:, k:] == 0)


def test_vec_option_values(dev):
    from vbcsr_b200 import _capi

    for bad in (3, 16, -1):
        with pytest.raises(RuntimeError):
            _capi.set_option("apply.vec_lanes", bad)
    for bad in (3, -1):
        with pytest.raises(RuntimeError):
            _capi.set_option("apply.vec_kernel", bad)
    assert _capi.get_option("apply.vec_lanes") == 0
    assert _capi.get_option("apply.vec_kernel") == 0


def test_device_status_clean(dev):
    """No pipelined apply in this module gave up waiting for staged data."""
    from vbcsr_b200 import _capi

    assert _capi.device_status(clear=True) == 0

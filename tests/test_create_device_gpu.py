"""Matrix construction from a structure already in device memory
(vbg_matrix_create_device): the same structure, kind, values and products
as the host constructor, real and complex; invalid structures (bad row
pointers, a column out of range, unsorted columns) are rejected with
VBG_E_ARG after the device-side check, without touching the data."""
import numpy as np
import pytest

from vbcsr_b200 import workloads as W

from .conftest import rel_err

pytestmark = pytest.mark.gpu


def _dev(H):
    import torch

    rp = torch.from_numpy(np.asarray(H.row_ptr, np.int32)).cuda()
    ci = torch.from_numpy(np.asarray(H.col_ind, np.int32)).cuda()
    v = torch.from_numpy(np.ascontiguousarray(H.values)).cuda()
    return rp, ci, v


@pytest.mark.parametrize("kind", ["tmd", "complex", "bsr", "csr"])
def test_create_device_matches_host(oracle, dev, kind):
    import torch

    from vbcsr_b200 import _capi

    from . import _gpu

    if kind == "tmd":
        H, _ = W.tmd_lattice(12, seed=41)
    elif kind == "complex":
        H, _ = W.tmd_lattice(8, seed=42, bond_phase=True)
    elif kind == "bsr":
        H = W.random_pattern(200, 4, 4, 5, seed=43)
    else:
        H = W.random_pattern(300, 1, 1, 6, seed=44)
    rp, ci, v = _dev(H)
    D = _capi.DeviceMatrix.create_device(H.block_sizes, rp, ci, v)
    Hh = _gpu.dmat(H)
    assert (D.n, D.nnzb, D.nnz, D.N, D.kind) == (Hh.n, Hh.nnzb, Hh.nnz, Hh.N, Hh.kind)
    G = D.to_blockcsr()
    assert np.array_equal(G.row_ptr, H.row_ptr) and np.array_equal(G.col_ind, H.col_ind)
    assert np.array_equal(G.values, H.values)
    rng = np.random.default_rng(1)
    for k in (1, 16):
        X = rng.normal(size=(H.N, k))
        if np.iscomplexobj(H.values):
            X = X + 1j * rng.normal(size=X.shape)
        want = oracle.apply(H, X)
        got = _gpu.apply(D, X)
        assert rel_err(got, want) < 1e-12
    # a product on the device-built matrix equals the one on the host-built one
    C1, _ = D.spgemm(D, 0.0)
    C2, _ = Hh.spgemm(Hh, 0.0)
    assert np.array_equal(C1.to_blockcsr().values, C2.to_blockcsr().values)


def test_create_device_rejects_bad_structures(dev):
    import torch

    from vbcsr_b200 import _capi

    H = W.random_pattern(50, 2, 5, 4, seed=45)
    rp, ci, v = _dev(H)
    bad_rp = rp.clone()
    bad_rp[5] = bad_rp[6] + 1  # not monotone
    with pytest.raises(RuntimeError, match="row_ptr"):
        _capi.DeviceMatrix.create_device(H.block_sizes, bad_rp, ci, v)
    bad_ci = ci.clone()
    bad_ci[3] = 50  # out of range
    with pytest.raises(RuntimeError, match="out of range"):
        _capi.DeviceMatrix.create_device(H.block_sizes, rp, bad_ci, v)
    uns = ci.clone()
    s0 = int(H.row_ptr[7])
    assert int(H.row_ptr[8]) - s0 >= 2
    uns[s0], uns[s0 + 1] = ci[s0 + 1], ci[s0]  # unsorted row
    with pytest.raises(RuntimeError, match="sorted"):
        _capi.DeviceMatrix.create_device(H.block_sizes, rp, uns, v)
    # the library is still usable afterwards
    D = _capi.DeviceMatrix.create_device(H.block_sizes, rp, ci, v)
    assert D.nnzb == H.nnzb

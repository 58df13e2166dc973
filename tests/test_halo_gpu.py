"""Row-partitioned apply on the GPU: each rank's local matrix (owned block
rows, columns renumbered owned-then-ghosts, empty ghost rows) multiplied by
the library, with the ghost rows of x supplied (one GPU runs every rank in
turn; the exchange itself is covered by the gloo tests).  Checked against
the oracle's product of the whole matrix at 1e-12, vectors and
multivectors, real and complex."""
import numpy as np
import pytest

from vbcsr_b200 import distributed as D
from vbcsr_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 4])
@pytest.mark.parametrize("kind", ["tmd", "complex"])
def test_row_partitioned_mult(oracle, dev, k, kind):
    import torch

    if kind == "tmd":
        H, _ = W.tmd_lattice(12, seed=9)
    else:
        H = W.random_pattern(150, 1, 6, 6, seed=10, dtype=np.complex128)
    rng = np.random.default_rng(k)
    x = rng.normal(size=(H.N, k))
    if np.iscomplexobj(H.values):
        x = x + 1j * rng.normal(size=x.shape)
    y = oracle.apply(H, x)
    so = H.scalar_offsets()
    world = 3
    parts = D.row_partition(H, world)
    for r in range(world):
        p = D.halo_plan_from_global(H, parts, r)
        op = D.RowPartitionedOperator(p, D.local_rows(H, *parts[r]).values)
        xo = x[so[parts[r][0]]:so[parts[r][1]]]
        xg = np.concatenate([x[so[g]:so[g + 1]] for g in p.ghosts])
        if k == 1:
            xo, xg = xo[:, 0], xg[:, 0]
        got = op.mult(torch.from_numpy(np.ascontiguousarray(xo)).cuda(),
                      ghosts=torch.from_numpy(np.ascontiguousarray(xg)).cuda()).cpu().numpy()
        want = y[so[parts[r][0]]:so[parts[r][1]]]
        if k == 1:
            want = want[:, 0]
        assert np.abs(got - want).max() <= 1e-12 * np.abs(y).max()

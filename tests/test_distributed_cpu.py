"""Host logic of the multi-GPU KPM sharding, run as two gloo ranks on CPU:
the column / Hamiltonian splits and the moment all-reduce must reproduce the
single-process result exactly.  The per-rank moment computation is the CPU
oracle here (no GPU), injected through moment_fn."""
import os
import socket

import numpy as np
import pytest

from vbcsr_b200 import distributed as D
from vbcsr_b200 import workloads as W


def test_column_shard_covers_and_balances():
    for total in (1, 7, 64, 100):
        for world in (1, 2, 3, 8):
            parts = [D.column_shard(total, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == total
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def test_rademacher_columns_split_invariant():
    full = D.rademacher_columns(50, 0, 10, seed=3)
    left = D.rademacher_columns(50, 0, 4, seed=3)
    right = D.rademacher_columns(50, 4, 10, seed=3)
    assert np.array_equal(full, np.hstack([left, right]))
    assert set(np.unique(full)) <= {-1.0, 1.0}


def test_hamiltonian_shard_lpt():
    costs = [10, 3, 7, 7, 1, 5]
    parts = D.hamiltonian_shard(costs, 2)
    assert sorted(i for p in parts for i in p) == list(range(6))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= max(costs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from oracle.oracle import Restated

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        orc = Restated()
        H, _ = W.tmd_lattice(4, seed=2)
        mu = D.kpm_moments_sharded(H, 24, 6, seed=11, moment_fn=lambda h, v, m: orc.kpm_moments(h, v, m, True))
        Hs = [W.tmd_lattice(L, seed=L)[0] for L in (2, 4, 3, 5)]
        mub = D.batched_kpm_moments_sharded(Hs, 16, 3, seed=5,
                                            moment_fn=lambda h, v, m: orc.kpm_moments(h, v, m, True))
        np.save(os.path.join(out_dir, f"mu_{rank}.npy"), mu)
        np.save(os.path.join(out_dir, f"mub_{rank}.npy"), mub)
    finally:
        dist.destroy_process_group()


def test_sharded_moments_two_ranks(tmp_path):
    import torch.multiprocessing as mp

    from oracle.oracle import Restated

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    orc = Restated()
    H, _ = W.tmd_lattice(4, seed=2)
    ref = orc.kpm_moments(H, D.rademacher_columns(H.N, 0, 6, 11), 24, True)
    Hs = [W.tmd_lattice(L, seed=L)[0] for L in (2, 4, 3, 5)]
    refb = np.stack([orc.kpm_moments(h, D.rademacher_columns(h.N, 0, 3, 5 + i), 16, True) for i, h in enumerate(Hs)])
    for r in range(2):
        mu = np.load(tmp_path / f"mu_{r}.npy")
        mub = np.load(tmp_path / f"mub_{r}.npy")
        assert np.abs(mu - ref).max() <= 1e-12 * abs(ref[0])
        assert np.abs(mub - refb).max() <= 1e-12 * np.abs(refb[:, 0]).max()

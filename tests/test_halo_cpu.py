"""Row-partitioned apply, host side: the halo plan (ghost numbering by owner
rank then global id, pack lists, counts), the plan built by exchanging
requests over gloo ranks against the plan read off the whole matrix, and the
ghost exchange itself (all_to_all_single into the ghost rows), real and
complex.  The local products are checked with the oracle (the checker)."""
import os
import socket

import numpy as np
import pytest

from vbcsr_b200 import distributed as D
from vbcsr_b200 import workloads as W


def _matrices():
    H, _ = W.tmd_lattice(6, seed=3)
    yield "tmd", H
    yield "random", W.random_pattern(90, 2, 7, 6, seed=4)
    yield "complex", W.random_pattern(60, 1, 5, 5, seed=5, dtype=np.complex128)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_plan_consistency(world):
    for _, H in _matrices():
        parts = D.row_partition(H, world)
        assert parts[0][0] == 0 and parts[-1][1] == H.n
        assert all(parts[k][1] == parts[k + 1][0] for k in range(world - 1))
        plans = [D.halo_plan_from_global(H, parts, r) for r in range(world)]
        so = H.scalar_offsets()
        gx = np.arange(H.N, dtype=np.float64)  # x = its own global scalar index
        for r, p in enumerate(plans):
            # ghosts ascending = (owner, gid) order; none owned by r
            assert np.all(np.diff(p.ghosts) > 0)
            own = D._owner(p.displs, p.ghosts)
            assert not np.any(own == r)
            assert np.array_equal(p.block_sizes[p.n_owned:], H.block_sizes[p.ghosts])
            # local columns ascend within every row (the library's slot order)
            for i in range(p.n_owned):
                assert np.all(np.diff(p.col_ind[p.row_ptr[i]:p.row_ptr[i + 1]]) > 0)
            # what r receives from q is what q packs for r, in r's ghost order
            for q in range(world):
                assert p.recv_counts[q] == plans[q].send_counts[r]
            xo = [gx[so[pl.displs[q]]:so[pl.displs[q + 1]]] for q, pl in enumerate(plans)]
            recv = []
            for q, pl in enumerate(plans):
                c = np.concatenate([[0], np.cumsum(pl.send_counts)])
                recv.append(xo[q][pl.send_rows[c[r]:c[r + 1]]])
            want = np.concatenate([gx[so[g]:so[g + 1]] for g in p.ghosts]) if len(p.ghosts) else np.zeros(0)
            assert np.array_equal(np.concatenate(recv) if recv else np.zeros(0), want)


@pytest.mark.parametrize("world", [2, 3])
def test_local_products_match_global(oracle, world):
    for _, H in _matrices():
        parts = D.row_partition(H, world)
        rng = np.random.default_rng(world)
        x = rng.normal(size=(H.N, 3))
        if np.iscomplexobj(H.values):
            x = x + 1j * rng.normal(size=x.shape)
        y = oracle.apply(H, x)
        so = H.scalar_offsets()
        for r in range(world):
            p = D.halo_plan_from_global(H, parts, r)
            loc = D.local_rows(H, *parts[r])
            L = p.local_matrix(loc.values)
            xl = np.concatenate([x[so[parts[r][0]]:so[parts[r][1]]]] + [x[so[g]:so[g + 1]] for g in p.ghosts])
            yl = oracle.apply(L, xl)[:p.N_owned]
            assert np.abs(yl - y[so[parts[r][0]]:so[parts[r][1]]]).max() <= 1e-12 * np.abs(y).max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = []
        for name, H in _matrices():
            parts = D.row_partition(H, world)
            loc = D.local_rows(H, *parts[rank])
            p = D.halo_plan(loc)
            ok_plan = p.same_as(D.halo_plan_from_global(H, parts, rank))
            so = H.scalar_offsets()
            rng = np.random.default_rng(7)
            gx = rng.normal(size=(H.N, 2))
            if np.iscomplexobj(H.values):
                gx = gx + 1j * rng.normal(size=gx.shape)
            xl = torch.zeros((p.N_local, 2), dtype=torch.from_numpy(gx).dtype)
            xl[:p.N_owned] = torch.from_numpy(gx[so[parts[rank][0]]:so[parts[rank][1]]])
            D.exchange_ghosts(xl, p)
            want = np.concatenate([gx[so[g]:so[g + 1]] for g in p.ghosts]) if len(p.ghosts) else np.zeros((0, 2))
            ok_x = np.array_equal(xl[p.N_owned:].numpy(), want)
            res.append(f"{name}:{int(ok_plan)}{int(ok_x)}")
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(" ".join(res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_gloo(tmp_path, world):
    import torch.multiprocessing as mp

    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    for r in range(world):
        txt = (tmp_path / f"rank{r}.txt").read_text()
        assert txt == "tmd:11 random:11 complex:11", (r, txt)

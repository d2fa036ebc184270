"""The host side of the z-slab decomposition (zebraflow_b200/slabs.py), on CPU:
the slabs' interiors tile the lattice, their halo planes are the neighbours'
planes (z periodic), and the ring exchange between two gloo ranks delivers
each face's buffer to the neighbour that pulls from it."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from zebraflow_b200 import slabs


def test_slab_interiors_tile_the_lattice_and_halos_match():
    rng = np.random.default_rng(0)
    nx, ny, nz, world = 5, 6, 48, 3
    b = rng.integers(-1, 3, size=(nx, ny, nz)).astype(np.int32)
    covered = np.zeros(nz, int)
    for r in range(world):
        z0, z1 = slabs.slab_bounds(nz, world, r)
        covered[z0:z1] += 1
        s = slabs.slab_lattice(b, world, r)
        assert s.shape == (nx, ny, z1 - z0 + 2 * slabs.HALO)
        assert np.array_equal(s[:, :, slabs.HALO:-slabs.HALO], b[:, :, z0:z1])
        below = slabs.slab_lattice(b, world, (r - 1) % world)
        above = slabs.slab_lattice(b, world, (r + 1) % world)
        # my bottom halo planes are the last interior planes of the rank below, and so on
        assert np.array_equal(s[:, :, :slabs.HALO], below[:, :, -2 * slabs.HALO:-slabs.HALO])
        assert np.array_equal(s[:, :, -slabs.HALO:], above[:, :, slabs.HALO:2 * slabs.HALO])
    assert np.all(covered == 1)
    with pytest.raises(ValueError):
        slabs.slab_bounds(50, 3, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    n = 7
    send_dn = torch.full((5 * n,), 100 * rank + 1, dtype=torch.int32)
    send_up = torch.full((5 * n,), 100 * rank + 2, dtype=torch.int32)
    recv_dn = torch.zeros(5 * n, dtype=torch.int32)
    recv_up = torch.zeros(5 * n, dtype=torch.int32)
    slabs.exchange_dist(send_dn, send_up, recv_dn, recv_up, rank, world)
    out[rank] = (int(recv_dn[0]), int(recv_dn[-1]), int(recv_up[0]), int(recv_up[-1]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ring_exchange_between_gloo_ranks(world):
    with mp.get_context("spawn").Manager() as m:  # a forked manager could inherit held locks
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        below, above = (r - 1) % world, (r + 1) % world
        # the bottom halo gets the rank below's last interior plane (its send_up), the top
        # halo the rank above's first interior plane (its send_dn)
        assert res[r] == (100 * below + 2, 100 * below + 2, 100 * above + 1, 100 * above + 1)


# the populations that cross a z face: e_z = +1 (pulled up into the plane
# above) and e_z = -1, in the reference's direction order
_ZUP, _ZDN = [4, 10, 12, 14, 16], [5, 11, 13, 15, 17]


def _slab_rank(rank, world, port, b, steps, out):
    """One rank of a real slab run: the FP64 oracle steps the rank's slab (its
    interior planes with HALO planes either side, z not periodic); after every
    step the rank sends the e_z = -1 populations of its first interior plane
    down and the e_z = +1 populations of its last interior plane up, and puts
    what it receives into its halo planes, as zebraflow_b200/slabs.py does."""
    import torch.distributed as dist
    from oracle.bind import OracleLBM
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    lbm = OracleLBM(slabs.slab_lattice(b, world, rank), wall_mode=0, periodic=(0, 0, 0), tau=0.8,
                    g=(0.0, 0.0, 2e-5), precision="f64")
    dom, _ = lbm.dom()
    nzs = slabs.slab_lattice(b, world, rank).shape[2]
    kb, kt = slabs.HALO, nzs - slabs.HALO - 1

    def plane(k):  # listed points of local plane k in (x, y) order
        idx = np.nonzero(dom[:, 2] == k)[0]
        return idx[np.lexsort((dom[idx, 1], dom[idx, 0]))]

    p_kb, p_kt, p_hb, p_ht = plane(kb), plane(kt), plane(kb - 1), plane(kt + 1)
    for _ in range(steps):
        lbm.step()
        f = lbm.get_f()
        send_dn = torch.from_numpy(np.ascontiguousarray(f[_ZDN][:, p_kb]))
        send_up = torch.from_numpy(np.ascontiguousarray(f[_ZUP][:, p_kt]))
        recv_dn, recv_up = torch.empty_like(send_up), torch.empty_like(send_dn)
        slabs.exchange_dist(send_dn, send_up, recv_dn, recv_up, rank, world)
        f[np.ix_(_ZUP, p_hb)] = recv_dn.numpy()  # from the rank below: its last interior plane
        f[np.ix_(_ZDN, p_ht)] = recv_up.numpy()  # from the rank above: its first interior plane
        lbm.set_f(f)
    z0, _ = slabs.slab_bounds(b.shape[2], world, rank)
    f = lbm.get_f()
    inner = (dom[:, 2] >= slabs.HALO) & (dom[:, 2] < nzs - slabs.HALO)
    glob = dom[inner].copy()
    glob[:, 2] += z0 - slabs.HALO
    out[rank] = (glob, f[:, inner])
    lbm.close()
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_step_the_split_lattice_exactly():
    """Two gloo ranks step the two z slabs of a periodic tube with the FP64
    oracle and exchange their faces after every step; after 30 steps every
    interior point holds the unsplit lattice's populations bit for bit."""
    from oracle.bind import OracleLBM
    import zebraflow_b200 as zf
    nx, ny, nz, world, steps = 12, 12, 32, 2, 30
    b = zf.gen_tube(nx, ny, nz, 5.5, 5.5, 4.5, True)
    ref = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.8, g=(0.0, 0.0, 2e-5), precision="f64")
    for _ in range(steps):
        ref.step()
    rdom, _ = ref.dom()
    rf = ref.get_f()
    ref.close()
    where = {tuple(p): i for i, p in enumerate(rdom)}
    with mp.get_context("spawn").Manager() as m:  # a forked manager could inherit held locks
        out = m.dict()
        mp.spawn(_slab_rank, args=(world, _free_port(), b, steps, out), nprocs=world, join=True)
        res = dict(out)
    seen = 0
    for r in range(world):
        glob, f = res[r]
        idx = np.array([where[tuple(p)] for p in glob])
        assert np.array_equal(f, rf[:, idx]), r
        seen += len(idx)
    assert seen == rf.shape[1]  # the interiors cover the lattice
    assert np.abs(rf - rf.mean(axis=1, keepdims=True)).max() > 0  # the flow is not trivial

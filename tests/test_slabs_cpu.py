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
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        below, above = (r - 1) % world, (r + 1) % world
        # the bottom halo gets the rank below's last interior plane (its send_up), the top
        # halo the rank above's first interior plane (its send_dn)
        assert res[r] == (100 * below + 2, 100 * below + 2, 100 * above + 1, 100 * above + 1)

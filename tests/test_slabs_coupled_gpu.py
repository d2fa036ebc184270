"""The coupled step split over z slabs (zebraflow_b200/slabs.py SlabCoupled,
zf_set_ib_slab, zf_cells_reduce_buffer) on one GPU: a periodic tube cut into
two slabs, each with IB_HALO planes of halo, all cells held by both, stepped
side by side (coupled_step_local: the halo exchange and the sum of the slabs'
partial node and repulsion velocities in place of the collectives).  Two slabs
of one process stand for two ranks; no kernel waits on another.

The split run must give the unsplit zf_step's cell positions and interior
populations.  The summation order of the velocities (per slab, then summed) and
of the spreading atomics differs, so the check is against the spread between
two unsplit runs, which differ by the same kind of rounding."""
import numpy as np
import pytest
import torch

import zebraflow_b200 as zf
from zebraflow_b200 import slabs

pytestmark = pytest.mark.gpu

NX, NY, NZ, R = 40, 40, 64, 16.0
CX = CY = 19.5
STAGGER, NSTEPS = 10, 100


def setup():
    b = zf.gen_tube(NX, NY, NZ, CX, CY, R, True)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest = xyz * np.array([3.5, 2.25, 1.0])
    rest_n = xyzn * np.array([1.25, 0.9, 0.6])
    mesh = (rest, tri, rest_n, zf.mesh_edges(trin))
    x, xn = zf.gen_cells(b, 6, rest, rest_n, (3.5, 2.25, 1.0), seed=11, margin=0.3)
    wall = zf.gen_wall_tube(CX, CY, R, NZ)
    kw = dict(tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB, g=(0.0, 0.0, 2e-5),
              storage=zf.STORE_F32, stagger=STAGGER, area0=0.0, volume0=0.0, origin=(0.0, 0.0, 0.0))
    return b, mesh, (x, xn), wall, kw


def unsplit(b, mesh, cells, wall, kw):
    ctx = zf.Context(zf.default_params(nx=NX, ny=NY, nz=NZ, periodic=(0, 0, 1), **kw))
    ctx.set_lattice(b)
    ctx.set_wall(*wall)
    ctx.set_mesh(*mesh)
    ctx.set_cells(*cells)
    ctx.step(NSTEPS)
    out = ctx.download_populations(), ctx.cells()[0], ctx.domlist()
    ctx.close()
    return out


def test_two_slabs_match_the_whole_coupled_step():
    b, mesh, cells, wall, kw = setup()
    x0 = cells[0]
    zc = x0[2].mean(axis=1)
    lz = NZ * 0.5
    # cells across the slabs' faces (z = 0 and z = 16 um) are the point of the test
    ext = np.abs(x0[2] - zc[:, None]).max()
    assert any(abs(((z - f + lz / 2) % lz) - lz / 2) < ext for z in zc for f in (0.0, lz / 2))
    f1, xa, dom = unsplit(b, mesh, cells, wall, kw)
    f2, xb, _ = unsplit(b, mesh, cells, wall, kw)
    index = {tuple(p): l for l, p in enumerate(dom.tolist())}

    stream = torch.cuda.Stream()
    parts = [slabs.SlabCoupled(b, wall, mesh, cells, world=2, rank=r, stream=stream, **kw) for r in range(2)]
    slabs.coupled_step_local(parts, NSTEPS)
    torch.cuda.synchronize()
    xs = [s.ctx.cells()[0] for s in parts]
    assert np.array_equal(xs[0], xs[1])  # every slab moves all cells the same way
    moved = np.abs(xa - x0).max()
    dx_runs = np.abs(xb - xa).max()
    dx_split = np.abs(xs[0] - xa).max()
    df_runs = np.abs(f2 - f1).max()
    df_split = 0.0
    for s in parts:
        sdom = s.ctx.domlist()
        inner, gz = s.interior(sdom)
        gl = np.array([index[(i, j, k % NZ)] for (i, j), k in zip(sdom[inner, :2].tolist(), gz[inner].tolist())])
        fs = s.ctx.download_populations()[:, inner]
        df_split = max(df_split, np.abs(fs - f1[:, gl]).max())
        s.close()
    print(f"moved {moved:.3e} um; positions: split {dx_split:.3e}, between runs {dx_runs:.3e}; "
          f"populations: split {df_split:.3e}, between runs {df_runs:.3e}")
    assert moved > 1e-3
    assert dx_split <= max(10 * dx_runs, 1e-9 * moved)
    assert df_split <= max(10 * df_runs, 1e-7)


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    b, mesh, cells, wall, kw = setup()
    s = slabs.SlabCoupled(b, wall, mesh, cells, world=world, rank=rank, device=0, **kw)
    s.step(NSTEPS)
    torch.cuda.synchronize()
    sdom = s.ctx.domlist()
    inner, gz = s.interior(sdom)
    np.savez(f"{out_dir}/rank{rank}.npz", x=s.ctx.cells()[0], ij=sdom[inner, :2], gz=gz[inner],
             f=s.ctx.download_populations()[:, inner])
    s.close()
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_the_whole_coupled_step(tmp_path):
    """SlabCoupled.step itself at world 2: two processes, one slab each, on the
    one GPU, with the halo ring and the velocities' all-reduce through
    torch.distributed (gloo, staged through host memory; no kernel waits on
    another rank's)."""
    import torch.multiprocessing as mp
    mp.start_processes(_gloo_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    b, mesh, cells, wall, kw = setup()
    f1, xa, dom = unsplit(b, mesh, cells, wall, kw)
    f2, xb, _ = unsplit(b, mesh, cells, wall, kw)
    index = {tuple(p): l for l, p in enumerate(dom.tolist())}
    r = [np.load(tmp_path / f"rank{k}.npz") for k in range(2)]
    assert np.array_equal(r[0]["x"], r[1]["x"])
    dx_runs = np.abs(xb - xa).max()
    dx_split = np.abs(r[0]["x"] - xa).max()
    df_runs = np.abs(f2 - f1).max()
    df_split = 0.0
    for q in r:
        gl = np.array([index[(i, j, k % NZ)] for (i, j), k in zip(q["ij"].tolist(), q["gz"].tolist())])
        df_split = max(df_split, np.abs(q["f"] - f1[:, gl]).max())
    print(f"positions: split {dx_split:.3e}, between runs {dx_runs:.3e}; "
          f"populations: split {df_split:.3e}, between runs {df_runs:.3e}")
    assert np.abs(xa - cells[0]).max() > 1e-3
    assert dx_split <= max(10 * dx_runs, 1e-9)
    assert df_split <= max(10 * df_runs, 1e-7)

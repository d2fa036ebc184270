"""A parent segment feeding the region (zebraflow_b200/inflow.py over two
contexts on the GPU): a periodic tube segment [0, 24) um whose one parent
cell straddles the exit plane, and a periodic region tube downstream with
free slots.  The parent is folded back into its segment and cloned into the
region's first free slot, whole across the exit plane; while slaved, the
clone's nodes behind the plane move exactly as the parent's do."""
import numpy as np
import pytest

import zebraflow_b200 as zf
from zebraflow_b200 import inflow

pytestmark = pytest.mark.gpu

NX, NY, NZ, R = 40, 40, 48, 16.0
CX = CY = 19.5
DX = 0.5
STAGGER = 10


def contexts():
    b = zf.gen_tube(NX, NY, NZ, CX, CY, R, True)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest = xyz * np.array([3.5, 2.25, 1.0])
    rest_n = xyzn * np.array([1.25, 0.9, 0.6])
    mesh = (rest, tri, rest_n, zf.mesh_edges(trin))
    kw = dict(nx=NX, ny=NY, nz=NZ, tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB, periodic=(0, 0, 1),
              g=(0.0, 0.0, 1e-4), storage=zf.STORE_F32, stagger=STAGGER, dx=DX, area0=0.0, volume0=0.0)
    lz = NZ * DX
    # the parent segment [0, lz) with one parent 0.3 um before its exit plane
    P = zf.Context(zf.default_params(origin=(0.0, 0.0, 0.0), **kw))
    P.set_lattice(b)
    P.set_wall(*zf.gen_wall_tube(CX, CY, R, NZ, dx=DX))
    P.set_mesh(*mesh)
    c = np.array([CX * DX, CY * DX, lz - 0.3])
    P.set_cells((rest + c).T[:, None, :], (rest_n + c).T[:, None, :])
    # the region downstream, [lz - 4, 2 lz - 4): one active cell, three free slots
    Rg = zf.Context(zf.default_params(origin=(0.0, 0.0, lz - 4.0), **kw))
    Rg.set_lattice(b)
    Rg.set_wall(*zf.gen_wall_tube(CX, CY, R, NZ, origin=(0.0, 0.0, lz - 4.0), dx=DX))
    Rg.set_mesh(*mesh)
    far = np.array([CX * DX, CY * DX, lz + 12.0])
    x = np.full((3, 4, rest.shape[0]), -5000.0)
    xn = np.full((3, 4, rest_n.shape[0]), -5000.0)
    x[:, 0] = (rest + far).T
    xn[:, 0] = (rest_n + far).T
    Rg.set_cells(x, xn)
    seg = inflow.Segment(0.0, lz, 1, DX)
    fl = inflow.Inflow(P, Rg, seg, free=[False, True, True, True], dt_stagger=P.params.dt * STAGGER)
    return P, Rg, fl, lz


def test_parent_is_cloned_whole_and_the_clone_follows_it():
    P, Rg, fl, lz = contexts()
    xp0 = P.cells()[0]
    fl.step(STAGGER)  # the first membrane iteration: the parent crosses its exit plane
    assert fl.clones == 1
    assert fl.status_r.tolist() == [1, -1, -5000, -5000] and fl.status_p.tolist() == [4]
    xp1 = P.cells()[0]
    xr1, _, st = Rg.cells()
    assert st.tolist() == [1, 1, -5000, -5000]  # the clone is an active cell on the GPU
    assert 0.0 <= xp1[2].min() and xp1[2].max() < lz  # folded into the segment
    clone = xr1[:, 1]
    assert clone[2].max() - clone[2].min() < 3.0  # whole: no node left one period behind
    # the clone is the parent, made contiguous across the plane
    unfold = np.where(xp1[2, 0] < 0.5 * lz, xp1[2, 0] + lz, xp1[2, 0])
    assert np.allclose(clone[2], unfold) and np.allclose(clone[:2], xp1[:2, 0])
    assert np.abs(xp1[2] - xp0[2]).max() > 0.0

    fl.step(STAGGER)  # slaved: nodes not yet 5 DX past the plane move with the parent's nodes
    xp2 = P.cells()[0]
    xr2 = Rg.cells()[0]
    behind = clone[2] <= lz + 5 * DX
    assert behind.sum() > 100
    dp = xp2[:, 0] - xp1[:, 0]
    dp[2] = (dp[2] + 0.5 * lz) % lz - 0.5 * lz  # modulo the fold
    dr = xr2[:, 1] - clone
    np.testing.assert_allclose(dr[:, behind], dp[:, behind], rtol=0, atol=1e-9)
    assert np.isfinite(xr2[:, :2]).all()
    P.close()
    Rg.close()

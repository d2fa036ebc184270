"""The GPU coupled step against the oracle on a bifurcation at the scale of the
benchmark's cell interactions: a periodic Y-bifurcation of 128x128x256
lattice points (parent radius 18, daughters 13, half-angle 20 degrees,
269,356 fluid points), halfway bounce-back, tau 0.9, Guo force 2e-6 along the
parent axis, 152 nucleated RBCs placed from seed 2024 (icosphere 642/1280
scaled to 7, 4.5, 2 lattice units, nucleus 162 nodes scaled to 2.5, 1.8,
1.2), the vessel's marching-tetrahedra wall mesh, membrane/IB block every 50
iterations, from rest.  After 50, 100 and 200 iterations the fluid velocity,
the wall shear stress and the node displacement are compared (relative L2).

 * fp32-deviation storage against the FP64 oracle storing the same fp32
   deviations: both resolve the slow start-up flow, so they agree to fp32
   arithmetic after the first membrane block, and the difference grows as
   the cells interact (the repulsions switch on at distance cut-offs and the
   float atomics of the spreading sum in no fixed order);
 * plain fp32 populations, GPU against the fp32 oracle: the stored f ~ 0.05
   has an ulp of 3.7e-9 while the start-up velocity is ~1e-4, so two fp32
   implementations that round in different places already differ by ~1e-3
   before the cells have moved; this is the floor of every plain-fp32
   comparison of this workload.
The bounds are written per checkpoint.
"""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleCells, OracleLBM, OracleWorld

pytestmark = pytest.mark.gpu

DIMS, RP, RD, ANGLE, G = (128, 128, 256), 18.0, 13.0, 20.0, 2e-6
N_CELLS, SEED = 160, 2024
CHECKS = (50, 100, 200)
# relative L2 bounds per checkpoint: u, WSS, displacement.  Measured on a
# B200: fp32 deviations against FP64, 8.0e-7 / 7.0e-7 / 1.9e-6 after the
# first membrane block (iteration 50), 6.5e-5 / 6.3e-5 / 9.3e-5 at 100 and
# 2.4e-3 / 2.4e-3 / 1.6e-3 at 200; plain fp32 against the fp32 oracle
# 2.7e-3 / 2.8e-3 / 2.6e-3, 2.9e-4 / 4.2e-4 / 5.1e-4 and 2.7e-3 / 3.0e-3 /
# 1.6e-3.  The bounds are twice the measured values after the first block,
# where the two sides differ only in rounding, and three times them later,
# where the amplification of those differences varies from run to run.
BOUNDS_DEV = {50: (2e-6, 2e-6, 4e-6), 100: (2e-4, 2e-4, 3e-4), 200: (7e-3, 7e-3, 5e-3)}
BOUNDS_F32 = {50: (6e-3, 6e-3, 6e-3), 100: (1e-3, 1.3e-3, 1.5e-3), 200: (8e-3, 9e-3, 5e-3)}


def rel(a, b):
    ok = np.isfinite(a) & np.isfinite(b)
    return float(np.linalg.norm((a - b)[ok]) / np.linalg.norm(b[ok]))


def node_normals(wall):
    xyz, tri1, nrm = wall
    t = tri1 - 1
    p = xyz.T.astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(p[t[1]] - p[t[0]], p[t[2]] - p[t[0]]), axis=1)
    acc = np.zeros((xyz.shape[1], 3))
    for v in range(3):
        np.add.at(acc, t[v], area[:, None] * nrm.T)
    acc /= np.linalg.norm(acc, axis=1, keepdims=True)
    return np.ascontiguousarray(acc.T, np.float32)


@pytest.fixture(scope="module")
def scene():
    nx, ny, nz = DIMS
    b, _ = zf.gen_bifurcation(nx, ny, nz, RP, RD, ANGLE)
    wall = zf.gen_wall_bifurcation(nx, ny, nz, RP, RD, ANGLE, dx=0.5)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest, rest_n = xyz * np.array([3.5, 2.25, 1.0]), xyzn * np.array([1.25, 0.9, 0.6])
    mesh = (rest, tri, rest_n, zf.mesh_edges(trin))
    cells = zf.gen_cells(b, N_CELLS, rest, rest_n, (3.5, 2.25, 1.0), seed=SEED, dx=0.5, margin=0.4)
    assert cells[0].shape[1] >= 150
    return b, wall, mesh, cells


def compare(scene, storage, precision, emulation, bounds):
    b, wall, mesh, cells = scene
    nx, ny, nz = DIMS
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                          periodic=(0, 0, 1), g=(0.0, 0.0, G), origin=(0.0, 0.0, 0.0), dx=0.5,
                          area0=0.0, volume0=0.0, storage=storage)
    nrm = node_normals(wall)
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.9, g=(0.0, 0.0, G), precision=precision)
    if emulation:
        lbm.set_storage_emulation(emulation, 1.0, 1.0)
    oc = OracleCells(*mesh, p, precision=precision)
    oc.set_cells(*cells)
    w = OracleWorld(lbm, oc, p)
    w.set_wall(*wall)
    dom = np.argwhere(b >= 0)
    fl = b[dom[:, 0], dom[:, 1], dom[:, 2]] > 0
    x0 = cells[0]
    errs = {}
    with zf.Context(p) as ctx:
        ctx.set_lattice(b)
        ctx.set_wall(*wall)
        ctx.set_mesh(*mesh)
        ctx.set_cells(*cells)
        done = 0
        for it in CHECKS:
            ctx.step(it - done)
            w.step(it - done)
            done = it
            wss_g, _, _ = ctx.wss(nrm)  # leaves the moments of the current populations
            Dg, Ug, Vg, Wg = ctx.download_moments()
            xg, _, sg = ctx.cells()
            D, U, V, W = lbm.moments()
            wss_o, _, _ = w.wss(nrm)
            go = oc.get()
            assert np.array_equal(sg, go["status"])
            live = go["status"] > 0
            err = (rel(np.stack([Ug, Vg, Wg])[:, fl], np.stack([U, V, W])[:, fl]),
                   rel(wss_g, wss_o),
                   rel((xg - x0)[:, live], (go["x"] - x0)[:, live]))
            errs[it] = err
            print(f"storage {storage} vs {precision} oracle, iteration {it}: u {err[0]:.2e}  WSS {err[1]:.2e}  "
                  f"disp {err[2]:.2e}")
    for o in (w, oc, lbm):
        o.close()
    for it, err in errs.items():
        for e, bound in zip(err, bounds[it]):
            assert e <= bound, (it, err)
    return errs


def test_fp32_deviation_storage_against_fp64_oracle(scene):
    # oracle storage emulation 2: populations kept as fp32 deviations f/w - 1
    compare(scene, zf.STORE_F32_DEV, "f64", 2, BOUNDS_DEV)


def test_plain_fp32_against_fp32_oracle(scene):
    compare(scene, zf.STORE_F32, "f32", 0, BOUNDS_F32)

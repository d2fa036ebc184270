"""GPU parity of the membrane set-up (zebraflow_b200/csrc/zf_mesh.cpp) and of
k_membrane (zebraflow_b200/csrc/zf_cells.cu) against the CPU oracle
(oracle/orc_cells.inc) through the C ABI.

Tolerances: topology is exact; calibrated parameters agree to 1e-5 relative
(both compute in fp32 from the same rest shape, with different grouping);
triangle geometry to 2e-5; node forces are sums of ~20 terms that cancel to a
few percent of the largest term, so they are compared with an absolute bound
of 1e-4 x the largest force of the cell set.
"""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleCells
from test_oracle_cells import deformed_cells, ellipsoid_meshes

pytestmark = pytest.mark.gpu


def make(rest, tri, rest_n, en, nx=16):
    p = zf.default_params(nx=nx, ny=nx, nz=nx, tau=0.9, tau_from_phase=0, area0=0.0,
                          volume0=0.0, wall_mode=zf.WALL_HALFWAY_BB)
    ctx = zf.Context(p)
    ctx.set_mesh(rest, tri, rest_n, en)
    return ctx, p


def test_mesh_topology_and_calibration_match_oracle():
    rest, tri, rest_n, en = ellipsoid_meshes()
    ctx, p = make(rest, tri, rest_n, en)
    o = OracleCells(rest, tri, rest_n, en, p, precision="f32")
    E, ep, epn, ae, av = o.topology()
    Eg, first = ctx.edges()
    assert np.array_equal(Eg, E)
    # first-visitor flags: the first edge (in order) naming a triangle does its terms
    seen = set()
    for e in range(o.ne):
        t1, t2 = E[e, 4], E[e, 5]
        assert bool(first[e] & 1) == (t1 not in seen)
        seen.add(t1)
        assert bool(first[e] & 2) == (t2 not in seen)
        seen.add(t2)
    epg, epng, aeg = ctx.edge_params()
    for r in (0, 1, 2, 4):  # LMAX, Plength, kp, cos(theta0)
        assert np.allclose(epg[r], ep[r], rtol=1e-5, atol=0)
    assert np.allclose(epng, epn, rtol=1e-5, atol=0)
    # sin(theta0) = +-sqrt(1 - cos^2) is fp32 rounding noise on nearly flat edges
    assert np.max(np.abs(epg[3] - ep[3])) < 3.5e-4
    assert np.allclose(aeg, ae, rtol=1e-6)
    assert abs(ctx.area0 - av[0]) < 1e-6 * av[0] and abs(ctx.volume0 - av[1]) < 1e-6 * av[1]
    ctx.close()


def test_membrane_forces_match_reference_output():
    """k_membrane against the reference's own membrane step:
    tests/golden/ref_cells.npz holds the node forces, triangle geometry,
    per-cell terms, screening counts and removals that the reference's force
    blocks of its main() (ZebraflowWT.c:5706-7535) computed for four deformed
    RBCs with nuclei built from the shipped meshes (the third with one screened
    force component, the fourth removed; fixture script:
    tests/golden/make_ref_golden.py).  Default parameters are the reference's
    constants (moduli, RBC_SURF, MCV).  Bounds as for the oracle comparison:
    node forces within 1e-4 of the largest force, geometry 2e-5; statuses exact."""
    import os
    here = os.path.join(os.path.dirname(__file__), "golden")
    G = np.load(os.path.join(here, "ref_setup.npz"))
    C = np.load(os.path.join(here, "ref_cells.npz"))
    p = zf.default_params(nx=16, ny=16, nz=16, tau=0.9, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB)
    ctx = zf.Context(p)
    ctx.set_mesh(G["mesh_x"], G["mesh_tri"], G["nuc_x"], G["nuc_edges"])
    ctx.set_cells(C["x"], C["xn"])
    ctx.cgsm_forces()
    _, _, status = ctx.cells()
    assert np.array_equal(status, C["status"][:, 0])
    f, fn = ctx.cell_forces()
    assert np.max(np.abs(f - C["ftot"])) < 1e-4 * np.abs(C["ftot"]).max()
    assert np.max(np.abs(fn - C["ftot_n"])) < 1e-4 * np.abs(C["ftot_n"]).max()
    ta, tn, tc, nrm, cf = ctx.cell_geometry()
    live = C["status"][:, 0] == 1
    assert np.allclose(ta[live], C["tri_area"][live], rtol=2e-5)
    assert np.max(np.abs(tn[:, live] - C["tri_normal"][:, live])) < 2e-5
    assert np.max(np.abs(tc[:, live] - C["tri_centroid"][:, live])) < 2e-5 * np.abs(C["tri_centroid"]).max()
    assert np.max(np.abs(nrm[:, live] - C["node_normal"][:, live])) < 2e-5
    assert np.allclose(cf[live, :2], C["cell"][live, :2], rtol=2e-5)      # area, volume
    assert np.allclose(cf[live, 2:5], C["cell"][live, 2:5], rtol=2e-6)    # centroid
    assert np.allclose(cf[live, 5:7], C["cell"][live, 5:7], rtol=2e-3, atol=1e-9)
    ctx.close()


def test_membrane_forces_match_oracle():
    rest, tri, rest_n, en = ellipsoid_meshes()
    ctx, p = make(rest, tri, rest_n, en)
    o = OracleCells(rest, tri, rest_n, en, p, precision="f32")
    X, XN = deformed_cells(rest, rest_n, 6, seed=11, amp=0.03, scale=1.05)
    ctx.set_cells(X, XN)
    o.set_cells(X, XN)
    ctx.cgsm_forces()
    o.forces()
    g = o.get()
    f, fn = ctx.cell_forces()
    scale = np.abs(g["ftot"]).max()
    assert scale > 1e-13
    assert np.max(np.abs(f - g["ftot"])) < 1e-4 * scale
    assert np.max(np.abs(fn - g["ftot_n"])) < 1e-4 * np.abs(g["ftot_n"]).max()
    ta, tn, tc, nrm, cf = ctx.cell_geometry()
    ota, otn, otc, onrm = o.geometry()
    assert np.allclose(ta, ota, rtol=2e-5)
    assert np.max(np.abs(tn - otn)) < 2e-5
    assert np.max(np.abs(tc - otc)) < 2e-5 * np.abs(otc).max()
    assert np.max(np.abs(nrm - onrm)) < 2e-5
    ocf = g["cell"]
    assert np.allclose(cf[:, :2], ocf[:, :2], rtol=2e-5)      # area, volume
    assert np.allclose(cf[:, 2:5], ocf[:, 2:5], rtol=2e-6)    # centroid
    assert np.allclose(cf[:, 5:7], ocf[:, 5:7], rtol=2e-3, atol=1e-9)  # F_AREA_GLOBAL, F_VOLUME_SCALAR
    # node velocities and repulsions are reset by the membrane step
    v, vn, w, wn = ctx.cell_kinematics()
    assert not v.any() and not w.any()
    ctx.close()


def test_screening_and_removal_match_oracle():
    """A cell inflated 3x produces terms above 1e-10 N: they are screened
    (ZebraflowWT.c:7083-7345) and the cell is removed after 500 of them
    (ZebraflowWT.c:7473-7501); the mildly deformed cells stay."""
    rest, tri, rest_n, en = ellipsoid_meshes()
    ctx, p = make(rest, tri, rest_n, en)
    o = OracleCells(rest, tri, rest_n, en, p, precision="f32")
    X, XN = deformed_cells(rest, rest_n, 3, seed=2, amp=0.01)
    c = X[:, 2, :].mean(axis=1, keepdims=True)
    X[:, 2, :] = c + 3.0 * (X[:, 2, :] - c)
    ctx.set_cells(X, XN)
    o.set_cells(X, XN)
    ctx.cgsm_forces()
    o.forces()
    g = o.get()
    xg, xng, st = ctx.cells()
    assert np.array_equal(st, g["status"])
    assert st[2] == -5000 and st[0] == 1 and st[1] == 1
    assert np.all(xg[:, 2, :] == -5000.0)
    s = ctx.status()
    assert s.cells_removed == 1 and s.screened_terms > 500
    ctx.close()

"""GPU parity of the IB coupling and cell interactions (zebraflow_b200/csrc/zf_ib.cu,
zf_wall.cpp, zf_ib_host.cpp) against the fp32 CPU oracle (oracle/orc_ib.inc).

One membrane iteration is compared stage by stage from an identical state
(populations copied from the GPU into the oracle), then a short coupled run
through zf_step.  Tolerances: wall indices and the wall-triangle choice are
exact; interpolated node velocities agree to 1e-5 of their largest value
(fp32 weights, fp64 sums in the same order); repulsion increments to 1e-5 of
their largest value (float sums in another order); spread body forces to 1e-4
of their largest value (float atomics); positions to 1e-6 um after one
membrane step and 2e-4 um after the coupled run.
"""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleCells, OracleLBM, OracleWorld

pytestmark = pytest.mark.gpu

NX, NY, NZ, R = 40, 40, 48, 16.0
CX = CY = 19.5


def setup(n_cells=10, seed=7, shift_to_wall=2.5, stagger=50):
    b = zf.gen_tube(NX, NY, NZ, CX, CY, R, True)
    p = zf.default_params(nx=NX, ny=NY, nz=NZ, tau=0.9, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, periodic=(0, 0, 1), g=(0, 0, 2e-5),
                          origin=(0.0, 0.0, 0.0), area0=0.0, volume0=0.0, stagger=stagger)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest = xyz * np.array([3.5, 2.25, 1.0])
    rest_n = xyzn * np.array([1.25, 0.9, 0.6])
    en = zf.mesh_edges(trin)
    x, xn = zf.gen_cells(b, n_cells, rest, rest_n, (3.5, 2.25, 1.0), seed=seed)
    # push cell 0 towards the wall so that the wall repulsion acts
    c0 = x[:, 0, :].mean(axis=1)
    d = c0[:2] - np.array([CX, CY]) * 0.5
    d = d / np.linalg.norm(d)
    x[:2, 0, :] += shift_to_wall * d[:, None]
    xn[:2, 0, :] += shift_to_wall * d[:, None]
    wall = zf.gen_wall_tube(CX, CY, R, NZ)
    return b, p, (rest, tri, rest_n, en), (x, xn), wall


def make_gpu(b, p, mesh, cells, wall):
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    ctx.set_wall(*wall)
    ctx.set_mesh(*mesh)
    ctx.set_cells(*cells)
    return ctx


def make_oracle(b, p, mesh, cells, wall):
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.9, g=tuple(p.g), precision="f32")
    oc = OracleCells(*mesh, p, precision="f32")
    oc.set_cells(*cells)
    w = OracleWorld(lbm, oc, p)
    w.set_wall(*wall)
    return lbm, oc, w


def rel_close(a, b, rel):
    scale = max(np.abs(b).max(), 1e-30)
    return np.max(np.abs(a - b)) <= rel * scale


def test_wall_index_and_void_velocity_match_oracle():
    b, p, mesh, cells, wall = setup()
    ctx = make_gpu(b, p, mesh, cells, wall)
    lbm, oc, w = make_oracle(b, p, mesh, cells, wall)
    wi_g, uv_g = ctx.wall_index()
    wi_o, uv_o = w.wall_index(b.shape)
    assert np.array_equal(wi_g, wi_o)
    assert (wi_g > 0).sum() > 1000
    assert np.max(np.abs(uv_g - uv_o)) <= 1e-9
    # the void velocity points into the lumen where it is non-zero
    i, j = np.meshgrid(np.arange(NX), np.arange(NY), indexing="ij")
    inward = -(i - CX)[:, :, None] * uv_g[0] - (j - CY)[:, :, None] * uv_g[1]
    assert np.all(inward[np.abs(uv_g).sum(axis=0) > 0] > 0)
    ctx.close()


def test_membrane_iteration_stage_by_stage():
    b, p, mesh, cells, wall = setup()
    ctx = make_gpu(b, p, mesh, cells, wall)
    lbm, oc, w = make_oracle(b, p, mesh, cells, wall)
    ctx.lbm_steps(300)                         # develop a flow on the GPU
    lbm.set_f(ctx.download_populations())      # identical fluid state
    dom = np.argwhere(b >= 0)
    fl = b[dom[:, 0], dom[:, 1], dom[:, 2]] > 0

    ctx.cgsm_forces()
    oc.forces()
    ctx.lbm_step(store_moments=True, zero_bodyforce=True)
    lbm.step(rbc_flag=True)
    mg, mo = ctx.download_moments(), lbm.moments()
    for a_, b_ in zip(mg[1:], mo[1:]):
        assert np.max(np.abs(a_[fl] - b_[fl])) < 3e-7

    ctx.ibm_interp()
    w.interp()
    vg, vng, wg, wng = ctx.cell_kinematics()
    vo, vno, wo, wno = w.kinematics()
    assert np.abs(vo).max() > 1e-5
    assert rel_close(vg, vo, 1e-5) and rel_close(vng, vno, 1e-5)
    assert np.abs(wo).max() > 0, "the wall repulsion did not act"
    assert rel_close(wg, wo, 1e-6)

    ctx.nuc_memb_repulsion(rebuild=True)
    w.nuc_memb(rebuild=True)
    _, _, wg, _ = ctx.cell_kinematics()
    _, _, wo, _ = w.kinematics()
    assert rel_close(wg, wo, 1e-5)

    ctx.rbc_rbc_repulsion()
    w.rbc_rbc()
    _, _, wg2, _ = ctx.cell_kinematics()
    _, _, wo2, _ = w.kinematics()
    assert np.abs(wo2 - wo).max() > 0, "the cell-cell repulsion did not act"
    assert rel_close(wg2, wo2, 1e-5)

    ctx.ibm_spread()
    w.spread()
    bfg, bfo = ctx.download_bodyforce(), lbm.get_bodyforce()
    assert np.abs(bfo[:, fl]).max() > 0
    assert rel_close(bfg[:, fl], bfo[:, fl], 1e-4)
    vg, vng, _, _ = ctx.cell_kinematics()
    vo, vno, _, _ = w.kinematics()
    assert rel_close(vg, vo, 1e-5)

    ctx.update_positions()
    w.update()
    xg, xng, sg = ctx.cells()
    go = oc.get()
    assert np.array_equal(sg, go["status"])
    assert np.max(np.abs(xg - go["x"])) < 1e-6
    assert np.max(np.abs(xng - go["xn"])) < 1e-6
    ctx.close()


def test_coupled_steps_match_oracle():
    b, p, mesh, cells, wall = setup(stagger=10)
    ctx = make_gpu(b, p, mesh, cells, wall)
    lbm, oc, w = make_oracle(b, p, mesh, cells, wall)
    ctx.step(60)
    w.step(60)
    assert ctx.iteration() == 60
    xg, xng, sg = ctx.cells()
    go = oc.get()
    assert np.array_equal(sg, go["status"])
    moved = np.abs(xg - cells[0]).max()
    assert moved > 1e-3
    assert np.max(np.abs(xg - go["x"])) < 2e-4
    assert np.max(np.abs(xng - go["xn"])) < 2e-4
    ctx.close()


def test_ib_stages_match_reference_output():
    """The CUDA IB coupling against the reference's own blocks:
    tests/golden/ref_ib.npz holds the state after each stage of one membrane
    iteration run by the reference's forces, IB interpolation with wall
    repulsion, nucleus-membrane and RBC-RBC repulsion, IB spreading and position
    update blocks of its main() (ZebraflowWT.c:5659-12189) on the scene of
    tests/golden/ib_scene.py (fixture script: tests/golden/make_ref_golden.py).
    Bounds as against the oracle: node velocities and repulsions 1e-5 of their
    largest value, spread body force 1e-4, positions 1e-6 um."""
    import os
    from golden import ib_scene as S
    here = os.path.join(os.path.dirname(__file__), "golden")
    G = np.load(os.path.join(here, "ref_setup.npz"))
    R = np.load(os.path.join(here, "ref_ib.npz"))
    b = S.lattice()
    p = zf.default_params(nx=S.NX, ny=S.NY, nz=S.NZ, origin=S.ORIGIN, tau=1.22, tau_from_phase=0,
                          wall_mode=zf.WALL_REF_EQ, periodic=(0, 0, 0), stagger=50)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    ctx.set_wall(*S.wall())
    ctx.set_mesh(G["mesh_x"], G["mesh_tri"], G["nuc_x"], G["nuc_edges"])
    ctx.set_cells(R["x"], R["xn"])
    ctx.upload_populations(S.populations(b).astype(np.float32))  # moments follow

    ctx.cgsm_forces()
    f, fn = ctx.cell_forces()
    assert rel_close(f, R["ftot"], 1e-4) and rel_close(fn, R["ftot_n"], 1e-4)
    ctx.ibm_interp()
    vg, vng, wg, wng = ctx.cell_kinematics()
    assert rel_close(vg, R["vel_interp"], 1e-5) and rel_close(vng, R["vel_n_interp"], 1e-5)
    assert np.abs(R["rep_interp"]).max() > 0
    assert rel_close(wg, R["rep_interp"], 1e-5)
    ctx.nuc_memb_repulsion(rebuild=True)
    ctx.rbc_rbc_repulsion()
    _, _, wg, wng = ctx.cell_kinematics()
    assert rel_close(wg, R["rep_rbc"], 1e-5) and rel_close(wng, R["rep_n_rbc"], 1e-5)
    ctx.ibm_spread()
    bf_ref = np.zeros((3, int(R["n_listed"])), np.float32)
    bf_ref[:, R["bf_idx"]] = R["bf_val"]
    assert rel_close(ctx.download_bodyforce(), bf_ref, 1e-4)
    vg, vng, _, _ = ctx.cell_kinematics()
    assert rel_close(vg, R["vel_spread"], 1e-5) and rel_close(vng, R["vel_n_spread"], 1e-5)
    ctx.update_positions()
    xg, xng, sg = ctx.cells()
    assert np.array_equal(sg, R["status"])
    assert np.max(np.abs(xg - R["x_new"])) < 1e-6 and np.max(np.abs(xng - R["xn_new"])) < 1e-6
    ctx.close()


def test_time_loop_matches_reference_output():
    """The CUDA time loop against the reference's own: tests/golden/ref_loop.npz
    holds populations (a sample), body force and node positions after 100
    iterations of the reference's loop (LBM blocks every step, its cell blocks at
    50 and 100; ZebraflowWT.c:5646-12189) on the capped scene of
    tests/golden/ib_scene.py.  Bounds: populations 2e-6 (they move by ~6e-4),
    body force 1e-3 of its largest value (float atomics in the spreading),
    positions 1e-5 um."""
    import os
    from golden import ib_scene as S
    here = os.path.join(os.path.dirname(__file__), "golden")
    G = np.load(os.path.join(here, "ref_setup.npz"))
    R = np.load(os.path.join(here, "ref_ib.npz"))
    L = np.load(os.path.join(here, "ref_loop.npz"))
    b = S.lattice(capped=True)
    p = zf.default_params(nx=S.NX, ny=S.NY, nz=S.NZ, origin=S.ORIGIN, tau=1.22, tau_from_phase=1,
                          wall_mode=zf.WALL_REF_EQ, periodic=(0, 0, 0), stagger=50)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    ctx.set_wall(*S.wall())
    ctx.set_mesh(G["mesh_x"], G["mesh_tri"], G["nuc_x"], G["nuc_edges"])
    ctx.set_cells(R["x"], R["xn"])
    ctx.upload_populations(S.populations(b).astype(np.float32))
    ctx.step(int(L["steps"]))
    f = ctx.download_populations()
    assert np.max(np.abs(f[:, L["sample"]] - L["f_sample"])) < 2e-6
    bf_ref = np.zeros((3, f.shape[1]), np.float32)
    bf_ref[:, L["bf_idx"]] = L["bf_val"]
    assert rel_close(ctx.download_bodyforce(), bf_ref, 1e-3)
    xg, xng, sg = ctx.cells()
    assert np.array_equal(sg, L["status"])
    assert np.max(np.abs(xg - L["x_new"])) < 1e-5 and np.max(np.abs(xng - L["xn_new"])) < 1e-5
    ctx.close()


def test_nucleus_membrane_stage_matches_reference_output():
    """k_nuc_memb against the reference's nucleus-membrane block, built with its
    sub-point array tp widened to the 20 rows its loops use (the shipped
    declaration holds 16, ZebraflowWT.c:2307): tests/golden/ref_nuc.npz holds
    the repulsion increments on the scene variant of tests/golden/ib_scene.py
    whose nuclei reach their membranes.  Bound: 1e-5 of the largest increment."""
    import os
    from golden import ib_scene as S
    here = os.path.join(os.path.dirname(__file__), "golden")
    G = np.load(os.path.join(here, "ref_setup.npz"))
    N = np.load(os.path.join(here, "ref_nuc.npz"))
    b = S.lattice()
    p = zf.default_params(nx=S.NX, ny=S.NY, nz=S.NZ, origin=S.ORIGIN, tau=1.22, tau_from_phase=0,
                          wall_mode=zf.WALL_REF_EQ, periodic=(0, 0, 0), stagger=50)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    ctx.set_wall(*S.wall())
    ctx.set_mesh(G["mesh_x"], G["mesh_tri"], G["nuc_x"], G["nuc_edges"])
    ctx.set_cells(N["x"], N["xn"])
    ctx.upload_populations(S.populations(b).astype(np.float32))
    ctx.cgsm_forces()
    ctx.ibm_interp()
    _, _, w0, _ = ctx.cell_kinematics()
    ctx.nuc_memb_repulsion(rebuild=True)
    _, _, w1, _ = ctx.cell_kinematics()
    d_ref = N["rep_nuc"].astype(np.float64) - N["rep_interp"]
    assert np.abs(d_ref).max() > 0
    assert rel_close(w1.astype(np.float64) - w0, d_ref, 1e-5)
    ctx.close()

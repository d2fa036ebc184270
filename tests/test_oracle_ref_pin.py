"""Pins the CPU oracle against outputs of the reference's own code.

tests/golden/ref_setup.npz was produced by tests/golden/make_ref_golden.py,
which compiles the reference's ZebraflowWT.c (unmodified, `main` renamed) with
oracle/ref/harness_setup.c and runs its set-up functions:
CGSM_ZFISHRBC_DATA_GEN + CGSM_FILAMENT_PARAMETERS + CGSM_EQUILIBRIUM_METRICS on
the shipped zebrafish RBC mesh (ZebraflowWT.c:1592-2223, :2336-2346) and
LBM_DOM_SETUP + LBM_BC_SETUP on a synthetic tube lattice (:1481-1589).

tests/golden/ref_step.npz comes from the same script and oracle/ref/harness_step.c:
five LBM steps run by the reference's own stream-collide, wall and copy blocks
of its main() (:6101-6145, :6292-6433, :6601-6626) on a capped tube with a
phase-5 ball, from perturbed populations under a random body force.

tests/golden/ref_ib.npz, from oracle/ref/harness_ib.c: one membrane iteration
of the reference's own blocks (forces, IB interpolation with wall repulsion,
nucleus-membrane and RBC-RBC repulsion, IB spreading, position update;
:5659-12189) on the scene of tests/golden/ib_scene.py, state after every stage.

tests/golden/ref_nuc.npz, from the same harness linked against a build of the
reference whose nucleus-membrane sub-point array tp holds the 20 rows its loops
use (declared with 16, ZebraflowWT.c:2307): the nucleus-membrane stage on the
scene's variant whose nuclei reach their membranes.

tests/golden/ref_loop.npz, from the same harness: 100 iterations of the
reference's time loop (LBM blocks every step, the cell blocks at 50 and 100)
on that scene with its z ends capped, from its flow at rest force.

tests/golden/ref_wss.npz: wall pressure, wall shear stress and validity of the
cylinder's wall nodes, printed by the unmodified post-processor
PostProWSSandPressure.c (:275-369) run on input files of the same scene with a
pressurised swirling flow.

tests/golden/ref_cells.npz, from oracle/ref/harness_cells.c: one membrane step
run by the reference's own force blocks of its main() (CGSM_NODAL_FORCE_ZERO,
CGSM_AREA, cell centroid/area, CGSM_LOCAL_FORCES, CGSM_VOLUME_CALC;
:5706-7535) on four deformed RBCs with nuclei built from the shipped meshes, the
third with one screened force component, the fourth screened past the removal
count and removed.
"""
import os

import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleCells, OracleLBM, OracleWorld
from oracle.refsrc import have_reference, reference_dir

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_setup.npz"))
STEP = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_step.npz"))
CELLS = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_cells.npz"))
IB = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_ib.npz"))
WSS = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_wss.npz"))
LOOP = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_loop.npz"))
NUC = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_nuc.npz"))

# the harness lattice: a tube of radius 6 around (i,j) = (20,30), fluid for
# 7 < k < 38, wall points linked to it, all 1-based in the reference box; the
# oracle runs on the sub-box i 10..30, j 20..40, k 4..41 (ordering and
# neighbours are unchanged by the crop since everything outside is solid)
I0, J0, K0 = 10, 20, 4


def harness_lattice():
    nx, ny, nz = 21, 21, 38
    b = -np.ones((nx, ny, nz), np.int32)
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                I, J, K = i + I0, j + J0, k + K0
                if (I - 20) ** 2 + (J - 30) ** 2 < 36 and 6 < K < 38:
                    b[i, j, k] = 1
    fl = b > 0
    nb = np.zeros_like(fl)
    for e in zf.E[:18]:
        nb |= np.roll(fl, shift=(e[0], e[1], e[2]), axis=(0, 1, 2))
    region = np.zeros_like(fl)
    region[1:20, 1:20, 1:37] = True  # the harness marks walls in i 11..29, j 21..39, k 5..40
    b[(~fl) & nb & region] = 0
    return b


def test_membrane_setup_matches_reference():
    P = zf.default_params()
    o = OracleCells(GOLD["mesh_x"], GOLD["mesh_tri"], GOLD["nuc_x"], GOLD["nuc_edges"], P,
                    precision="f32")
    E, ep, epn, ae, av = o.topology()
    assert np.array_equal(E, GOLD["edges"])
    # LMAX, Plength, kp and cos(theta0) of every edge, and the nucleus springs,
    # to fp32 rounding of the same formulas
    for r in (0, 1, 2, 4):
        assert np.allclose(ep[r], GOLD["epar"][r], rtol=1e-6, atol=0)
    assert np.allclose(epn, GOLD["epar_n"], rtol=1e-6, atol=0)
    # sin(theta0) = +-sqrtf(1 - cos^2) cancels on nearly flat edges
    # (ZebraflowWT.c:2213-2214): there the reference's own value is fp32
    # rounding noise of size sqrt(2*2^-24) ~ 3.5e-4
    assert np.max(np.abs(ep[3] - GOLD["epar"][3])) < 3.5e-4
    curved = np.abs(GOLD["epar"][3]) > 0.05
    assert np.allclose(ep[3][curved], GOLD["epar"][3][curved], rtol=1e-4)


def test_lattice_setup_matches_reference():
    b = harness_lattice()
    o = OracleLBM(b, wall_mode=1)
    dom, bcnb = o.dom()
    ref_dom = GOLD["domlist"] - np.array([I0, J0, K0])
    assert np.array_equal(dom, ref_dom)
    # boundary list: every wall point, in listed order, with its designated neighbour
    ref_bc = GOLD["bclist"]
    ref_nb = GOLD["bcnlist"] - np.array([I0, J0, K0])
    wall = bcnb >= 0
    assert np.array_equal(dom[wall], ref_bc[:, :3] - np.array([I0, J0, K0]))
    assert np.all(ref_bc[:, 3] == 0)
    assert np.array_equal(dom[bcnb[wall]], ref_nb)


def step_lattice():
    """The step harness's lattice cropped to its listed points' bounding box
    (listed order is unchanged by the crop), and the crop's origin."""
    listed = STEP["listed"]
    lo = listed[:, :3].min(0)
    b = -np.ones(tuple(listed[:, :3].max(0) - lo + 1), np.int32)
    b[tuple((listed[:, :3] - lo).T)] = listed[:, 3]
    return b, lo


def run_oracle_steps(precision, **kw):
    b, lo = step_lattice()
    args = dict(wall_mode=1, tau_from_phase=True, dt=0.5, precision=precision)
    args.update(kw)
    o = OracleLBM(b, **args)
    dom, _ = o.dom()
    assert np.array_equal(dom, STEP["listed"][:, :3] - lo)
    o.set_f(STEP["f0"].astype(np.float64))
    o.set_bodyforce(STEP["bf0"].astype(np.float64))
    out = {}
    steps = int(STEP["steps"])
    for s in range(1, steps + 1):
        o.step(rbc_flag=(s == steps))  # the harness's last step is a membrane step
        if s == 1:
            out["f1"] = o.get_f()
    out["fN"] = o.get_f()
    out["D"], out["U"], out["V"], out["W"] = o.moments()
    out["bfN"] = o.get_bodyforce()
    return out


# The reference evaluates the step in float storage with double temporaries
# (its equilibrium constants are double), the oracle in pure fp32 or fp64: the
# populations agree to a few fp32 ulp (|f| <= 0.35, ulp 3e-8) per step.  The
# body force moves them by ~4e-3 over the five steps, so an error in a
# direction, a weight, the force term or a relaxation time shows up orders of
# magnitude above these bounds (see test_lbm_step_pin_detects_a_wrong_tau).
F_TOL = 3e-7
D_TOL = 1e-6
U_TOL = 1e-7


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_lbm_step_matches_reference(precision):
    out = run_oracle_steps(precision)
    assert np.max(np.abs(STEP["fN"] - STEP["f0"])) > 3e-3
    assert np.max(np.abs(out["f1"] - STEP["f1"])) < F_TOL
    assert np.max(np.abs(out["fN"] - STEP["fN"])) < F_TOL
    assert np.max(np.abs(out["D"] - STEP["D"])) < D_TOL
    for a in "UVW":
        assert np.max(np.abs(out[a] - STEP[a])) < U_TOL
    # the membrane step clears the body force at every listed point
    assert np.all(STEP["bfN"] == 0) and np.all(out["bfN"] == 0)


def test_lbm_step_pin_detects_a_wrong_tau():
    """A mistake planted in the oracle: one relaxation time for every phase
    (the 33 phase-5 points relax with tau = 1.22 instead of 4.1)."""
    out = run_oracle_steps("f64", tau_from_phase=False, tau=1.22)
    assert np.max(np.abs(out["fN"] - STEP["fN"])) > 100 * F_TOL


PRESSURE = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_pressure.npz"))


def run_oracle_pressure(precision, run, shift=0):
    """The fixture's pressure-inlet run `run` through the oracle (shift moves
    the waveform's time by that many iterations)."""
    from golden import pressure_scene as PS
    lo, hi, it0 = (int(v) for v in PRESSURE["runs"][run])
    b = PS.lattice(lo, hi)
    o = OracleLBM(b, wall_mode=1, tau_from_phase=True, dt=0.5, precision=precision)
    f0, bf0 = PS.initial_state(o.n)
    o.set_f(f0.astype(np.float64))
    o.set_bodyforce(bf0.astype(np.float64))
    o.set_iter(it0 + shift)
    for s in range(1, PS.STEPS + 1):
        o.step(rbc_flag=(s == PS.STEPS))
    return o.get_f(), np.stack(o.moments())


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_pressure_inlets_match_reference(precision):
    """Pressure inlet/outlet points (codes 1001-1009, ZebraflowWT.c:6316-6426)
    against the reference's own blocks on five runs covering the waveforms:
    moments of every listed point and the populations of the boundary points
    after five steps."""
    for run in range(len(PRESSURE["runs"])):
        f, mom = run_oracle_pressure(precision, run)
        ref = PRESSURE[f"run{run}_mom"]
        bc = PRESSURE[f"run{run}_bc"]
        assert np.max(np.abs(f[:, bc] - PRESSURE[f"run{run}_fN_bc"])) < F_TOL, run
        assert np.max(np.abs(mom[0] - ref[0])) < D_TOL, run
        assert np.max(np.abs(mom[1:] - ref[1:])) < U_TOL, run
        # the inlet layers are driven: their density is the waveform's, not 1
        codes = PRESSURE["runs"][run][:2]
        assert np.abs(ref[0, bc] - 1).max() > 0.03, codes


def test_pressure_pin_detects_a_wrong_waveform_time():
    """A mistake planted in the oracle: the waveforms read a time 0.18 s late."""
    f, mom = run_oracle_pressure("f64", 0, shift=360000)
    assert np.max(np.abs(mom[0] - PRESSURE["run0_mom"][0])) > 100 * D_TOL


def run_oracle_cells(precision, **params):
    o = OracleCells(GOLD["mesh_x"], GOLD["mesh_tri"], GOLD["nuc_x"], GOLD["nuc_edges"],
                    zf.default_params(**params), precision=precision)
    ae = o.topology()[3]
    o.set_cells(CELLS["x"], CELLS["xn"])
    o.forces()
    return o, ae, o.get(), o.geometry()


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


# Bounds, relative to the largest value of each array.  The reference keeps
# coordinates in double and geometry and forces in float; the fp32 oracle
# evaluates the same float expressions (triangle geometry and per-cell sums come
# out identical here) and its node forces differ by summation order, a few
# 1e-6 of the largest force.  The fp64 oracle carries none of the reference's
# float rounding: its triangle areas differ by ~3e-5, node forces by ~1e-4.
# The fp64 oracle's normals of the smallest triangles of the distorted cells
# differ from the reference's float ones by up to ~3e-4.
CELL_TOL = {"f32": dict(geo=1e-6, nrm=1e-6, f=3e-5, fn=3e-6, cell=1e-6, glob=1e-5, vol=1e-4),
            "f64": dict(geo=1e-4, nrm=1e-3, f=5e-4, fn=1e-3, cell=1e-5, glob=3e-4, vol=3e-4)}


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_membrane_step_matches_reference(precision):
    t = CELL_TOL[precision]
    o, ae, g, (ta, tn, tc, nn) = run_oracle_cells(precision)
    # the reference's shape constants are the defaults (RBC_SURF, MCV, moduli)
    assert rel(ae, CELLS["tri_area_eq"]) < t["geo"]
    assert rel(ta, CELLS["tri_area"]) < t["geo"]
    assert np.max(np.abs(tn - CELLS["tri_normal"])) < t["nrm"]
    assert rel(tc, CELLS["tri_centroid"]) < t["geo"]
    assert np.max(np.abs(nn - CELLS["node_normal"])) < 10 * t["nrm"]
    assert np.abs(CELLS["ftot"]).max() > 1e-13
    assert rel(g["ftot"], CELLS["ftot"]) < t["f"]
    assert rel(g["ftot_n"], CELLS["ftot_n"]) < t["fn"]
    cf, rc = g["cell"], CELLS["cell"]
    assert np.allclose(cf[:, :5], rc[:, :5], rtol=t["cell"], atol=0)  # area, volume, centroid
    assert np.allclose(cf[:, 5], rc[:, 5], rtol=t["glob"], atol=0)     # F_AREA_GLOBAL
    assert np.allclose(cf[:, 6], rc[:, 6], rtol=t["vol"], atol=0)      # F_VOLUME_SCALAR
    # force screening and removal (ZebraflowWT.c:7083-7359, :7473-7501): cells 0
    # and 1 pass, cell 2 has one screened force component, cell 3 more than 500
    # and is removed; the per-cell counts and the global failure count match
    assert list(CELLS["status"][:, 0]) == [1, 1, 1, -5000]
    assert np.array_equal(g["status"], CELLS["status"][:, 0])
    assert CELLS["status"][2, 1] > 0 and CELLS["status"][3, 1] > 500
    assert np.array_equal(g["cell"][:, 7].astype(np.int64), CELLS["status"][:, 1])
    assert g["counters"][0] == int(CELLS["simfailure"]) and g["counters"][1] == 1


def test_membrane_pin_detects_a_wrong_modulus():
    """A mistake planted in the oracle: the shear modulus 1 % too large."""
    o, _, g, _ = run_oracle_cells("f32", Es=3.03e-6)
    assert rel(g["ftot"], CELLS["ftot"]) > 30 * CELL_TOL["f32"]["f"]


def run_oracle_ib(precision, **overrides):
    from golden import ib_scene as S
    mesh = (GOLD["mesh_x"], GOLD["mesh_tri"], GOLD["nuc_x"], GOLD["nuc_edges"])
    b, p, lbm, oc, w = S.oracle_world(mesh, IB["x"], IB["xn"], precision, **overrides)
    assert lbm.n == int(IB["n_listed"])
    if precision == "f32" and not overrides:
        # the scene regenerates as the fixture's script made it (fp32 oracle)
        _, U, V, W = lbm.moments()
        assert np.array_equal(np.stack([U, V, W]).astype(np.float32).astype(np.float64).sum(axis=1),
                              IB["sum_vel"])
        wi, uv = w.wall_index(b.shape)
        assert int(wi.sum()) == int(IB["sum_windex"])
        assert uv.astype(np.float64).sum() == float(IB["sum_uvoid"])
    out = {}
    oc.forces()
    g = oc.get()
    out["ftot"], out["ftot_n"] = g["ftot"], g["ftot_n"]
    w.interp()
    out["vel_interp"], out["vel_n_interp"], out["rep_interp"], out["rep_n_interp"] = w.kinematics()
    w.nuc_memb(rebuild=True)
    _, _, out["rep_nuc"], out["rep_n_nuc"] = w.kinematics()
    w.rbc_rbc()
    _, _, out["rep_rbc"], out["rep_n_rbc"] = w.kinematics()
    w.spread()
    out["vel_spread"], out["vel_n_spread"], _, _ = w.kinematics()
    out["bf"] = lbm.get_bodyforce()
    w.update()
    g = oc.get()
    out["x_new"], out["xn_new"], out["status"] = g["x"], g["xn"], g["status"]
    return out


# Bounds relative to the largest value of each array (positions: um).  The
# fp32 oracle evaluates the reference's float expressions; its sums run in
# another order (node forces ~2e-5, spread body force ~5e-6, velocities ~2e-7
# here) while the wall and RBC-RBC repulsions come out identical.  The fp64
# oracle carries none of the reference's float rounding.
IB_TOL = {"f32": dict(f=1e-4, fn=1e-5, v=2e-6, rep=1e-6, bf=5e-5, x=1e-6),
          "f64": dict(f=1e-3, fn=3e-4, v=1e-5, rep=1e-5, bf=3e-4, x=1e-6)}


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_ib_stages_match_reference(precision):
    t = IB_TOL[precision]
    o = run_oracle_ib(precision)
    bf_ref = np.zeros_like(o["bf"])
    bf_ref[:, IB["bf_idx"]] = IB["bf_val"]
    assert rel(o["ftot"], IB["ftot"]) < t["f"] and rel(o["ftot_n"], IB["ftot_n"]) < t["fn"]
    # interpolated node velocities, and the wall repulsion (it acts on cell 2)
    assert rel(o["vel_interp"], IB["vel_interp"]) < t["v"]
    assert rel(o["vel_n_interp"], IB["vel_n_interp"]) < t["v"]
    assert np.abs(IB["rep_interp"]).max() > 0
    assert rel(o["rep_interp"], IB["rep_interp"]) < t["rep"]
    # the nuclei stay out of reach of their membranes in this scene
    assert np.array_equal(IB["rep_nuc"], IB["rep_interp"])
    assert np.array_equal(o["rep_nuc"], o["rep_interp"])
    # RBC-RBC repulsion (cells 0 and 1), as an increment
    d_ref = IB["rep_rbc"].astype(np.float64) - IB["rep_nuc"]
    assert np.abs(d_ref).max() > 0
    assert rel(o["rep_rbc"] - o["rep_nuc"], d_ref) < t["rep"] * 10
    # IB spreading: body force on the lattice and the node velocities after it
    assert np.abs(bf_ref).max() > 0
    assert rel(o["bf"], bf_ref) < t["bf"]
    assert rel(o["vel_spread"], IB["vel_spread"]) < t["v"]
    assert rel(o["vel_n_spread"], IB["vel_n_spread"]) < t["v"]
    # position update
    assert np.abs(IB["x_new"] - IB["x"]).max() > 0.01
    assert np.abs(o["x_new"] - IB["x_new"]).max() < t["x"]
    assert np.abs(o["xn_new"] - IB["xn_new"]).max() < t["x"]
    assert np.array_equal(o["status"], IB["status"]) and int(IB["simfailure"][0]) == 0


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_nucleus_membrane_stage_matches_reference(precision):
    from golden import ib_scene as S
    mesh = (GOLD["mesh_x"], GOLD["mesh_tri"], GOLD["nuc_x"], GOLD["nuc_edges"])
    b, p, lbm, oc, w = S.oracle_world(mesh, NUC["x"], NUC["xn"], precision)
    oc.forces()
    w.interp()
    _, _, r0, rn0 = w.kinematics()
    w.nuc_memb(rebuild=True)
    _, _, r1, rn1 = w.kinematics()
    d_ref = NUC["rep_nuc"].astype(np.float64) - NUC["rep_interp"]
    touched = np.any(d_ref != 0, axis=0)
    assert touched.sum() > 20
    assert np.array_equal(np.any(r1 - r0 != 0, axis=0), touched)
    # fp32: the same float expressions (6e-9 of the largest increment here); fp64: 3e-6
    assert rel(r1 - r0, d_ref) < (1e-6 if precision == "f32" else 3e-5)
    assert np.array_equal(rn1, rn0) and np.array_equal(NUC["rep_n_nuc"], NUC["rep_n_interp"])


def test_ib_pin_detects_a_wrong_velocity_scale():
    """A mistake planted in the oracle: the lattice-to-physical velocity scale
    1 % too large."""
    o = run_oracle_ib("f32", vel_scale=zf.default_params().vel_scale * 1.01)
    assert rel(o["vel_interp"], IB["vel_interp"]) > 100 * IB_TOL["f32"]["v"]


def run_oracle_wss(precision, origin_shift=0.0):
    from golden import ib_scene as S
    b = S.lattice()
    lbm = OracleLBM(b, wall_mode=1, periodic=(0, 0, 0), tau=1.22, dt=0.5, precision=precision)
    lbm.set_f(S.wss_populations(b))
    lbm.moments_from_f()
    if precision == "f32":
        D, U, V, W = lbm.moments()
        assert np.array_equal(np.stack([U, V, W, D]).astype(np.float32).astype(np.float64).sum(axis=1),
                              WSS["sum_vel"])
    origin = tuple(o + origin_shift for o in S.ORIGIN)
    w = OracleWorld(lbm, None, zf.default_params(nx=S.NX, ny=S.NY, nz=S.NZ, origin=origin,
                                                 periodic=(0, 0, 0)))
    xyz, tri, nrm = S.wall()
    w.set_wall(xyz, tri, nrm)
    return w.wss(S.wall_node_normals(xyz), pgauge=120.0)


# The post-processor prints pressure and WSS with six decimals (Pa): the fp32
# oracle agrees to that rounding (5e-7); the fp64 oracle to the post-processor's
# own float rounding (WSS ~5e-6 of its largest value, pressure ~6e-4 Pa from
# (D - 1) * 10000 / 3 in float).
WSS_TOL = {"f32": dict(wss=1e-6, press=1e-6), "f64": dict(wss=2e-5, press=2e-3)}


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_wss_matches_reference_postprocessor(precision):
    wss, press, valid = run_oracle_wss(precision)
    assert np.array_equal(valid, WSS["valid"]) and valid.sum() > 0.9 * valid.size
    assert np.abs(WSS["wss"]).max() > 0.5
    assert np.max(np.abs(wss - WSS["wss"])) < WSS_TOL[precision]["wss"]
    assert np.max(np.abs(press - WSS["press"])) < WSS_TOL[precision]["press"]


def test_wss_pin_detects_a_shifted_lattice():
    """A mistake planted in the oracle: the lattice origin off by a quarter of
    a lattice spacing."""
    wss, _, _ = run_oracle_wss("f32", origin_shift=0.125)
    assert np.max(np.abs(wss - WSS["wss"])) > 1000 * WSS_TOL["f32"]["wss"]


# 100 coupled iterations: populations change by ~6e-4 and agree to ~3e-7
# (fp32 and fp64 oracles alike: the reference's own float rounding), spread
# body force to ~3e-5 of its largest value, positions to ~2e-6 um.
LOOP_TOL = {"f32": dict(f=1e-6, bf=2e-4, x=1e-5), "f64": dict(f=2e-6, bf=3e-4, x=1e-5)}


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_time_loop_matches_reference(precision):
    from golden import ib_scene as S
    t = LOOP_TOL[precision]
    mesh = (GOLD["mesh_x"], GOLD["mesh_tri"], GOLD["nuc_x"], GOLD["nuc_edges"])
    b, p, lbm, oc, w = S.oracle_world(mesh, IB["x"], IB["xn"], precision, capped=True)
    f0 = S.populations(b)
    lbm.set_f(f0)
    w.step(int(LOOP["steps"]))
    f = lbm.get_f()
    smp = LOOP["sample"]
    assert np.abs(LOOP["f_sample"] - f0[:, smp]).max() > 1e-4
    assert np.max(np.abs(f[:, smp] - LOOP["f_sample"])) < t["f"]
    assert np.allclose(f.sum(axis=1), LOOP["f_sum"], rtol=1e-5, atol=0)
    bf = lbm.get_bodyforce()
    bf_ref = np.zeros_like(bf)
    bf_ref[:, LOOP["bf_idx"]] = LOOP["bf_val"]
    assert np.abs(bf_ref).max() > 0
    assert rel(bf, bf_ref) < t["bf"]
    g = oc.get()
    assert np.abs(LOOP["x_new"] - IB["x"]).max() > 0.01
    assert np.max(np.abs(g["x"] - LOOP["x_new"])) < t["x"]
    assert np.max(np.abs(g["xn"] - LOOP["xn_new"])) < t["x"]
    assert np.array_equal(g["status"], LOOP["status"]) and int(LOOP["simfailure"][0]) == 0


@pytest.mark.skipif(not have_reference(), reason="reference tree not present")
def test_fixtures_regenerate_from_the_reference(tmp_path):
    """The committed fixtures are what tests/golden/make_ref_golden.py makes
    from the reference tree: regenerated into a scratch folder, every array is
    identical."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run([sys.executable, os.path.join(root, "tests", "golden", "make_ref_golden.py"),
                    reference_dir(), str(tmp_path)], check=True, capture_output=True)
    for name in ("ref_setup", "ref_step", "ref_cells", "ref_ib", "ref_nuc", "ref_loop", "ref_wss", "ref_output",
                 "ref_pressure"):
        a = np.load(os.path.join(root, "tests", "golden", name + ".npz"))
        b = np.load(os.path.join(str(tmp_path), name + ".npz"))
        assert sorted(a.files) == sorted(b.files), name
        for k in a.files:
            assert np.array_equal(a[k], b[k]), (name, k)

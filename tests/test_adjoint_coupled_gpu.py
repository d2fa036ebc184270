"""Adjoint of the coupled step with moving cells (zf_adjoint_move_cells,
k_ib_vjp and k_membrane_vjp in zebraflow_b200/csrc/zf_adjoint_cells.cu, the
coupled driver in zf_adjoint.cpp) against central finite differences of the
FP64 CPU oracle (oracle/orc_*.inc) running the same forward.

1. The membrane and nucleus forces' vector-Jacobian product at deformed
   cells: lam^T dF/dx along a random direction, lam^T dF/dEs and dF/dkb.
2. The repulsion velocities' vector-Jacobian product (wall, nucleus-membrane,
   RBC-RBC).
3. The coupled forward: a bounce-back tube from rest with two deformed cells
   and the IB coupling every 10 iterations (the cells are interpolated,
   spread and moved 4 times in the window), J = mean |WSS| over a wall patch
   and steps 20..40.  Gradients with respect to tau, Es, kb, the body-force
   field (along a random direction) and the cells' starting positions (along
   a random direction); once with the repulsions off, then with each on.

The GPU adjoint runs in fp32 against the FP64 differences (measured: forces
x 2e-6, xn 5e-6, Es 3e-6, kb 4e-6; coupled tau 3e-5, Es 1e-6, kb 9e-5,
fb 6e-7, x_0 2e-5 relative).  The oracle forms the Peskin weights from the
fp64 positions here (OracleWorld.set_exact): with the reference's fp32
positions a position step below fp32 resolution is quantised, and a wider one
moves stencil points across the support sphere, where the weight jumps.
"""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleCells, OracleLBM, OracleWorld

pytestmark = pytest.mark.gpu

NX, NY, NZ, R = 40, 40, 48, 16.0
CX = CY = 19.5
TAU, G = 0.9, (0.0, 0.0, 2e-5)
NSTEPS, T0, T1, STAGGER = 40, 20, 40, 10


def node_normals(xyz, tri1, nrm):
    t = tri1 - 1
    p = xyz.T.astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(p[t[1]] - p[t[0]], p[t[2]] - p[t[0]]), axis=1)
    acc = np.zeros((xyz.shape[1], 3))
    for v in range(3):
        np.add.at(acc, t[v], area[:, None] * nrm.T)
    acc /= np.linalg.norm(acc, axis=1, keepdims=True)
    return np.ascontiguousarray(acc.T, np.float32)


def case():
    b = zf.gen_tube(NX, NY, NZ, CX, CY, R, True)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    # thick cells, clear of the wall and of each other: the repulsions (wall,
    # nucleus-membrane, and RBC-RBC, which also pushes apart the facing sides
    # of one thin cell) stay off in the window
    rest = xyz * np.array([3.5, 2.25, 2.0])
    rest_n = xyzn * np.array([1.25, 0.9, 0.6])
    mesh = (rest, tri, rest_n, zf.mesh_edges(trin))
    x, xn = zf.gen_cells(b, 2, rest, rest_n, (3.5, 2.25, 2.0), seed=5, margin=1.5, wall_clear=1.5)
    rng = np.random.default_rng(9)
    c0 = x.mean(axis=2, keepdims=True)
    x = c0 + (x - c0) * np.array([1.06, 0.97, 1.0])[:, None, None] + 0.02 * rng.standard_normal(x.shape)
    wall = zf.gen_wall_tube(CX, CY, R, NZ)
    z = wall[0][2]
    patch = np.nonzero((z > 6.0) & (z < 16.0))[0].astype(np.int32)
    return b, mesh, (x, xn), wall, patch


def params(**kw):
    base = dict(nx=NX, ny=NY, nz=NZ, tau=TAU, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                periodic=(0, 0, 1), g=G, origin=(0.0, 0.0, 0.0), area0=0.0, volume0=0.0,
                storage=zf.STORE_F32_DEV, stagger=STAGGER)
    base.update(kw)
    return zf.default_params(**base)


def gpu_ctx(b, mesh, cells, wall, **kw):
    ctx = zf.Context(params(**kw))
    ctx.set_lattice(b)
    ctx.set_wall(*wall)
    ctx.set_mesh(*mesh)
    ctx.set_cells(*cells)
    return ctx


def oracle_forces(mesh, cells, **kw):
    oc = OracleCells(*mesh, params(**kw), precision="f64")
    oc.set_cells(*cells)
    oc.forces()
    g = oc.get()
    oc.close()
    return g["ftot"], g["ftot_n"]


TOL = 1e-4  # the membrane forces alone


def test_membrane_vjp_matches_fp64_finite_differences():
    b, mesh, cells, wall, _ = case()
    ctx = gpu_ctx(b, mesh, cells, wall)
    x, xn = cells
    rng = np.random.default_rng(4)
    lam = rng.standard_normal(x.shape).astype(np.float32)
    lam_n = rng.standard_normal(xn.shape).astype(np.float32)
    gx, gxn, gEs, gkb = ctx.membrane_vjp(lam, lam_n)
    ctx.close()

    def lf(xx, xxn, **kw):
        f, fn = oracle_forces(mesh, (xx, xxn), **kw)
        return float(np.sum(lam * f) + np.sum(lam_n * fn))

    v = rng.standard_normal(x.shape)
    vn = rng.standard_normal(xn.shape)
    # small steps: bending switches off where |cos| of a dihedral exceeds 0.99,
    # a jump that a wider difference could straddle
    h = 1e-8
    fd = {"x.v": (lf(x + h * v, xn) - lf(x - h * v, xn)) / (2 * h),
          "xn.vn": (lf(x, xn + h * vn) - lf(x, xn - h * vn)) / (2 * h)}
    P = params()
    for name, base in (("Es", P.Es), ("kbend", P.kbend)):
        d = 1e-4 * base
        fd[name] = (lf(x, xn, **{name: base + d}) - lf(x, xn, **{name: base - d})) / (2 * d)
    ad = {"x.v": float(np.sum(gx * v)), "xn.vn": float(np.sum(gxn * vn)), "Es": gEs, "kbend": gkb}
    print({k: (ad[k], fd[k], abs(ad[k] - fd[k]) / abs(fd[k])) for k in fd})
    for k in fd:
        assert fd[k] != 0.0
        assert abs(ad[k] - fd[k]) <= TOL * abs(fd[k]), (k, ad[k], fd[k])


def oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0, **kw):
    """The coupled forward on the FP64 oracle: the reference loop from
    iteration 0 with BF_0 = S F(x_0) + fb and fb added to every spread field."""
    p = params(**kw)
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=p.tau, g=tuple(p.g), precision="f64")
    lbm.set_f(f0)
    oc = OracleCells(*mesh, p, precision="f64")
    oc.set_cells(*cells)
    w = OracleWorld(lbm, oc, p)
    w.set_wall(*wall)
    # weights from the fp64 positions: the reference's fp32 positions would
    # quantise the small position steps of the differences below
    w.set_exact(True)
    oc.forces()
    w.spread()
    lbm.set_bodyforce(lbm.get_bodyforce() + fb)
    J = 0.0
    for t in range(1, NSTEPS + 1):
        membrane = t % STAGGER == 0
        if membrane:
            oc.forces()
        lbm.step(rbc_flag=membrane)
        if membrane:
            w.interp()
            w.nuc_memb(rebuild=(t % p.nuc_list_period == 0))
            w.rbc_rbc()
            w.spread()
            lbm.set_bodyforce(lbm.get_bodyforce() + fb)
            w.update()
        if T0 <= t <= T1:
            wss, _, _ = w.wss(nrm)
            J += np.linalg.norm(wss[:, patch].astype(np.float64), axis=0).mean()
    kin = w.kinematics()
    for o in (w, oc, lbm):
        o.close()
    return J / (T1 - T0 + 1), kin


TOL_COUPLED = 3e-4


def rep_case():
    """Thick cells stacked 0.6 um apart along z, 0.15 um from the wall, with a
    nucleus 0.15 um inside each membrane: the wall, nucleus-membrane and
    RBC-RBC repulsions are all on, and their forward stays smooth under small
    steps (facing surfaces, no rims in reach)."""
    b = zf.gen_tube(NX, NY, NZ, CX, CY, R, True)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest = xyz * np.array([3.5, 2.25, 2.0])
    rest_n = xyzn * np.array([1.25, 0.9, 1.85])
    mesh = (rest, tri, rest_n, zf.mesh_edges(trin))
    rng = np.random.default_rng(9)
    cen = np.array([[14.1, 9.75, 6.0], [14.1, 9.75, 10.6]])
    x = np.stack([(rest + c).T for c in cen], axis=1) + 0.02 * rng.standard_normal((3, 2, rest.shape[0]))
    xn = np.stack([(rest_n + c).T for c in cen], axis=1)
    wall = zf.gen_wall_tube(CX, CY, R, NZ)
    z = wall[0][2]
    patch = np.nonzero((z > 6.0) & (z < 16.0))[0].astype(np.int32)
    return b, mesh, (x, xn), wall, patch


def one_repulsion_case(kind):
    """Thick cells with one repulsion on: "wall" (a cell 0.15 um from the
    wall), "nuc" (nucleus 0.15 um inside its membrane), "rbc" (two cells
    stacked 0.6 um apart)."""
    b = zf.gen_tube(NX, NY, NZ, CX, CY, R, True)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest = xyz * np.array([3.5, 2.25, 2.0])
    rest_n = xyzn * np.array([1.25, 0.9, 1.85 if kind == "nuc" else 1.2])
    mesh = (rest, tri, rest_n, zf.mesh_edges(trin))
    rng = np.random.default_rng(9)
    cen = {"wall": [[14.1, 9.75, 6.0], [9.75, 9.75, 16.0]], "nuc": [[9.75, 9.75, 6.0], [9.75, 9.75, 16.0]],
           "rbc": [[9.75, 9.75, 6.0], [9.75, 9.75, 10.6]]}[kind]
    x = np.stack([(rest + np.array(c)).T for c in cen], axis=1) + 0.02 * rng.standard_normal((3, 2, rest.shape[0]))
    xn = np.stack([(rest_n + np.array(c)).T for c in cen], axis=1)
    wall = zf.gen_wall_tube(CX, CY, R, NZ)
    z = wall[0][2]
    patch = np.nonzero((z > 6.0) & (z < 16.0))[0].astype(np.int32)
    return b, mesh, (x, xn), wall, patch


def oracle_wrep(b, mesh, cells, base, wall):
    """Repulsion velocities of one membrane iteration on the FP64 oracle from
    the fp64 positions (nucleus-membrane lists built at `base`)."""
    p = params()
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=p.tau, g=tuple(p.g), precision="f64")
    oc = OracleCells(*mesh, p, precision="f64")
    w = OracleWorld(lbm, oc, p)
    w.set_wall(*wall)
    w.set_exact(True)
    oc.set_cells(*base)
    oc.forces()
    w.nuc_memb(rebuild=True)
    oc.set_cells(*cells)
    oc.forces()
    w.interp()
    w.nuc_memb(rebuild=False)
    w.rbc_rbc()
    k = w.kinematics()[2]
    for o in (w, oc, lbm):
        o.close()
    return k


def test_repulsion_vjp_matches_fp64_finite_differences():
    """zf_repulsion_vjp: the wall, nucleus-membrane and RBC-RBC repulsion
    velocities' vector-Jacobian product (measured 2e-6 and 1e-6 relative)."""
    b, mesh, cells, wall, _ = rep_case()
    x, xn = cells
    ctx = gpu_ctx(b, mesh, cells, wall)
    rng = np.random.default_rng(7)
    lam = rng.standard_normal(x.shape).astype(np.float32)
    gx, gxn = ctx.repulsion_vjp(lam)
    ctx.close()
    parts = oracle_wrep(b, mesh, cells, cells, wall)
    assert (np.abs(parts) > 0).any(axis=0).sum() > 50  # the repulsions are on
    v = rng.standard_normal(x.shape)
    vn = rng.standard_normal(xn.shape)
    h = 1e-8
    lf = lambda xx, xxn: float(np.sum(lam * oracle_wrep(b, mesh, (xx, xxn), cells, wall)))  # noqa: E731
    fd = {"x.v": (lf(x + h * v, xn) - lf(x - h * v, xn)) / (2 * h),
          "xn.vn": (lf(x, xn + h * vn) - lf(x, xn - h * vn)) / (2 * h)}
    ad = {"x.v": float(np.sum(gx * v)), "xn.vn": float(np.sum(gxn * vn))}
    print({k: (ad[k], fd[k], abs(ad[k] - fd[k]) / abs(fd[k])) for k in fd})
    for k in fd:
        assert fd[k] != 0.0
        assert abs(ad[k] - fd[k]) <= TOL * abs(fd[k]), (k, ad[k], fd[k])


@pytest.mark.parametrize("scene", ["clear", "wall", "nuc", "rbc"])
def test_coupled_adjoint_matches_fp64_finite_differences(scene):
    """clear: the repulsions stay off in the window; wall, nuc, rbc: that
    repulsion acts on every membrane iteration (measured x_0 1e-6, 1e-5,
    7e-6).  One scene per repulsion: in the scene with all three on
    (rep_case) their position gradients cancel to a sixth of each, and the
    agreement measured there was 9e-4."""
    b, mesh, cells, wall, patch = case() if scene == "clear" else one_repulsion_case(scene)
    nrm = node_normals(*wall)
    ctx = gpu_ctx(b, mesh, cells, wall)
    ctx.adjoint_move_cells(True)
    rng = np.random.default_rng(3)
    fb = (1e-5 * rng.standard_normal((3, ctx.n_listed))).astype(np.float32)
    f0 = ctx.download_populations().astype(np.float64)
    x_before = ctx.cells()[0]
    J, gfb, gtau, gEs, gkb = ctx.wss_adjoint(NSTEPS, T0, T1, patch, fb=fb, node_normals=nrm, checkpoint=7)
    gx, gxn = ctx.adjoint_position_gradient()
    assert np.array_equal(ctx.cells()[0], x_before)  # the positions are put back
    J2 = ctx.wss_objective(NSTEPS, T0, T1, patch, fb=fb, node_normals=nrm)
    assert J2 == pytest.approx(J, rel=1e-6)
    ctx.close()

    Jo, kin = oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0)
    active = int((np.abs(kin[2]) > 0).any(axis=0).sum())
    print("nodes with repulsion", active)
    assert (active == 0) if scene == "clear" else (active > 5)
    assert J == pytest.approx(Jo, rel=1e-4)
    x, xn = cells
    P = params()
    fd = {}
    for name, base, rel in (("tau", P.tau, 1e-4), ("Es", P.Es, 1e-4), ("kbend", P.kbend, 1e-4)):
        d = rel * base
        jp = oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0, **{name: base + d})[0]
        jm = oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0, **{name: base - d})[0]
        fd[name] = (jp - jm) / (2 * d)
    h = 1e-4
    v = rng.standard_normal(fb.shape)
    v *= 1e-5 / np.abs(v).max()
    jp = oracle_J(b, mesh, cells, wall, patch, nrm, fb + h * v, f0)[0]
    jm = oracle_J(b, mesh, cells, wall, patch, nrm, fb - h * v, f0)[0]
    fd["fb.v"] = (jp - jm) / (2 * h)
    vx = rng.standard_normal(x.shape)
    vxn = rng.standard_normal(xn.shape)
    hx = 1e-8
    jp = oracle_J(b, mesh, (x + hx * vx, xn + hx * vxn), wall, patch, nrm, fb, f0)[0]
    jm = oracle_J(b, mesh, (x - hx * vx, xn - hx * vxn), wall, patch, nrm, fb, f0)[0]
    fd["x.v"] = (jp - jm) / (2 * hx)
    ad = {"tau": gtau, "Es": gEs, "kbend": gkb, "fb.v": float(np.sum(gfb.astype(np.float64) * v)),
          "x.v": float(np.sum(gx * vx) + np.sum(gxn * vxn))}
    print({k: (ad[k], fd[k], abs(ad[k] - fd[k]) / abs(fd[k])) for k in fd})
    for k in fd:
        assert fd[k] != 0.0
        assert abs(ad[k] - fd[k]) <= TOL_COUPLED * abs(fd[k]), (k, ad[k], fd[k])

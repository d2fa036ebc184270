"""Hand-written adjoint of the coupled step for the WSS objective
(zebraflow_b200/csrc/zf_adjoint.cpp, k_lbm_adj in zf_lbm.cu, the adjoint
pieces in zf_ib.cu) against central finite differences of the FP64 CPU
oracle running the same forward (oracle/orc_*.inc).

Forward (cells held at their positions): BODYFORCE = spread(membrane forces)
+ fb, 40 LBM steps of a bounce-back tube from rest, J = mean |WSS| over a wall
patch and steps 20..40.  The reference gradient is the FP64 oracle's central
difference with relative step 1e-4 (for fb: along a random direction).  The
GPU adjoint runs in fp32: its gradients agree with the FP64 reference to 1e-4
relative (measured: tau 2e-5, Es 4e-7, kb 7e-6, fb 5e-7), J to 1e-4; checkpointing (every 7 steps) gives the same gradients
as keeping every state (to 1e-5: float atomics reorder the last bits).
"""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleCells, OracleLBM, OracleWorld

pytestmark = pytest.mark.gpu

NX, NY, NZ, R = 40, 40, 48, 16.0
CX = CY = 19.5
TAU, G = 0.9, (0.0, 0.0, 2e-5)
NSTEPS, T0, T1 = 40, 20, 40


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
    rest = xyz * np.array([3.5, 2.25, 1.0])
    rest_n = xyzn * np.array([1.25, 0.9, 0.6])
    mesh = (rest, tri, rest_n, zf.mesh_edges(trin))
    x, xn = zf.gen_cells(b, 2, rest, rest_n, (3.5, 2.25, 1.0), seed=5, margin=0.4)
    # deformed cells (at their rest shape the spring and bending forces vanish)
    rng = np.random.default_rng(9)
    c0 = x.mean(axis=2, keepdims=True)
    x = c0 + (x - c0) * np.array([1.06, 0.97, 1.0])[:, None, None] + 0.02 * rng.standard_normal(x.shape)
    cells = (x, xn)
    wall = zf.gen_wall_tube(CX, CY, R, NZ)
    z = wall[0][2]
    patch = np.nonzero((z > 6.0) & (z < 16.0))[0].astype(np.int32)
    return b, mesh, cells, wall, patch


def params(**kw):
    base = dict(nx=NX, ny=NY, nz=NZ, tau=TAU, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                periodic=(0, 0, 1), g=G, origin=(0.0, 0.0, 0.0), area0=0.0, volume0=0.0,
                storage=zf.STORE_F32_DEV)
    base.update(kw)
    return zf.default_params(**base)


def gpu_ctx(b, mesh, cells, wall, **kw):
    ctx = zf.Context(params(**kw))
    ctx.set_lattice(b)
    ctx.set_wall(*wall)
    ctx.set_mesh(*mesh)
    ctx.set_cells(*cells)
    return ctx


def oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0, **kw):
    """The same forward on the FP64 oracle."""
    p = params(**kw)
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=p.tau, g=tuple(p.g), precision="f64")
    lbm.set_f(f0)
    oc = OracleCells(*mesh, p, precision="f64")
    oc.set_cells(*cells)
    w = OracleWorld(lbm, oc, p)
    w.set_wall(*wall)
    oc.forces()
    w.spread()
    lbm.set_bodyforce(lbm.get_bodyforce() + fb)
    J = 0.0
    for t in range(1, NSTEPS + 1):
        lbm.step(rbc_flag=False)
        if T0 <= t <= T1:
            wss, _, _ = w.wss(nrm)
            J += np.linalg.norm(wss[:, patch].astype(np.float64), axis=0).mean()
    for o in (w, oc, lbm):
        o.close()
    return J / (T1 - T0 + 1)


def test_adjoint_matches_fp64_finite_differences():
    b, mesh, cells, wall, patch = case()
    nrm = node_normals(*wall)
    ctx = gpu_ctx(b, mesh, cells, wall)
    rng = np.random.default_rng(3)
    fb = (1e-5 * rng.standard_normal((3, ctx.n_listed))).astype(np.float32)
    f0 = ctx.download_populations().astype(np.float64)
    J, gfb, gtau, gEs, gkb = ctx.wss_adjoint(NSTEPS, T0, T1, patch, fb=fb, node_normals=nrm, checkpoint=7)
    J2, gfb2, gtau2, gEs2, gkb2 = ctx.wss_adjoint(NSTEPS, T0, T1, patch, fb=fb, node_normals=nrm,
                                                   checkpoint=NSTEPS)
    # float atomics (spreading, the WSS seed) change the last bits from call to call
    assert abs(J2 - J) <= 1e-6 * abs(J)
    assert np.max(np.abs(gfb2 - gfb)) <= 1e-5 * np.abs(gfb).max()
    assert abs(gtau2 - gtau) <= 1e-5 * abs(gtau) and abs(gEs2 - gEs) <= 1e-5 * abs(gEs)
    assert abs(gkb2 - gkb) <= 1e-5 * abs(gkb)
    assert ctx.wss_objective(NSTEPS, T0, T1, patch, fb=fb, node_normals=nrm) == pytest.approx(J, rel=1e-6)

    Jo = oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0)
    assert J == pytest.approx(Jo, rel=1e-4)
    h = 1e-4
    P = params()
    fd = {}
    for name, base in (("tau", P.tau), ("Es", P.Es), ("kbend", P.kbend)):
        d = h * base
        jp = oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0, **{name: base + d})
        jm = oracle_J(b, mesh, cells, wall, patch, nrm, fb, f0, **{name: base - d})
        fd[name] = (jp - jm) / (2 * d)
    v = rng.standard_normal(fb.shape)
    v *= 1e-5 / np.abs(v).max()
    jp = oracle_J(b, mesh, cells, wall, patch, nrm, fb + h * v, f0)
    jm = oracle_J(b, mesh, cells, wall, patch, nrm, fb - h * v, f0)
    fd["fb.v"] = (jp - jm) / (2 * h)
    ad = {"tau": gtau, "Es": gEs, "kbend": gkb, "fb.v": float(np.sum(gfb.astype(np.float64) * v))}
    print({k: (ad[k], fd[k], abs(ad[k] - fd[k]) / abs(fd[k])) for k in fd})
    for k in fd:
        assert fd[k] != 0.0
        assert abs(ad[k] - fd[k]) <= 1e-4 * abs(fd[k]), (k, ad[k], fd[k])
    ctx.close()


def test_adjoint_leaves_state_and_costs():
    """The calls leave populations and body force as they were."""
    import time
    b, mesh, cells, wall, patch = case()
    ctx = gpu_ctx(b, mesh, cells, wall)
    ctx.lbm_steps(5)
    f_before = ctx.download_populations()
    bf_before = ctx.download_bodyforce()
    ctx.sync()
    t0 = time.perf_counter()
    ctx.wss_objective(NSTEPS, T0, T1, patch)
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    ctx.wss_adjoint(NSTEPS, T0, T1, patch, checkpoint=10)
    t_adj = time.perf_counter() - t0
    assert np.array_equal(ctx.download_populations(), f_before)
    assert np.array_equal(ctx.download_bodyforce(), bf_before)
    print(f"forward {t_fwd*1e3:.1f} ms, forward+adjoint {t_adj*1e3:.1f} ms")
    ctx.close()


# ---- flux-split objective, mixed-precision forward -------------------------------
#
# A periodic Y-bifurcation (parent radius 8, daughters 6 at +-20 degrees) in a
# 40x40x96 box, no cells: J = mean over steps 20..40 of the share of the axial
# flux through the +x daughter's mid cross-section.  The adjoint's dJ/dfb
# along a random direction agrees with central finite differences of the
# FP64 oracle to 1e-4 relative (measured 1e-8).  dJ/dtau is a near
# cancellation (in slow flow the split between two branches hardly depends on
# the viscosity), so it is checked to 5e-4 (measured 9e-5).

FNX, FNY, FNZ = 40, 40, 96


def flux_case():
    b, layout = zf.gen_bifurcation(FNX, FNY, FNZ, 8.0, 6.0, 20.0)
    return b, layout


def flux_sets(dom, b, layout):
    z2, z3 = layout[1], layout[2]
    k = int(round(0.5 * (z2 + z3)))
    cx = 0.5 * (FNX - 1)
    fluid = b[dom[:, 0], dom[:, 1], dom[:, 2]] > 0
    plane = fluid & (dom[:, 2] == k)
    return (np.nonzero(plane & (dom[:, 0] > cx))[0].astype(np.int32),
            np.nonzero(plane & (dom[:, 0] < cx))[0].astype(np.int32))


def flux_params(**kw):
    base = dict(nx=FNX, ny=FNY, nz=FNZ, tau=TAU, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                periodic=(0, 0, 1), g=G, origin=(0.0, 0.0, 0.0), storage=zf.STORE_F32_DEV)
    base.update(kw)
    return zf.default_params(**base)


def oracle_flux_J(b, pts0, pts1, fb, f0, tau):
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=tau, g=G, precision="f64")
    lbm.set_f(f0)
    lbm.set_bodyforce(fb.astype(np.float64))
    J = 0.0
    for t in range(1, NSTEPS + 1):
        lbm.step(rbc_flag=False)
        if T0 <= t <= T1:
            _, _, _, W = lbm.moments()
            q0, q1 = W[pts0].sum(), W[pts1].sum()
            J += q0 / (q0 + q1)
    lbm.close()
    return J / (T1 - T0 + 1)


def test_flux_adjoint_matches_fp64_finite_differences():
    b, layout = flux_case()
    ctx = zf.Context(flux_params())
    ctx.set_lattice(b)
    pts0, pts1 = flux_sets(ctx.domlist(), b, layout)
    assert pts0.size > 20 and pts1.size > 20
    n = (0.0, 0.0, 1.0)
    rng = np.random.default_rng(4)
    fb = (1e-5 * rng.standard_normal((3, ctx.n_listed))).astype(np.float32)
    f0 = ctx.download_populations().astype(np.float64)
    J, gfb, gtau, _, _ = ctx.flux_adjoint(NSTEPS, T0, T1, pts0, n, pts1, n, fb=fb, checkpoint=7)
    assert ctx.flux_objective(NSTEPS, T0, T1, pts0, n, pts1, n, fb=fb) == pytest.approx(J, rel=1e-6)
    Jo = oracle_flux_J(b, pts0, pts1, fb, f0, TAU)
    assert J == pytest.approx(Jo, rel=1e-4)
    h = 1e-4
    d = h * TAU
    fd_tau = (oracle_flux_J(b, pts0, pts1, fb, f0, TAU + d) - oracle_flux_J(b, pts0, pts1, fb, f0, TAU - d)) / (2 * d)
    v = rng.standard_normal(fb.shape)
    v *= 1e-5 / np.abs(v).max()
    fd_fb = (oracle_flux_J(b, pts0, pts1, fb + h * v, f0, TAU) -
             oracle_flux_J(b, pts0, pts1, fb - h * v, f0, TAU)) / (2 * h)
    ad_fb = float(np.sum(gfb.astype(np.float64) * v))
    print(f"J {J} oracle {Jo}; tau {gtau} fd {fd_tau}; fb.v {ad_fb} fd {fd_fb}")
    assert fd_tau != 0.0 and fd_fb != 0.0
    assert abs(gtau - fd_tau) <= 5e-4 * abs(fd_tau)
    assert abs(ad_fb - fd_fb) <= 1e-4 * abs(fd_fb)
    ctx.close()


def test_flux_adjoint_fp16_storage_against_fp32():
    """The same adjoint with the forward in fp16 deviation storage (stochastic
    rounding, fixed per step so that recomputation repeats it): J and the
    gradient field stay within MIXED_BOUNDS of the fp32-deviation adjoint
    (measured: J 3.4e-6, dJ/dfb 4.6e-6 relative L2, dJ/dtau 3.0e-3, the last
    a near-cancelling derivative as above)."""
    b, layout = flux_case()
    out = {}
    for st in (zf.STORE_F32_DEV, zf.STORE_F16):
        ctx = zf.Context(flux_params(storage=st))
        ctx.set_lattice(b)
        pts0, pts1 = flux_sets(ctx.domlist(), b, layout)
        n = (0.0, 0.0, 1.0)
        fb = (1e-5 * np.random.default_rng(4).standard_normal((3, ctx.n_listed))).astype(np.float32)
        r1 = ctx.flux_adjoint(NSTEPS, T0, T1, pts0, n, pts1, n, fb=fb, checkpoint=7)
        r2 = ctx.flux_adjoint(NSTEPS, T0, T1, pts0, n, pts1, n, fb=fb, checkpoint=NSTEPS)
        # recomputation repeats the rounding: any checkpoint interval gives the same result
        assert r2[0] == pytest.approx(r1[0], rel=1e-6)
        assert np.max(np.abs(r2[1] - r1[1])) <= 1e-5 * np.abs(r1[1]).max()
        out[st] = r1
        ctx.close()
    J32, g32, t32 = out[zf.STORE_F32_DEV][:3]
    J16, g16, t16 = out[zf.STORE_F16][:3]
    eJ = abs(J16 - J32) / abs(J32)
    eg = float(np.linalg.norm(g16.astype(np.float64) - g32) / np.linalg.norm(g32.astype(np.float64)))
    et = abs(t16 - t32) / abs(t32)
    print(f"fp16 vs fp32 adjoint: J {eJ:.2e}, dJ/dfb {eg:.2e}, dJ/dtau {et:.2e}")
    assert eJ <= MIXED_BOUNDS[0] and eg <= MIXED_BOUNDS[1] and et <= MIXED_BOUNDS[2]


MIXED_BOUNDS = (5e-5, 5e-5, 3e-2)

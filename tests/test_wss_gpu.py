"""Wall shear stress (zebraflow_b200/csrc/zf_ib.cu, k_wss) against the CPU
restatement of the reference post-processor (oracle/orc_ib.inc,
orc_world_wss; PostProWSSandPressure.c:275-369) and against Poiseuille flow.

Parity runs both from the same populations (downloaded from the GPU), so the
comparison isolates the WSS step: fp32 sums in the same order, moments
computed from deviations on the GPU and from populations on the CPU, hence
WSS within 1e-5 of its largest magnitude and pressure within 2e-3 Pa; the
valid flags are exact.
"""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleLBM, OracleWorld

pytestmark = pytest.mark.gpu

NX, NY, NZ, R = 40, 40, 48, 16.0
CX = CY = 19.5
G = 2e-5
TAU = 0.9


def node_normals(xyz, tri1, nrm):
    """Area-weighted node normals of the wall mesh (as zf_wss uses with NULL)."""
    t = tri1 - 1
    p = xyz.T.astype(np.float64)
    a = p[t[1]] - p[t[0]]
    b = p[t[2]] - p[t[0]]
    area = 0.5 * np.linalg.norm(np.cross(a, b), axis=1)
    acc = np.zeros((xyz.shape[1], 3))
    for v in range(3):
        np.add.at(acc, t[v], area[:, None] * nrm.T)
    acc /= np.linalg.norm(acc, axis=1, keepdims=True)
    return np.ascontiguousarray(acc.T, np.float32)


def make(steps):
    b = zf.gen_tube(NX, NY, NZ, CX, CY, R, True)
    p = zf.default_params(nx=NX, ny=NY, nz=NZ, tau=TAU, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, periodic=(0, 0, 1), g=(0, 0, G),
                          origin=(0.0, 0.0, 0.0), storage=zf.STORE_F32_DEV)
    wall = zf.gen_wall_tube(CX, CY, R, NZ)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    ctx.set_wall(*wall)
    ctx.lbm_steps(steps)
    return b, p, wall, ctx


def test_wss_matches_oracle():
    b, p, wall, ctx = make(400)
    nrm = node_normals(*wall)
    pg = -1000.0  # pressures near +1000 Pa, so that the valid flags are exercised
    wg, pgpu, vg = ctx.wss(nrm, pgauge=pg)
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=TAU, g=(0, 0, G), precision="f32")
    lbm.set_f(ctx.download_populations())
    lbm.moments_from_f()
    w = OracleWorld(lbm, None, p)
    w.set_wall(*wall)
    wo, po, vo = w.wss(nrm, pgauge=pg)
    assert np.abs(wo).max() > 0.1
    assert np.max(np.abs(wg - wo)) <= 1e-5 * np.abs(wo).max()
    assert np.array_equal(vg, vo)
    assert vo.sum() > 0.5 * vo.size
    assert np.max(np.abs(pgpu - po)[vo > 0]) <= 2e-3
    # the mesh's own node normals give the same result
    wn, _, _ = ctx.wss(None, pgauge=pg)
    assert np.max(np.abs(wn - wg)) <= 1e-5 * np.abs(wg).max()
    ctx.close()


def test_wss_poiseuille():
    """Developed flow in the tube: |WSS| = 0.0012 Pa.s * u(R - 1) / 0.5 um with
    u(r) = g (R^2 - r^2) / (4 nu), along -z, within the staircase error."""
    b, p, wall, ctx = make(12000)
    w, _, _ = ctx.wss(None)
    nu = (TAU - 0.5) / 3.0
    u = G * (R ** 2 - (R - 1) ** 2) / (4 * nu)
    expected = 0.0012 * u / 0.5e-6
    mean_z = w[2].mean()
    assert mean_z < 0
    assert abs(-mean_z - expected) <= 0.1 * expected
    assert np.abs(w[:2]).mean() <= 0.05 * expected
    ctx.close()


def test_wss_matches_reference_postprocessor():
    """k_wss against the reference's own post-processor: tests/golden/ref_wss.npz
    holds the wall pressure, WSS and validity that the unmodified
    PostProWSSandPressure.c (:275-369) printed (six decimals, Pa) for the
    cylinder of tests/golden/ib_scene.py under a pressurised swirling flow
    (fixture script: tests/golden/make_ref_golden.py).  Bound: 1e-5 of the
    largest WSS plus the print rounding; pressure 2e-3 Pa (one fp32 ulp of the
    density is 4e-4 Pa of (D - 1) * 10000 / 3)."""
    import os
    from golden import ib_scene as S
    R = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_wss.npz"))
    b = S.lattice()
    p = zf.default_params(nx=S.NX, ny=S.NY, nz=S.NZ, origin=S.ORIGIN, tau=1.22, tau_from_phase=0,
                          wall_mode=zf.WALL_REF_EQ, periodic=(0, 0, 0))
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    xyz, tri, nrm = S.wall()
    ctx.set_wall(xyz, tri, nrm)
    ctx.upload_populations(S.wss_populations(b).astype(np.float32))
    wss, press, valid = ctx.wss(S.wall_node_normals(xyz), pgauge=120.0)
    assert np.array_equal(valid, R["valid"])
    assert np.max(np.abs(wss - R["wss"])) < 1e-5 * np.abs(R["wss"]).max() + 1e-6
    assert np.max(np.abs(press - R["press"])) < 2e-3
    ctx.close()

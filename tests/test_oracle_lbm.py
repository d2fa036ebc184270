"""The CPU oracle (oracle/orc_lbm.inc) against the lattice-Boltzmann invariants
the reference scheme must satisfy.  The reference ships no tests or golden
vectors; these pins follow from its equations (ZebraflowWT.c:6100-6145,
:6290-6315, :6599-6626) and from the analytic Poiseuille profile."""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleLBM


def test_d3q19_lattice():
    E, W = zf.E, zf.W
    assert abs(W.sum() - 1) < 1e-15
    assert np.allclose(W @ E, 0)
    assert np.allclose((E.T * W) @ E, np.eye(3) / 3)
    opp = [q ^ 1 if q < 18 else 18 for q in range(19)]
    assert np.array_equal(E[opp], -E)  # ZebraflowWT.c:6114-6115


def periodic_box(n=6):
    return np.ones((n, n, n), np.int32)


def test_guo_momentum_and_mass_exact():
    """One fully periodic step: mass is conserved and sum_q c f_post = m + F_eff
    with F_eff = dt*BODYFORCE + g (the Guo scheme of ZebraflowWT.c:6133-6141)."""
    rng = np.random.default_rng(1)
    b = periodic_box()
    o = OracleLBM(b, wall_mode=0, periodic=(1, 1, 1), tau=0.8, dt=0.5, g=(1e-5, -2e-5, 3e-5))
    n = o.n
    f = zf.W[:, None] * (1 + 0.05 * rng.standard_normal((19, n)))
    bf = 1e-4 * rng.standard_normal((3, n))
    o.set_f(f)
    o.set_bodyforce(bf)
    # streaming on a fully periodic box permutes populations: totals are unchanged
    m0 = (zf.E.T.astype(float) @ f).sum(axis=1)
    M0 = f.sum()
    o.step()
    f1 = o.get_f()
    feff = 0.5 * bf.sum(axis=1) + n * np.array([1e-5, -2e-5, 3e-5])
    assert abs(f1.sum() - M0) < 1e-12 * M0
    assert np.allclose((zf.E.T.astype(float) @ f1).sum(axis=1), m0 + feff, atol=1e-13)


def test_rest_state_is_stationary():
    b = zf.gen_tube(16, 16, 8, 7.5, 7.5, 5, True)
    for mode in (0, 1):
        o = OracleLBM(b, wall_mode=mode, periodic=(0, 0, 1), tau=0.9)
        f0 = o.get_f()
        for _ in range(5):
            o.step()
        assert np.allclose(o.get_f(), f0, atol=1e-15)


def test_mass_conservation_bounce_back():
    rng = np.random.default_rng(2)
    b = zf.gen_tube(20, 20, 12, 9.5, 9.5, 7, True)
    o = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.7, g=(0, 0, 1e-5))
    f = zf.W[:, None] * (1 + 0.01 * rng.standard_normal((19, o.n)))
    o.set_f(f)
    m0 = o.mass()
    for _ in range(50):
        o.step()
    assert abs(o.mass() - m0) < 1e-11 * m0


def test_reference_wall_equilibrium():
    """Wall points carry feq(D[m], 0) of their designated neighbour
    (ZebraflowWT.c:6303-6315) and the moments pass sees them (:6601-6616)."""
    b = zf.gen_tube(16, 16, 8, 7.5, 7.5, 5, True)
    o = OracleLBM(b, wall_mode=1, periodic=(0, 0, 1), tau=0.9, g=(0, 0, 1e-4))
    for _ in range(3):
        o.step()
    f = o.get_f()
    D, U, V, W = o.moments()
    dom = np.argwhere(b >= 0)  # DOMLIST order (i outer, k inner)
    wall = b[dom[:, 0], dom[:, 1], dom[:, 2]] == 0
    fw = f[:, wall]
    ratio = fw / zf.W[:, None]
    assert np.allclose(ratio, ratio[0:1], rtol=1e-12)
    assert np.allclose(D[wall], fw.sum(axis=0), rtol=1e-12)
    assert np.all(np.abs(W[wall]) < 1e-14)


def test_poiseuille_profile():
    """Steady body-force flow in a bounce-back tube follows g(R^2-r^2)/(4 nu)."""
    R, tau, g = 7.0, 0.8, 1e-6
    nx = 18
    b = zf.gen_tube(nx, nx, 4, 8.5, 8.5, R, True)
    o = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=tau, g=(0, 0, g))
    for _ in range(3000):
        o.step()
    D, U, V, W = o.moments()
    dom = np.argwhere(b >= 0)
    fl = b[dom[:, 0], dom[:, 1], dom[:, 2]] > 0
    r2 = (dom[fl, 0] - 8.5) ** 2 + (dom[fl, 1] - 8.5) ** 2
    nu = (tau - 0.5) / 3
    # moments are post-collision without the half-force shift: add it back
    w = W[fl] + 0.5 * g / D[fl]
    # effective radius of a staircase bounce-back wall: fit R_eff, then check shape
    A = np.vstack([np.ones_like(r2), -r2]).T * g / (4 * nu)
    coef, *_ = np.linalg.lstsq(A, w, rcond=None)
    Reff2 = coef[0] / coef[1]
    assert abs(np.sqrt(Reff2) - R) < 0.6
    assert abs(coef[1] - 1) < 0.05          # curvature fixed by the viscosity (tau-0.5)/3
    pred = g / (4 * nu) * (Reff2 - r2) * coef[1]
    core = r2 < (R - 2) ** 2                # staircase-wall error stays near the wall
    assert np.max(np.abs(pred - w)[core]) < 0.03 * w.max()
    assert np.all(np.abs(U[fl]) < 1e-3 * w.max())


def test_oracle_wss_poiseuille():
    """The oracle's WSS (PostProWSSandPressure.c:275-369) on developed flow in a
    small periodic tube: mean axial WSS within 10 % of 0.0012 u(R-1)/0.5 um."""
    import zebraflow_b200 as zf
    from oracle.bind import OracleLBM, OracleWorld
    nx = ny = 22
    nz, R, c, g, tau = 8, 8.0, 10.5, 1e-4, 0.9
    b = zf.gen_tube(nx, ny, nz, c, c, R, True)
    lbm = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=tau, g=(0, 0, g), precision="f64")
    lbm.time_steps(4000)
    lbm.moments_from_f()
    p = zf.default_params(nx=nx, ny=ny, nz=nz, origin=(0.0, 0.0, 0.0), periodic=(0, 0, 1))
    w = OracleWorld(lbm, None, p)
    xyz, tri, nrm = zf.gen_wall_tube(c, c, R, nz)
    w.set_wall(xyz, tri, nrm)
    t = tri - 1
    pts = xyz.T.astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross((pts[t[1]] - pts[t[0]]), (pts[t[2]] - pts[t[0]])), axis=1)
    acc = np.zeros((xyz.shape[1], 3))
    for v in range(3):
        np.add.at(acc, t[v], area[:, None] * nrm.T)
    acc /= np.linalg.norm(acc, axis=1, keepdims=True)
    wss, _, _ = w.wss(np.ascontiguousarray(acc.T, np.float32))
    nu = (tau - 0.5) / 3.0
    expected = 0.0012 * g * (R ** 2 - (R - 1) ** 2) / (4 * nu) / 0.5e-6
    assert wss[2].mean() < 0
    assert abs(-wss[2].mean() - expected) <= 0.1 * expected
    w.close()
    lbm.close()

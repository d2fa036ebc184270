"""Periodic parent segments and cloning (include/zf.h zf_inflow_*, driven by
zebraflow_b200/inflow.py) against the oracle's restatement of the reference's
blocks (oracle/orc_inflow.c: ZebraflowWT.c:11926-11960, :12193-12403), on
random parents and region slots over many membrane iterations, both flow
directions.  The host steps run on the CPU; on the GPU the position update
that precedes them is the context's own (k_update), emulated here as
x += v dt for every active cell."""
import numpy as np
import pytest

from oracle.bind import lib as olib
from zebraflow_b200 import inflow

Z0, Z1, DX, DT = 10.0, 40.0, 0.5, 0.75
NN, NNN, NP, NR = 24, 6, 7, 10


def _p(a):
    return None if a is None else a.ctypes.data


def scenario(rng, direction):
    L = Z1 - Z0
    cen = rng.uniform(Z0 + 2, Z1 - 2, NP)
    xp = rng.normal(0.0, 1.0, (3, NP, NN))
    xp[2] = cen[:, None] + rng.uniform(-2.0, 2.0, (NP, NN))
    xnp = rng.normal(0.0, 0.5, (3, NP, NNN))
    xnp[2] = cen[:, None] + rng.uniform(-1.0, 1.0, (NP, NNN))
    status_p = rng.choice([2, 4], NP).astype(np.int32)
    regress_p = np.where(status_p == 2, rng.integers(0, 2, NP), 1).astype(np.int32)
    xr = np.full((3, NR, NN), -5000.0)
    xnr = np.full((3, NR, NNN), -5000.0)
    status_r = np.full(NR, -5000, np.int32)
    for m in range(NR - 4):  # slaves of random parents and independent cells, past the exit plane
        status_r[m] = -(int(rng.integers(0, NP)) + 1) if m % 2 == 0 else 1
        edge = Z1 if direction > 0 else Z0
        c = edge + direction * rng.uniform(-1.0, 4.0)
        xr[:, m] = rng.normal(0.0, 1.0, (3, NN))
        xr[2, m] = c + rng.uniform(-2.0, 2.0, NN)
        xnr[:, m] = rng.normal(0.0, 0.5, (3, NNN))
        xnr[2, m] = c + rng.uniform(-1.0, 1.0, NNN)
    assert L > 0
    return xp, xnp, status_p, regress_p, xr, xnr, status_r


def velocities(rng, direction, n, nn):
    v = rng.normal(0.0, 0.05, (3, n, nn))
    v[2] += direction * rng.uniform(0.5, 2.0, (n, 1))
    return v


@pytest.mark.parametrize("direction", [1, -1])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_inflow_steps_match_the_oracle(direction, seed):
    rng = np.random.default_rng(seed)
    seg = inflow.Segment(Z0, Z1, direction, DX)
    xp, xnp, st_p, rg_p, xr, xnr, st_r = scenario(rng, direction)
    o = [a.copy() for a in (xp, xnp, st_p, rg_p, xr, xnr, st_r)]
    oxp, oxnp, ost_p, org_p, oxr, oxnr, ost_r = o
    ocl = np.zeros(NP, np.int32)
    cl = np.zeros(NP, np.int32)
    L = olib()
    seen = {"clones": 0, "released": 0, "rearmed": 0}
    for it in range(40):
        vp, vnp = velocities(rng, direction, NP, NN), velocities(rng, direction, NP, NNN)
        vr, vnr = velocities(rng, direction, NR, NN), velocities(rng, direction, NR, NNN)
        # oracle: the reference's blocks with their own position updates
        L.orc_inflow_roi_update(Z0, Z1, direction, DX, DT, NR, NN, NNN, _p(oxr), _p(oxnr), _p(vr), _p(vnr),
                                _p(ost_r), NP, _p(vp), _p(vnp))
        before = ost_p.copy()
        L.orc_inflow_parent_update(Z0, Z1, direction, DT, NP, NN, NNN, _p(oxp), _p(oxnp), _p(vp), _p(vnp),
                                   _p(ost_p), _p(org_p), _p(ocl))
        seen["rearmed"] += int(((before == 4) & (ost_p == 2)).sum())
        seen["clones"] += int((ocl > 0).sum())
        L.orc_inflow_clone(Z0, Z1, direction, NP, NN, NNN, _p(oxp), _p(oxnp), _p(ost_p), _p(org_p), _p(ocl), NR,
                           _p(oxr), _p(oxnr), _p(ost_r))
        # product: the GPU update moved every active cell, then the host steps
        active = st_r != -5000
        xr[:, active] += vr[:, active] * DT
        xnr[:, active] += vnr[:, active] * DT
        xp += vp * DT
        xnp += vnp * DT
        slaves_before = (st_r < 0) & (st_r > -4998)
        inflow.slaves(seg, DT, xr, xnr, vr, vnr, st_r, vp, vnp)
        seen["released"] += int((slaves_before & (st_r == 1)).sum())
        inflow.parents(seg, xp, xnp, st_p, rg_p, cl)
        inflow.clone(seg, xp, xnp, st_p, rg_p, cl, xr, xnr, st_r)
        assert np.array_equal(st_p, ost_p) and np.array_equal(rg_p, org_p) and np.array_equal(st_r, ost_r), it
        np.testing.assert_allclose(xp, oxp, rtol=0, atol=1e-9)
        np.testing.assert_allclose(xnp, oxnp, rtol=0, atol=1e-9)
        np.testing.assert_allclose(xr, oxr, rtol=0, atol=1e-9)
        np.testing.assert_allclose(xnr, oxnr, rtol=0, atol=1e-9)
        # the parents stay in their segment
        assert xp[2].min() >= Z0 - 1e-9 and xp[2].max() < Z1 + 1e-9
        free = st_r == -5000
        if free.sum() < 3:  # recycle slots far downstream, as the region's exit would
            far = np.nonzero(st_r == 1)[0][:2]
            for a, b in ((st_r, ost_r),):
                a[far] = -5000
                b[far] = -5000
    print(seen)
    assert seen["clones"] > 0 and seen["released"] > 0


def test_clone_is_whole_across_the_exit_plane():
    """A parent straddling the periodic fold is copied whole: the nodes that
    were folded back behind the entry go one period on."""
    seg = inflow.Segment(Z0, Z1, 1, DX)
    xp = np.zeros((3, 1, 4))
    xp[2, 0] = [39.5, 39.9, 40.3, 40.6]  # two nodes already past z1
    xnp = np.zeros((3, 1, 1))
    xnp[2, 0] = 39.8
    st, rg, cl = np.array([2], np.int32), np.zeros(1, np.int32), np.zeros(1, np.int32)
    inflow.parents(seg, xp, xnp, st, rg, cl)
    assert cl[0] == 1 and np.allclose(xp[2, 0], [39.5, 39.9, 10.3, 10.6])
    xr = np.full((3, 2, 4), -5000.0)
    xnr = np.full((3, 2, 1), -5000.0)
    sr = np.array([1, -5000], np.int32)
    into = inflow.clone(seg, xp, xnp, st, rg, cl, xr, xnr, sr)
    assert into[0] == 1 and sr[1] == -1 and st[0] == 4 and rg[0] == 1 and cl[0] == 0
    assert np.allclose(xr[2, 1], [39.5, 39.9, 40.3, 40.6])

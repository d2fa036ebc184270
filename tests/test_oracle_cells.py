"""The CPU oracle of the membrane set-up and membrane forces
(oracle/orc_cells.inc) against invariants the reference scheme satisfies:
topology of the rhombus list (ZebraflowWT.c:1640-1805), zero force at the
calibrated rest shape (:1989-1990, :2195-2197, :2422), and conservation of
momentum and angular momentum by the internal forces (:6800-7535)."""
import gzip
import os

import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleCells
from oracle.refsrc import reference_dir

REF = reference_dir()


def ellipsoid_meshes():
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest = xyz * np.array([3.5, 2.25, 1.0])
    rest_n = xyzn * np.array([1.25, 0.9, 0.6])
    return rest, tri, rest_n, zf.mesh_edges(trin)


def rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a*a+b*b-c*c-d*d, 2*(b*c-a*d), 2*(b*d+a*c)],
                     [2*(b*c+a*d), a*a-b*b+c*c-d*d, 2*(c*d-a*b)],
                     [2*(b*d-a*c), 2*(c*d+a*b), a*a-b*b-c*c+d*d]])


def deformed_cells(rest, rest_n, n, seed, amp=0.03, scale=1.04):
    rng = np.random.default_rng(seed)
    X = np.empty((3, n, rest.shape[0]))
    XN = np.empty((3, n, rest_n.shape[0]))
    for c in range(n):
        R = rotation(rng)
        t = rng.uniform(20, 40, 3)
        X[:, c, :] = (scale * rest @ R.T + t + amp * rng.standard_normal(rest.shape)).T
        XN[:, c, :] = (rest_n @ R.T + t + 0.5 * amp * rng.standard_normal(rest_n.shape)).T
    return X, XN


def test_icosphere_rhombus_topology():
    rest, tri, rest_n, en = ellipsoid_meshes()
    o = OracleCells(rest, tri, rest_n, en, zf.default_params(area0=0, volume0=0))
    E, ep, epn, ae, av = o.topology()
    assert o.ne == 1920 and en.shape == (480, 2)
    t = tri - 1
    for e in range(o.ne):
        n1, n2, n3, n4, t1, t2 = E[e] - 1
        v1, v2 = list(t[t1]), list(t[t2])
        # tri1 holds (n1,n2,n3) in its own cyclic order; tri2 holds (n2,n1,n4)
        i = v1.index(n1)
        assert v1[(i + 1) % 3] == n2 and v1[(i + 2) % 3] == n3
        j = v2.index(n2)
        assert v2[(j + 1) % 3] == n1 and v2[(j + 2) % 3] == n4
    # edges appear in first-use order over triangles (v1v2, v2v3, v3v1)
    seen, order = set(), []
    for a, b, c in t:
        for p, q in ((a, b), (b, c), (c, a)):
            k = (min(p, q), max(p, q))
            if k not in seen:
                seen.add(k)
                order.append((p, q))
    assert np.array_equal(E[:, :2] - 1, np.array(order))


def test_rest_shape_has_zero_force():
    rest, tri, rest_n, en = ellipsoid_meshes()
    P = zf.default_params(area0=0, volume0=0)
    o = OracleCells(rest, tri, rest_n, en, P)
    o.set_cells(rest.T[:, None, :] + 10.0, rest_n.T[:, None, :] + 10.0)
    o.forces()
    g = o.get()
    # typical membrane force scale is 1e-13..1e-11 N
    assert np.abs(g["ftot"]).max() < 1e-21
    assert np.abs(g["ftot_n"]).max() < 1e-21
    assert abs(g["cell"][0, 0] - o.topology()[4][0]) < 1e-6 * g["cell"][0, 0]


def test_internal_forces_conserve_momentum():
    rest, tri, rest_n, en = ellipsoid_meshes()
    P = zf.default_params(area0=0, volume0=0)
    o = OracleCells(rest, tri, rest_n, en, P)
    # node noise small enough that no triangle becomes a sliver: the sliver
    # push (ZebraflowWT.c:6042-6084) is the one term that is not pairwise
    X, XN = deformed_cells(rest, rest_n, 3, seed=5, amp=0.01)
    o.set_cells(X, XN)
    o.forces()
    g = o.get()
    F = g["ftot"]
    scale = np.abs(F).max()
    assert scale > 1e-14
    for c in range(3):
        tot = F[:, c, :].sum(axis=1)
        assert np.all(np.abs(tot) < 1e-9 * scale * F.shape[2])
        x = X[:, c, :] - X[:, c, :].mean(axis=1, keepdims=True)
        torque = np.cross(x.T, F[:, c, :].T).sum(axis=0)
        assert np.all(np.abs(torque) < 1e-7 * scale * F.shape[2] * np.abs(x).max())
        assert np.abs(g["ftot_n"][:, c, :].sum(axis=1)).max() < 1e-9 * np.abs(g["ftot_n"]).max() * 162


def read_ref_mesh():
    def rd(name, conv):
        lines = gzip.open(os.path.join(REF, name), "rt").read().split("\n")[1:]
        return np.array([conv(v) for ln in lines for v in ln.split()])
    X = rd("ZFISHRBCNODES.dat.gz", float).reshape(-1, 3)
    T = rd("ZFISHRBCTRIANGLES.dat.gz", int).reshape(-1, 3).astype(np.int32)
    XN = rd("NucleusNodes.dat.gz", float).reshape(-1, 3)
    EN = rd("NucleusEdges.dat.gz", int).reshape(-1, 2).astype(np.int32)
    return X, T, XN, EN


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_reference_mesh_sizes_and_constants():
    """The shipped zebrafish RBC mesh yields the reference's compile-time sizes
    (NodeM 504, TriM 1004, EdgeM 1506, NodeM_N 121, EdgeM_N 544; ZebraflowWT.c:117-122)
    and its rest area equals RBC_SURF (ZebraflowWT.c:127)."""
    X, T, XN, EN = read_ref_mesh()
    assert X.shape == (504, 3) and T.shape == (1004, 3) and XN.shape == (121, 3) and EN.shape == (544, 2)
    o = OracleCells(X, T, XN, EN, zf.default_params(area0=0, volume0=0))
    E, ep, epn, ae, av = o.topology()
    assert o.ne == 1506
    assert abs(av[0] - 144.916e-12) < 1e-4 * 144.916e-12

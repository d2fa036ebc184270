"""Pins the CPU oracle against outputs of the reference's own code.

tests/golden/ref_setup.npz was produced by tests/golden/make_ref_golden.py,
which compiles the reference's ZebraflowWT.c (unmodified, `main` renamed) with
oracle/ref/harness_setup.c and runs its set-up functions:
CGSM_ZFISHRBC_DATA_GEN + CGSM_FILAMENT_PARAMETERS + CGSM_EQUILIBRIUM_METRICS on
the shipped zebrafish RBC mesh (ZebraflowWT.c:1592-2223, :2336-2346) and
LBM_DOM_SETUP + LBM_BC_SETUP on a synthetic tube lattice (:1481-1589).
"""
import os

import numpy as np

import zebraflow_b200 as zf
from oracle.bind import OracleCells, OracleLBM

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_setup.npz"))

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

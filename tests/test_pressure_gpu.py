"""Pressure inlet/outlet points (reference codes 1001-1009, the cardiac
waveforms of ZebraflowWT.c:6316-6426) in the CUDA step, held to the
reference's own blocks: tests/golden/ref_pressure.npz keeps the reference's
moments after five steps of oracle/ref/harness_step.c in its pressure mode
and the populations of its boundary points, for five runs that cover the
nine waveforms; the lattice and initial state are rebuilt by
tests/golden/pressure_scene.py.  Bounds as the plain step's reference pin
(tests/test_lbm_gpu.py)."""
import os

import numpy as np
import pytest

import zebraflow_b200 as zf
from golden import pressure_scene as PS

pytestmark = pytest.mark.gpu

REF = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_pressure.npz"))


@pytest.mark.parametrize("run", range(5))
def test_pressure_inlets_match_reference_output(run):
    lo, hi, it0 = (int(v) for v in REF["runs"][run])
    b = PS.lattice(lo, hi)
    nx, ny, nz = b.shape
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau_from_phase=1, wall_mode=zf.WALL_REF_EQ,
                          periodic=(0, 0, 0), dt=0.5)
    with zf.Context(p) as ctx:
        ctx.set_lattice(b)
        f0, bf0 = PS.initial_state(ctx.n_listed)
        ctx.upload_populations(f0)
        ctx.upload_bodyforce(bf0)
        ctx.set_iteration(it0)
        for s in range(1, PS.STEPS + 1):
            last = s == PS.STEPS
            ctx.lbm_step(store_moments=last, zero_bodyforce=last)
        assert ctx.iteration() == it0 + PS.STEPS
        f = ctx.download_populations()
        mom = np.stack(ctx.download_moments())
        bf = ctx.download_bodyforce()
    bc = REF[f"run{run}_bc"]
    ref = REF[f"run{run}_mom"]
    assert np.max(np.abs(f[:, bc] - REF[f"run{run}_fN_bc"])) < 5e-7
    assert np.max(np.abs(mom[0] - ref[0])) < 2e-6
    assert np.max(np.abs(mom[1:] - ref[1:])) < 2e-7
    assert np.all(bf == 0)  # the membrane step clears the body force everywhere


def test_pressure_codes_need_the_reference_wall_mode():
    b = PS.lattice(1001, 1002)
    nx, ny, nz = b.shape
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB)
    with zf.Context(p) as ctx:
        with pytest.raises(zf.ZfError) as e:
            ctx.set_lattice(b)
        assert "ZF_WALL_REF_EQ" in str(e.value)

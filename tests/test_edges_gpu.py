"""Edge cases of the CUDA path (zebraflow_b200/csrc) through the C ABI: a
lattice without listed points, a coupled run with a mesh but no cells, and a
single 4x4x4 tile periodic along every axis against the fp32 oracle
(oracle/orc_lbm.inc; |df| < 2e-6 as in tests/test_lbm_gpu.py)."""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleLBM

pytestmark = pytest.mark.gpu


def make_ctx(b, **kw):
    nx, ny, nz = b.shape
    kw.setdefault("tau_from_phase", 0)  # the default takes tau from the phase code
    ctx = zf.Context(zf.default_params(nx=nx, ny=ny, nz=nz, **kw))
    ctx.set_lattice(b)
    return ctx


def test_lattice_without_listed_points_steps_as_a_no_op():
    b = -np.ones((8, 8, 8), np.int32)
    ctx = make_ctx(b, wall_mode=zf.WALL_REF_EQ)
    assert ctx.n_listed == 0
    ctx.upload_populations(np.zeros((19, 0), np.float32))
    ctx.lbm_step(store_moments=True, zero_bodyforce=True)
    ctx.lbm_steps(5)
    assert ctx.mass() == 0.0
    assert ctx.step_mass() == 0.0
    assert ctx.download_populations().shape == (19, 0)
    ctx.close()


def test_mesh_without_cells_runs_the_lbm_alone():
    b = zf.gen_tube(24, 24, 32, 11.5, 11.5, 9.0, True)
    kw = dict(tau=0.9, wall_mode=zf.WALL_HALFWAY_BB, periodic=(0, 0, 1), g=(0.0, 0.0, 2e-5),
              area0=0.0, volume0=0.0, stagger=50)
    xyz, tri = zf.gen_icosphere(2)
    xyzn, trin = zf.gen_icosphere(1)
    coupled = make_ctx(b, **kw)
    coupled.set_wall(*zf.gen_wall_tube(11.5, 11.5, 9.0, 32))
    coupled.set_mesh(xyz * 2.0, tri, xyzn, zf.mesh_edges(trin))
    coupled.set_cells(np.zeros((3, 0, xyz.shape[0])), np.zeros((3, 0, xyzn.shape[0])))
    coupled.step(120)  # crosses two membrane iterations
    alone = make_ctx(b, **kw)
    alone.lbm_steps(120)
    fc, fa = coupled.download_populations(), alone.download_populations()
    assert np.abs(fc - zf.W[:, None]).max() > 1e-6  # the force drove a flow
    assert np.max(np.abs(fc - fa)) < 1e-7
    coupled.close()
    alone.close()


def test_single_tile_periodic_box_matches_oracle():
    rng = np.random.default_rng(3)
    b = np.ones((4, 4, 4), np.int32)
    g = (1e-5, -2e-5, 3e-5)
    ctx = make_ctx(b, tau=0.7, wall_mode=zf.WALL_HALFWAY_BB, periodic=(1, 1, 1), g=g)
    o = OracleLBM(b, wall_mode=0, periodic=(1, 1, 1), tau=0.7, g=g, precision="f32")
    f0 = (zf.W[:, None] * (1 + 0.01 * rng.standard_normal((19, 64)))).astype(np.float32)
    bf = (1e-4 * rng.standard_normal((3, 64))).astype(np.float32)
    ctx.upload_populations(f0)
    ctx.upload_bodyforce(bf)
    o.set_f(f0)
    o.set_bodyforce(bf)
    m0 = ctx.mass()
    for _ in range(10):
        ctx.lbm_step(store_moments=True, zero_bodyforce=False)
        o.step()
    assert np.max(np.abs(ctx.download_populations() - o.get_f())) < 2e-6
    assert abs(ctx.mass() - m0) < 1e-6 * m0  # fp32 populations: round-off only
    ctx.close()

"""Exact checkpoints (zf_save_state / zf_load_state).  A run of the coupled
step saved at iteration 120 and loaded into a fresh context holds exactly
the saved state (a second save gives the same bytes), and continued for 130
more iterations (three membrane blocks) it stays within ten times the
run-to-run spread of uninterrupted runs (the largest of two samples: the
spreading's float atomics sum in no fixed order, and a pair of runs can
happen to stay close), for plain fp32 and for fp16 storage with stochastic
rounding (whose
bits are seeded by the restored iteration count).  A context with another
lattice refuses the file."""
import numpy as np
import pytest

import zebraflow_b200 as zf

pytestmark = pytest.mark.gpu

NX, NY, NZ, R, C = 40, 40, 48, 16.0, 19.5


def setup(storage):
    b = zf.gen_tube(NX, NY, NZ, C, C, R, True)
    p = zf.default_params(nx=NX, ny=NY, nz=NZ, tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                          periodic=(0, 0, 1), g=(0, 0, 2e-5), origin=(0.0, 0.0, 0.0), area0=0.0, volume0=0.0,
                          storage=storage)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest, rest_n = xyz * np.array([3.5, 2.25, 1.0]), xyzn * np.array([1.25, 0.9, 0.6])
    cells = zf.gen_cells(b, 4, rest, rest_n, (3.5, 2.25, 1.0), seed=11, margin=0.4)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    ctx.set_wall(*zf.gen_wall_tube(C, C, R, NZ))
    ctx.set_mesh(rest, tri, rest_n, zf.mesh_edges(trin))
    ctx.set_cells(*cells)
    return ctx, cells


def state(ctx):
    x, xn, st = ctx.cells()
    return dict(f=ctx.download_populations(), bf=ctx.download_bodyforce(), mom=np.stack(ctx.download_moments()),
                x=x, xn=xn, st=st, it=ctx.iteration())


@pytest.mark.parametrize("storage", [zf.STORE_F32, zf.STORE_F16])
def test_continued_run_is_the_saved_run(storage, tmp_path):
    s1, s2 = str(tmp_path / "s1.bin"), str(tmp_path / "s2.bin")
    a, cells = setup(storage)
    a.step(120)
    a.save_state(s1)
    a.step(130)
    A = state(a)
    a.close()
    b, _ = setup(storage)
    b.load_state(s1)
    assert b.iteration() == 120
    # everything the checkpoint holds is back: saving again gives the same bytes
    b.save_state(s2)
    assert open(s1, "rb").read() == open(s2, "rb").read()
    b.step(130)
    B = state(b)
    b.close()
    # the same 250 iterations uninterrupted once more: the run-to-run spread
    # that the float atomics of the spreading leave (with fp16 storage their
    # last-bit differences also flip some stochastic roundings)
    spreads = []
    for _ in range(2):
        c, _ = setup(storage)
        c.step(250)
        spreads.append(state(c))
        c.close()
    assert A["it"] == B["it"] == 250
    assert np.array_equal(A["st"], B["st"])
    assert np.abs(A["x"] - cells[0]).max() > 1e-3  # the cells moved
    floor = 1e-6 if storage == zf.STORE_F32 else 1e-5
    for k in ("x", "xn", "f", "mom"):
        # two samples of the spread: one pair of runs can happen to stay close
        spread = max(np.abs(A[k] - A2[k]).max() for A2 in spreads)
        assert np.abs(A[k] - B[k]).max() <= 10 * spread + floor, (k, np.abs(A[k] - B[k]).max(), spread)


def test_other_lattice_refuses_the_file(tmp_path):
    path = str(tmp_path / "state.bin")
    a, _ = setup(zf.STORE_F32)
    a.step(10)
    a.save_state(path)
    a.close()
    b = zf.gen_tube(NX, NY, NZ + 4, C, C, R, True)
    p = zf.default_params(nx=NX, ny=NY, nz=NZ + 4, tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                          periodic=(0, 0, 1))
    with zf.Context(p) as ctx:
        ctx.set_lattice(b)
        with pytest.raises(zf.ZfError) as e:
            ctx.load_state(path)
        assert "another lattice" in str(e.value)


def test_async_cell_copy_holds_the_state_it_was_queued_after():
    """zf_get_cells_async queued after a membrane iteration copies the
    positions and statuses of that moment, although the next cycle (whose
    position update comes at its end) is queued before the copy is waited
    for; zf_set_cells waits for a copy still reading the old buffers."""
    torch = pytest.importorskip("torch")
    ctx, cells = setup(zf.STORE_F32)
    ctx.step(100)
    x_ref, xn_ref, st_ref = ctx.cells()
    hx = torch.empty(x_ref.size, dtype=torch.float64).pin_memory()
    hxn = torch.empty(xn_ref.size, dtype=torch.float64).pin_memory()
    hst = torch.empty(st_ref.size, dtype=torch.int32).pin_memory()
    zf._check(zf.lib().zf_get_cells_async(ctx._h, hx.data_ptr(), hxn.data_ptr(), hst.data_ptr()))
    ctx.step(50)  # queued at once: 49 LBM iterations, then a membrane iteration that moves the nodes
    ctx.wait_cells()
    assert np.array_equal(hx.numpy().reshape(x_ref.shape), x_ref)
    assert np.array_equal(hxn.numpy().reshape(xn_ref.shape), xn_ref)
    assert np.array_equal(hst.numpy(), st_ref)
    x_new, _, _ = ctx.cells()
    assert not np.array_equal(x_new, x_ref)  # the queued cycle did move them
    zf._check(zf.lib().zf_get_cells_async(ctx._h, hx.data_ptr(), hxn.data_ptr(), hst.data_ptr()))
    ctx.set_cells(*cells)  # replaces the buffers the copy reads
    ctx.wait_cells()
    assert np.array_equal(hx.numpy().reshape(x_ref.shape), x_new)
    ctx.close()

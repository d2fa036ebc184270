"""GPU parity of the fused LBM kernel (zebraflow_b200/csrc/zf_lbm.cu) against
the CPU oracle (oracle/orc_lbm.inc) through the C ABI.

Tolerances: the fp32 kernel and the fp32 oracle evaluate the same formulas in
a different order (FMA contraction on the GPU), so populations agree to a few
ulp per step: max |df| <= 2e-6 absolute (populations are O(0.03-0.3)) after
20 steps, density to 1e-6 and velocity to 3e-7 absolute.  The fp16 / bf16 storage forms are
checked against the fp64 oracle with the bounds stated per test.
"""
import numpy as np
import pytest

import zebraflow_b200 as zf
from oracle.bind import OracleLBM

pytestmark = pytest.mark.gpu


def make_ctx(b, wall_mode, tau=0.8, g=(0, 0, 0), storage=zf.STORE_F32, tau_from_phase=0,
             periodic=(0, 0, 1)):
    nx, ny, nz = b.shape
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau=tau, tau_from_phase=tau_from_phase,
                          wall_mode=wall_mode, storage=storage, periodic=periodic, g=g)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    return ctx


def perturbed(n, rng, amp=0.01):
    return (zf.W[:, None] * (1 + amp * rng.standard_normal((19, n)))).astype(np.float32)


def listed_codes(b):
    dom = np.argwhere(b >= 0)
    return b[dom[:, 0], dom[:, 1], dom[:, 2]]


@pytest.mark.parametrize("wall_mode", [zf.WALL_HALFWAY_BB, zf.WALL_REF_EQ])
def test_lbm_parity_fp32(wall_mode):
    rng = np.random.default_rng(10 + wall_mode)
    b = zf.gen_tube(24, 22, 32, 11.3, 10.6, 9.0, True)
    g = (1e-6, -2e-6, 5e-6)
    ctx = make_ctx(b, wall_mode, tau=0.83, g=g)
    o = OracleLBM(b, wall_mode=wall_mode, periodic=(0, 0, 1), tau=0.83, g=g, precision="f32")
    assert ctx.n_listed == o.n
    assert np.array_equal(ctx.domlist(), np.argwhere(b >= 0))
    f0 = perturbed(o.n, rng)
    bf = (1e-4 * rng.standard_normal((3, o.n))).astype(np.float32)
    ctx.upload_populations(f0)
    ctx.upload_bodyforce(bf)
    o.set_f(f0)
    o.set_bodyforce(bf)
    for s in range(20):
        ctx.lbm_step(store_moments=True, zero_bodyforce=(s == 10))
        o.step(rbc_flag=(s == 10))
    codes = listed_codes(b)
    sel = codes > 0 if wall_mode == zf.WALL_HALFWAY_BB else codes >= 0
    fg, fo = ctx.download_populations(), o.get_f()
    assert np.max(np.abs(fg[:, sel] - fo[:, sel])) < 2e-6
    Dg, *ug = ctx.download_moments()
    Do, *uo = o.moments()
    assert np.max(np.abs(Dg[sel] - Do[sel])) <= 1e-6
    # velocities are differences of O(0.05) populations: fp32 absolute bound
    for a, b_ in zip(ug, uo):
        assert np.max(np.abs(a[sel] - b_[sel])) <= 3e-7
    # BODYFORCE was cleared on step 10 at every point the step updates
    assert np.all(ctx.download_bodyforce()[:, sel] == 0)


def test_lbm_matches_reference_output():
    """The CUDA step against the reference's own: tests/golden/ref_step.npz
    holds five steps run by the reference's stream-collide, wall and copy
    blocks of its main() (ZebraflowWT.c:6101-6145, :6292-6433, :6601-6626) on a
    capped tube with a phase-5 ball (fixture script: tests/golden/make_ref_golden.py).
    The reference keeps fp32 populations with double temporaries, the kernel
    fp32 with FMA contraction: a few fp32 ulp per step, |df| < 5e-7 after five
    steps in which the populations move by ~4e-3."""
    import os
    st = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_step.npz"))
    listed = st["listed"]
    lo = listed[:, :3].min(0)
    b = -np.ones(tuple(listed[:, :3].max(0) - lo + 1), np.int32)
    b[tuple((listed[:, :3] - lo).T)] = listed[:, 3]
    ctx = make_ctx(b, zf.WALL_REF_EQ, tau=1.22, tau_from_phase=1, periodic=(0, 0, 0))
    assert np.array_equal(ctx.domlist(), listed[:, :3] - lo)
    ctx.upload_populations(st["f0"])
    ctx.upload_bodyforce(st["bf0"])
    steps = int(st["steps"])
    for s in range(1, steps + 1):
        ctx.lbm_step(store_moments=True, zero_bodyforce=(s == steps))
        if s == 1:
            assert np.max(np.abs(ctx.download_populations() - st["f1"])) < 2e-7
    assert np.max(np.abs(ctx.download_populations() - st["fN"])) < 5e-7
    Dg, Ug, Vg, Wg = ctx.download_moments()
    assert np.max(np.abs(Dg - st["D"])) < 2e-6
    for a, r in zip((Ug, Vg, Wg), (st["U"], st["V"], st["W"])):
        assert np.max(np.abs(a - r)) < 2e-7
    assert np.all(ctx.download_bodyforce() == 0)


def test_lbm_tau_from_phase():
    rng = np.random.default_rng(3)
    b = zf.gen_tube(20, 20, 16, 9.5, 9.5, 8.0, True)
    fl = b > 0
    b[fl] = rng.integers(1, 4, size=int(fl.sum()))  # phases 1..3: tau = 0.5 + 0.72*B
    ctx = make_ctx(b, zf.WALL_REF_EQ, tau_from_phase=1)
    o = OracleLBM(b, wall_mode=1, periodic=(0, 0, 1), tau_from_phase=True, precision="f32")
    f0 = perturbed(o.n, rng)
    ctx.upload_populations(f0)
    o.set_f(f0)
    for _ in range(10):
        ctx.lbm_step()
        o.step()
    assert np.max(np.abs(ctx.download_populations() - o.get_f())) < 2e-6


@pytest.mark.parametrize("storage,bound", [(zf.STORE_F32, 1e-5), (zf.STORE_F32_DEV, 1e-9)])
def test_lbm_mass_conservation_gpu(storage, bound):
    """Relative drift of the FP64 mass sum over 200 bounce-back steps: fp32
    populations round O(0.05) values each step; fp32 deviations round O(1e-3)."""
    rng = np.random.default_rng(4)
    b = zf.gen_tube(32, 32, 64, 15.5, 15.5, 14.0, True)
    ctx = make_ctx(b, zf.WALL_HALFWAY_BB, g=(0, 0, 1e-5), storage=storage)
    ctx.upload_populations(perturbed(ctx.n_listed, rng))
    m0 = ctx.mass()
    ctx.lbm_steps(200)
    m1 = ctx.mass()
    assert abs(m1 - m0) < bound * m0
    # the mass fused into the step kernel (sum of the pre-collision fp32
    # densities) agrees with the separate reduction of the stored populations
    # to fp32 rounding
    import ctypes
    mf = ctypes.c_double()
    zf._check(zf.lib().zf_lbm_step_mass(ctx._h, 0, 0, ctypes.byref(mf)))
    assert abs(mf.value - ctx.mass()) < 1e-7 * m0


def test_lbm_periodic_bifurcation_runs():
    b, _ = zf.gen_bifurcation(64, 48, 128, 8, 6, 20.0)
    ctx = make_ctx(b, zf.WALL_HALFWAY_BB, tau=0.9, g=(0, 0, 1e-5))
    m0 = ctx.mass()
    ctx.lbm_steps(100)
    D, U, V, W = ctx.download_moments()
    fl = listed_codes(b) > 0
    assert np.isfinite(W[fl]).all() and W[fl].mean() > 0
    assert abs(ctx.mass() - m0) < 2e-6 * m0


_POIS = {}


def poiseuille_oracle(steps):
    if steps not in _POIS:
        b = zf.gen_tube(20, 20, 8, 9.5, 9.5, 8.0, True)
        o = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.8, g=(0, 0, 2e-6),
                      precision="f64")
        for _ in range(steps):
            o.step()
        _POIS[steps] = (b, o.moments()[3][listed_codes(b) > 0])
    return _POIS[steps]


def poiseuille_run(storage, steps=3000, stochastic=1):
    b, wo = poiseuille_oracle(steps)
    p = zf.default_params(nx=20, ny=20, nz=8, tau=0.8, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, storage=storage, periodic=(0, 0, 1),
                          g=(0, 0, 2e-6), stochastic_round=stochastic)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    ctx.lbm_steps(steps)
    wg = ctx.download_moments()[3][listed_codes(b) > 0].astype(np.float64)
    return np.linalg.norm(wg - wo) / np.linalg.norm(wo)


# (storage, stochastic rounding, bound on the relative L2 velocity error after
# 3000 steps of Poiseuille flow driven by g = 2e-6, against the fp64 oracle).
# The run has no atomics, so it repeats exactly; the bounds are twice what a
# B200 measured: raw fp32 1.0e-4, fp32 deviation 9.6e-7, fp16 deviation
# 3.7e-4 with stochastic rounding and 2.7e-3 with round-to-nearest, bf16
# deviation 1.7e-3 with stochastic rounding.  (The CPU emulation of each
# storage rounding on the fp64 oracle gives raw fp32 3.3e-4, fp32 deviation
# 3.3e-7, fp16 1.3e-4 / 2.5e-3, bf16 with round-to-nearest 5.7e-2.)
STORAGE_BOUNDS = [
    (zf.STORE_F32, 1, 2.1e-4),
    (zf.STORE_F32_DEV, 1, 2e-6),
    (zf.STORE_F16, 1, 7.4e-4),
    (zf.STORE_F16, 0, 5.4e-3),
    (zf.STORE_BF16, 1, 3.4e-3),
]


@pytest.mark.parametrize("storage,stochastic,bound", STORAGE_BOUNDS)
def test_storage_forms_against_fp64_oracle(storage, stochastic, bound):
    err = poiseuille_run(storage, stochastic=stochastic)
    print(f"storage {storage} stochastic {stochastic}: rel L2 velocity error {err:.3e}")
    assert err < bound


def test_fp16_round_to_nearest_matches_emulated_oracle():
    """fp16 deviation storage with round-to-nearest against the fp32 oracle
    whose stored populations are rounded the same way (5 steps)."""
    rng = np.random.default_rng(12)
    b = zf.gen_tube(20, 20, 16, 9.5, 9.5, 8.0, True)
    p = zf.default_params(nx=20, ny=20, nz=16, tau=0.8, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, storage=zf.STORE_F16,
                          periodic=(0, 0, 1), g=(0, 0, 1e-5), stochastic_round=0)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    o = OracleLBM(b, wall_mode=0, periodic=(0, 0, 1), tau=0.8, g=(0, 0, 1e-5), precision="f32")
    o.set_storage_emulation(3, 65536.0, 1.0)
    f0 = perturbed(o.n, rng, amp=0.002)
    ctx.upload_populations(f0)
    o.set_f(ctx.download_populations())  # the same fp16-rounded start
    for _ in range(5):
        ctx.lbm_step()
        o.step()
    fl = listed_codes(b) > 0
    assert np.max(np.abs(ctx.download_populations()[:, fl] - o.get_f()[:, fl])) < 2e-6


def test_storage_roundtrip_fp16():
    """Upload/download through the deviation codec is exact to fp16 rounding."""
    rng = np.random.default_rng(5)
    b = zf.gen_tube(16, 16, 8, 7.5, 7.5, 6.0, True)
    ctx = make_ctx(b, zf.WALL_HALFWAY_BB, storage=zf.STORE_F16)
    f0 = perturbed(ctx.n_listed, rng, amp=0.001)
    ctx.upload_populations(f0)
    f1 = ctx.download_populations()
    dev = f0 / zf.W[:, None].astype(np.float32) - 1
    err = np.abs(f1 - f0) / zf.W[:, None]
    # fp16 keeps 11 significant bits of the deviation; the fp32 f = w(1+d)
    # of the download adds one rounding of f
    assert np.all(err <= np.abs(dev) * 2 ** -11 + 2e-7)

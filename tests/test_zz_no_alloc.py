"""zf_lbm_step_mass_noalloc, the allocation-free variant of zf_lbm_step_mass.

It exists for callers that cannot call cudaMalloc once their run has
started: code whose device memory belongs to another allocator that has
already reserved the GPU, and time loops that must not take cudaMalloc's
implicit device synchronisation or an out-of-memory failure mid-run.  Its
reduction scratch is a file-scope device array instead of cudaMalloc'd memory.

Checked here through the C ABI: two calls in a row give the same mass and the
same populations as the allocating entry point on an identical context, and a
lattice larger than the fixed scratch is refused with a clear error.  This file
sorts last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

import zebraflow_b200 as zf

pytestmark = pytest.mark.gpu


def make_context(b, rng_seed):
    nx, ny, nz = b.shape
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau=0.85, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, periodic=(0, 0, 1), g=(0, 0, 1e-5))
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    rng = np.random.default_rng(rng_seed)
    f0 = (zf.W[:, None] * (1 + 0.01 * rng.standard_normal((19, ctx.n_listed)))).astype(np.float32)
    bf = (1e-4 * rng.standard_normal((3, ctx.n_listed))).astype(np.float32)
    ctx.upload_populations(f0)
    ctx.upload_bodyforce(bf)
    return ctx


def test_noalloc_matches_allocating_step_twice():
    b = zf.gen_tube(32, 30, 48, 15.2, 14.7, 13.0, True)
    ref = make_context(b, 21)
    new = make_context(b, 21)
    for call in range(2):
        m_ref, m_new = ctypes.c_double(), ctypes.c_double()
        zf._check(zf.lib().zf_lbm_step_mass(ref._h, 0, 0, ctypes.byref(m_ref)))
        zf._check(zf.lib().zf_lbm_step_mass_noalloc(new._h, 0, 0, ctypes.byref(m_new)))
        # the same step kernel on the same inputs: the sums agree to fp64 rounding
        assert abs(m_new.value - m_ref.value) <= 1e-12 * abs(m_ref.value), call
        assert m_new.value > 0
        # and the populations the step wrote agree within the fp32 parity bound
        assert np.max(np.abs(new.download_populations() - ref.download_populations())) < 2e-6
    ref.close()
    new.close()


def test_noalloc_refuses_lattice_beyond_its_scratch():
    # 64 x 64 x 65 tiles with fluid = 66,560 blocks of four tiles > 65,536
    b = np.ones((256, 256, 260), np.int32)
    p = zf.default_params(nx=256, ny=256, nz=260, tau=0.9, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, periodic=(1, 1, 1))
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    m = ctypes.c_double()
    rc = zf.lib().zf_lbm_step_mass_noalloc(ctx._h, 0, 0, ctypes.byref(m))
    assert rc == zf.ZF_ERR_ARG
    assert b"allocation-free" in zf.lib().zf_last_error()
    ctx.close()

"""zf_lbm_step_mass_noalloc, the allocation-free variant of zf_lbm_step_mass.

It exists for callers that cannot call cudaMalloc once their run has
started: code whose device memory belongs to another allocator that has
already reserved the GPU, and time loops that must not take cudaMalloc's
implicit device synchronisation or an out-of-memory failure mid-run.  Its
reduction scratch is a file-scope device array instead of cudaMalloc'd memory.

Checked here through the C ABI, for every population storage form and with
and without the moments written: two calls in a row give the same mass,
populations and moments as the allocating entry point on an identical
context; the mass equals an FP64 sum of the densities of the populations
downloaded before each call; neither the context's device memory nor the
GPU's free memory changes across the calls; and a lattice larger than the
fixed scratch is refused with a clear error.  This file sorts last so that a
run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

import zebraflow_b200 as zf

pytestmark = pytest.mark.gpu

STORAGES = {"f32": zf.STORE_F32, "f16": zf.STORE_F16, "bf16": zf.STORE_BF16, "f32dev": zf.STORE_F32_DEV}


def make_context(b, rng_seed, storage):
    nx, ny, nz = b.shape
    p = zf.default_params(nx=nx, ny=ny, nz=nz, tau=0.85, tau_from_phase=0,
                          wall_mode=zf.WALL_HALFWAY_BB, periodic=(0, 0, 1), g=(0, 0, 1e-5),
                          storage=storage)
    ctx = zf.Context(p)
    ctx.set_lattice(b)
    rng = np.random.default_rng(rng_seed)
    f0 = (zf.W[:, None] * (1 + 0.01 * rng.standard_normal((19, ctx.n_listed)))).astype(np.float32)
    bf = (1e-4 * rng.standard_normal((3, ctx.n_listed))).astype(np.float32)
    ctx.upload_populations(f0)
    ctx.upload_bodyforce(bf)
    return ctx


@pytest.mark.parametrize("store_moments", [0, 1])
@pytest.mark.parametrize("storage", sorted(STORAGES))
def test_noalloc_matches_allocating_step_twice(storage, store_moments):
    import torch
    b = zf.gen_tube(32, 30, 48, 15.2, 14.7, 13.0, True)
    ref = make_context(b, 21, STORAGES[storage])
    new = make_context(b, 21, STORAGES[storage])
    dom = new.domlist()
    fluid = b[dom[:, 0], dom[:, 1], dom[:, 2]] > 0
    L = zf.lib()
    # the allocating entry sizes its scratch on its first call: make that call
    # on both contexts before memory is compared
    m_ref, m_new = ctypes.c_double(), ctypes.c_double()
    zf._check(L.zf_lbm_step_mass(ref._h, store_moments, 0, ctypes.byref(m_ref)))
    zf._check(L.zf_lbm_step_mass_noalloc(new._h, store_moments, 0, ctypes.byref(m_new)))
    # the download kernels' first launches too, so that the driver loading
    # their code cannot fall between the two free-memory readings
    for ctx in (ref, new):
        ctx.download_populations()
        ctx.download_moments()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    ctx_bytes0 = new.device_bytes()
    for call in range(2):
        f_before = new.download_populations().astype(np.float64)
        zf._check(L.zf_lbm_step_mass(ref._h, store_moments, 0, ctypes.byref(m_ref)))
        zf._check(L.zf_lbm_step_mass_noalloc(new._h, store_moments, 0, ctypes.byref(m_new)))
        # the same step kernel on the same inputs: the sums agree to fp64 rounding
        assert abs(m_new.value - m_ref.value) <= 1e-12 * abs(m_ref.value), call
        # and the sum is the FP64 total of the pre-step densities (each formed
        # in fp32 inside the kernel, hence the fp32-rounding tolerance)
        direct = float(f_before[:, fluid].sum())
        assert abs(m_new.value - direct) <= 1e-6 * direct, (call, m_new.value, direct)
        # the populations (and moments) the step wrote agree within the fp32 parity bound
        assert np.max(np.abs(new.download_populations() - ref.download_populations())) < 2e-6
        if store_moments:
            for a, r in zip(new.download_moments(), ref.download_moments()):
                assert np.max(np.abs(a[fluid] - r[fluid])) < 2e-6
    torch.cuda.synchronize()
    assert new.device_bytes() == ctx_bytes0
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    ref.close()
    new.close()


def test_noalloc_counts_its_launches():
    b = zf.gen_tube(24, 24, 16, 11.5, 11.5, 9.0, True)
    ctx = make_context(b, 5, zf.STORE_F32)
    n0 = ctx.launch_count()
    m = ctypes.c_double()
    zf._check(zf.lib().zf_lbm_step_mass_noalloc(ctx._h, 0, 0, ctypes.byref(m)))
    assert ctx.launch_count() - n0 == 2  # the step kernel and the sum (no wall pass in bounce-back mode)
    ctx.close()


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

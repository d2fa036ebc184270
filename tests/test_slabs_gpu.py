"""The z-slab decomposition of the LBM step (zebraflow_b200/slabs.py,
zf_plane_pack / zf_plane_unpack) on one GPU: the lattice cut into two slabs,
each with its halo tile layers, stepped side by side with the halo exchange
after every step (in-process, exchange_local), must reproduce the populations
of the unsplit lattice bit for bit at every interior point.  Two slabs of one
process stand for two ranks; no kernel waits on another."""
import numpy as np
import pytest
import torch

import zebraflow_b200 as zf
from zebraflow_b200 import slabs

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 64


@pytest.mark.parametrize("storage,sr", [(zf.STORE_F32, 1), (zf.STORE_F32_DEV, 1), (zf.STORE_F16, 0)])
def test_two_slabs_match_the_whole_lattice(storage, sr):
    b, _ = zf.gen_bifurcation(NX, NY, NZ, 6.0, 5.0, 20.0)
    kw = dict(tau=0.8, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB, g=(0.0, 0.0, 2e-5),
              storage=storage, stochastic_round=sr)
    full = zf.Context(zf.default_params(nx=NX, ny=NY, nz=NZ, periodic=(0, 0, 1), **kw))
    full.set_lattice(b)
    dom = full.domlist()
    index = {tuple(p): l for l, p in enumerate(dom.tolist())}
    rng = np.random.default_rng(1)
    f0 = full.download_populations()
    f0 = (f0 * (1.0 + 1e-3 * rng.standard_normal(f0.shape))).astype(np.float32)  # a state with gradients
    full.upload_populations(f0)
    stream = torch.cuda.Stream()
    parts = [slabs.SlabLBM(b, world=2, rank=r, stream=stream, **kw) for r in range(2)]
    gls = []
    for s in parts:
        sdom = s.ctx.domlist()
        gz = (s.z0 + sdom[:, 2] - slabs.HALO) % NZ
        gl = np.array([index[(i, j, k)] for (i, j), k in zip(sdom[:, :2].tolist(), gz.tolist())])
        s.ctx.upload_populations(f0[:, gl])
        gls.append(gl)
    slabs.exchange_local(parts)
    for _ in range(40):
        full.lbm_step(store_moments=False, zero_bodyforce=False)
        for s in parts:
            s.ctx.lbm_step(store_moments=False, zero_bodyforce=False)
        slabs.exchange_local(parts)
    ff = full.download_populations()
    for s, gl in zip(parts, gls):
        fs = s.ctx.download_populations()
        inner, _ = s.interior()
        assert inner.sum() > 1000
        assert np.array_equal(fs[:, inner], ff[:, gl[inner]])
        s.close()
    # the flow moved: the state is not the initial one
    assert np.abs(ff - f0).max() > 1e-6
    full.close()


def _setup(storage, sr, world):
    b, _ = zf.gen_bifurcation(NX, NY, NZ, 6.0, 5.0, 20.0)
    kw = dict(tau=0.8, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB, g=(0.0, 0.0, 2e-5),
              storage=storage, stochastic_round=sr)
    full = zf.Context(zf.default_params(nx=NX, ny=NY, nz=NZ, periodic=(0, 0, 1), **kw))
    full.set_lattice(b)
    index = {tuple(p): l for l, p in enumerate(full.domlist().tolist())}
    rng = np.random.default_rng(2)
    f0 = full.download_populations()
    f0 = (f0 * (1.0 + 1e-3 * rng.standard_normal(f0.shape))).astype(np.float32)
    full.upload_populations(f0)
    stream = torch.cuda.Stream()
    parts = [slabs.SlabLBM(b, world=world, rank=r, stream=stream, **kw) for r in range(world)]
    gls = []
    for s in parts:
        sdom = s.ctx.domlist()
        gz = (s.z0 + sdom[:, 2] - slabs.HALO) % NZ
        gl = np.array([index[(i, j, k)] for (i, j), k in zip(sdom[:, :2].tolist(), gz.tolist())])
        s.ctx.upload_populations(f0[:, gl])
        gls.append(gl)
    return full, parts, gls, f0


def _check(full, parts, gls, f0):
    ff = full.download_populations()
    for s, gl in zip(parts, gls):
        fs = s.ctx.download_populations()
        inner, _ = s.interior()
        assert inner.sum() > 1000
        assert np.array_equal(fs[:, inner], ff[:, gl[inner]])
        s.close()
    assert np.abs(ff - f0).max() > 1e-6
    full.close()


@pytest.mark.parametrize("storage,sr", [(zf.STORE_F32, 1), (zf.STORE_F16, 0)])
def test_two_slabs_stepped_in_parts_match_the_whole_lattice(storage, sr):
    """Each step as the overlapped slab step runs it: the inner tile layers,
    then (halos filled) the two face layers; the halo layers are not stepped."""
    full, parts, gls, f0 = _setup(storage, sr, 2)
    for _ in range(40):
        full.lbm_step(store_moments=False, zero_bodyforce=False)
        slabs.exchange_local(parts)  # halos of the current state
        for s in parts:
            s.ctx.lbm_step_part(0, False)
            s.ctx.lbm_step_part(1, True)
    _check(full, parts, gls, f0)


def test_one_slab_exchanging_with_itself_matches_the_whole_lattice():
    """SlabLBM.step on one rank: pack, inner layers, unpack, face layers."""
    full, parts, gls, f0 = _setup(zf.STORE_F32, 1, 1)
    for _ in range(40):
        full.lbm_step(store_moments=False, zero_bodyforce=False)
    parts[0].step(40)
    torch.cuda.synchronize()
    _check(full, parts, gls, f0)


def test_slab_parts_need_whole_tile_layers():
    full, parts, gls, f0 = _setup(zf.STORE_F32, 1, 1)
    with pytest.raises(zf.ZfError):
        parts[0].ctx.set_slab(slabs.HALO + 1, parts[0].nzs - slabs.HALO)
    for s in parts:
        s.close()
    full.close()

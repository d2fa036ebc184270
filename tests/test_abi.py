"""The C ABI library loads and exports every symbol include/zf.h declares;
the ctypes mirror matches the struct layout; generators produce reference
B_index codes.  No compute call needs a GPU here."""
import ctypes
import os
import re

import numpy as np
import pytest

import zebraflow_b200 as zf
from conftest import ROOT, has_gpu


def declared_functions():
    src = open(os.path.join(ROOT, "include", "zf.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(zf_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(zf.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_layout_and_defaults():
    p = zf.default_params()
    assert zf.lib().zf_params_size() == ctypes.sizeof(zf.Params)
    # reference constants, ZebraflowWT.c:34-161
    assert (p.nx, p.ny, p.nz) == (249, 547, 723)
    assert p.dx == 0.5 and p.dt == 0.5 and p.stagger == 50
    assert abs(p.tau - 1.22) < 1e-6
    assert abs(p.unit_mass - 1.25e-15) < 1e-27
    assert abs(p.bforce_scale - 2e6 / 3) < 1e-6
    assert p.wall_mode == zf.WALL_REF_EQ


def test_ctypes_mirror_signatures_cover_header():
    # the generators and parameter defaults are bound by zf.Inputs under a prefix
    mirrored = set(zf._SIGS) | {"zf_" + n for n in zf._GEN_SIGS}
    assert set(declared_functions()) <= mirrored


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_create_without_device_fails_cleanly():
    with pytest.raises(zf.ZfError) as e:
        zf.Context(zf.default_params(nx=8, ny=8, nz=8))
    assert "device" in str(e.value).lower()


def test_gen_tube_codes():
    b = zf.gen_tube(20, 20, 8, 9.5, 9.5, 6.0, True)
    i, j = np.meshgrid(np.arange(20), np.arange(20), indexing="ij")
    inside = (i - 9.5) ** 2 + (j - 9.5) ** 2 < 36
    assert np.array_equal(b[:, :, 0] > 0, inside)
    assert np.all(b[:, :, 0] == b[:, :, 5])
    # every wall point is linked to a fluid point, no solid point is
    fl = b > 0
    nb = np.zeros_like(fl)
    for e in zf.E[:18]:
        nb |= np.roll(fl, shift=(-e[0], -e[1], -e[2]), axis=(0, 1, 2))
    assert np.array_equal(b == 0, nb & ~fl)


def test_gen_bifurcation_periodic_and_size():
    b, layout = zf.gen_bifurcation(96, 64, 256, 10, 7, 20.0)
    nf = int((b > 0).sum())
    # parent and daughter cross-sections bound the fluid volume
    assert 256 * np.pi * 49 * 1.5 < nf < 256 * np.pi * 100 * 2
    # periodic in z: the first and last slices are both parent slices
    assert np.array_equal(b[:, :, 0] > 0, b[:, :, -1] > 0)
    # two daughters at the middle slice
    mid = b[:, 32, 128] > 0
    runs = np.diff(np.concatenate([[0], mid.astype(int), [0]]))
    assert (runs == 1).sum() == 2
    z1, z2, z3, z4, D, _ = layout
    assert 0 < z1 < z2 < z3 < z4 < 256 and D > 0

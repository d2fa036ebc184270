"""The workload inputs of the two bench arms.  The GPU library (libzf.so,
zf_*) and the CPU library (oracle/liboracle.so, orc_*) compile the same
generator source; these tests hold the two builds to byte-identical outputs,
and check that the reference arm of bench.py builds its inputs without loading
the GPU library."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import zebraflow_b200 as zf  # noqa: E402
from oracle.bind import inputs as oracle_inputs  # noqa: E402


@pytest.fixture(scope="module")
def both():
    return zf.inputs(), oracle_inputs()


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()


def test_params_default_identical(both):
    g, o = both
    assert bytes(g.default_params()) == bytes(o.default_params())
    kw = dict(nx=30, ny=20, nz=40, tau=0.9, storage=1, g=(0.0, 0.0, 1e-6))
    assert bytes(g.default_params(**kw)) == bytes(o.default_params(**kw))


def test_lattice_generators_identical(both):
    g, o = both
    assert _same(g.gen_tube(24, 22, 16, 11.5, 10.5, 9.0, True), o.gen_tube(24, 22, 16, 11.5, 10.5, 9.0, True))
    bg, lg = g.gen_bifurcation(64, 48, 128, 10.0, 7.0, 20.0)
    bo, lo = o.gen_bifurcation(64, 48, 128, 10.0, 7.0, 20.0)
    assert _same(bg, bo) and lg == lo


def test_mesh_and_wall_generators_identical(both):
    g, o = both
    for level in (2, 3):
        for a, b in zip(g.gen_icosphere(level), o.gen_icosphere(level)):
            assert _same(a, b)
    for a, b in zip(g.gen_wall_tube(11.5, 11.5, 9.0, 16), o.gen_wall_tube(11.5, 11.5, 9.0, 16)):
        assert _same(a, b)
    wg = g.gen_wall_bifurcation(64, 48, 96, 10.0, 7.0, 20.0, dx=0.5)
    wo = o.gen_wall_bifurcation(64, 48, 96, 10.0, 7.0, 20.0, dx=0.5)
    assert wg[1].shape[1] > 1000
    for a, b in zip(wg, wo):
        assert _same(a, b)


def test_cell_placement_identical(both):
    g, o = both
    b, _ = g.gen_bifurcation(64, 48, 128, 10.0, 7.0, 20.0)
    xyz, _ = g.gen_icosphere(3)
    xyzn, _ = g.gen_icosphere(2)
    axes = (3.5, 2.25, 1.0)
    rest, rest_n = xyz * np.array(axes), xyzn * np.array([1.25, 0.9, 0.6])
    xg, xng = g.gen_cells(b, 12, rest, rest_n, axes, seed=2024, dx=0.5, margin=0.4)
    xo, xno = o.gen_cells(b, 12, rest, rest_n, axes, seed=2024, dx=0.5, margin=0.4)
    assert xg.shape[1] >= 8
    assert _same(xg, xo) and _same(xng, xno)


def test_reference_arm_does_not_load_the_gpu_library():
    code = (
        "import sys, io, contextlib\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', "
        "'bifurcation_small_128x96x256_60rbc', '--cells', '4', '--steps', '1', '--warmup', '1', "
        "'--reference-seconds', '1']\n"
        "import bench\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LINE', buf.getvalue().strip())\n"
        "print('LIBZF', 'libzf.so' in maps, 'LIBORACLE', 'liboracle.so' in maps)\n"
    )
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900,
                         env=dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4")))
    assert out.returncode == 0, out.stderr[-2000:]
    assert "LIBZF False LIBORACLE True" in out.stdout
    import json
    line = json.loads(out.stdout.split("LINE", 1)[1].split("\n", 1)[0])
    assert line["impl"] == "reference" and line["value"] > 0
    assert "parallelism" not in line["config"]

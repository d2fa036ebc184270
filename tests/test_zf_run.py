"""The C host driver zf_run (zebraflow_b200/csrc/zf_run.c), the reference's
main() time loop (ZebraflowWT.c:5646-12412) written as a C program against
include/zf.h: it links against libzf.so and runs; on a GPU its final node
positions, cell status, wall shear stress and fluid moments match the same
inputs stepped through the Python mirror of the C ABI."""
import os
import subprocess

import numpy as np
import pytest

import zebraflow_b200 as zf
from conftest import ROOT, has_gpu

EXE = os.path.join(ROOT, "zebraflow_b200", "zf_run")


def test_driver_is_built_and_linked():
    assert os.path.exists(EXE), "build with make -C zebraflow_b200/csrc"
    out = subprocess.run(["ldd", EXE], capture_output=True, text=True)
    assert "libzf.so" in out.stdout and "not found" not in out.stdout
    bad = subprocess.run([EXE, "--storage", "f8"], capture_output=True, text=True)
    assert bad.returncode == 2 and "usage" in bad.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_driver_fails_cleanly_without_a_device():
    out = subprocess.run([EXE, "--steps", "1"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 1 and "zf_create" in out.stderr


def read_dump(path):
    raw = open(path, "rb").read()
    assert raw[:8] == b"ZFRUN001"
    nc, nn, nnn, nw = np.frombuffer(raw, np.int32, 4, 8)
    it, nl = np.frombuffer(raw, np.int64, 2, 24)
    o = 40
    x = np.frombuffer(raw, np.float64, 3 * nc * nn, o).reshape(3, nc, nn)
    o += x.nbytes
    xn = np.frombuffer(raw, np.float64, 3 * nc * nnn, o).reshape(3, nc, nnn)
    o += xn.nbytes
    st = np.frombuffer(raw, np.int32, nc, o)
    o += st.nbytes
    wss = np.frombuffer(raw, np.float32, 3 * nw, o).reshape(3, nw)
    o += wss.nbytes
    mom = np.frombuffer(raw, np.float32, 4 * nl, o).reshape(4, nl)
    assert o + mom.nbytes == len(raw)
    return dict(iter=int(it), x=x, xn=xn, status=st, wss=wss, mom=mom)


@pytest.mark.gpu
def test_driver_matches_the_python_path(tmp_path):
    steps, stagger = 200, 50
    dump = str(tmp_path / "run.bin")
    out = subprocess.run([EXE, "--steps", str(steps), "--stagger", str(stagger), "--out", dump],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert "membrane blocks" in out.stdout
    d = read_dump(dump)
    assert d["iter"] == steps and d["x"].shape[1] == 8

    # the same workload through the ctypes mirror: 48x48x128 tube, R = 20, 8 cells
    b = zf.gen_tube(48, 48, 128, 23.5, 23.5, 20.0, True)
    p = zf.default_params(nx=48, ny=48, nz=128, tau=0.9, tau_from_phase=0, wall_mode=zf.WALL_HALFWAY_BB,
                          periodic=(0, 0, 1), g=(0.0, 0.0, 1e-6), origin=(0.0, 0.0, 0.0), dx=0.5,
                          stagger=stagger, area0=0.0, volume0=0.0)
    xyz, tri = zf.gen_icosphere(3)
    xyzn, trin = zf.gen_icosphere(2)
    rest, rest_n = xyz * np.array([3.5, 2.25, 1.0]), xyzn * np.array([1.25, 0.9, 0.6])
    x0, xn0 = zf.gen_cells(b, 8, rest, rest_n, (3.5, 2.25, 1.0), seed=1234, dx=0.5, margin=0.4)
    with zf.Context(p) as ctx:
        ctx.set_lattice(b)
        ctx.set_wall(*zf.gen_wall_tube(23.5, 23.5, 20.0, 128))
        ctx.set_mesh(rest, tri, rest_n, zf.mesh_edges(trin))
        ctx.set_cells(x0, xn0)
        for _ in range(steps // stagger):
            ctx.step(stagger)
        x, xn, st = ctx.cells()
        wss = ctx.wss()[0]
        mom = np.stack(ctx.download_moments())
    # the cells moved, and both paths moved them alike (float atomics of the
    # spreading differ in order between runs, which shows in the fourth
    # membrane block's WSS at ~2e-5 of its largest value)
    assert np.abs(x - x0).max() > 1e-3
    assert np.abs(d["x"] - x).max() < 1e-6 and np.abs(d["xn"] - xn).max() < 1e-6
    assert np.array_equal(d["status"], st)
    assert np.abs(d["wss"] - wss).max() <= 2e-4 * np.abs(wss).max()
    assert np.abs(d["mom"] - mom).max() < 1e-6


@pytest.mark.gpu
def test_driver_writes_reference_files_and_restarts_exactly(tmp_path):
    out_dir = tmp_path / "SimulationOutputData"
    out_dir.mkdir()
    full, half, cont = (str(tmp_path / n) for n in ("full.bin", "half.bin", "cont.bin"))
    state = str(tmp_path / "state.bin")
    r = subprocess.run([EXE, "--steps", "100", "--output-every", "50", "--output-dir", str(out_dir), "--out", half,
                        "--save-state", state], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    names = sorted(os.listdir(out_dir))
    for it in (0, 50, 100):
        for stem, ext in (("FLUIDdomain", "csv"), ("AllCellMemb", "csv"), ("AllCellNucleus", "csv"),
                          ("AllNucEdgeMesh", "csv"), ("Wallpressure", "vtk")):
            assert f"{stem}-{it:09d}.{ext}" in names
    assert "VolumeAreaHistory.dat" in names
    d = read_dump(half)
    # the last snapshot holds the dumped state, to its printed digits
    b = zf.gen_tube(48, 48, 128, 23.5, 23.5, 20.0, True)
    D, U, V, W, bf, en, wi, rows = zf.read_fluid_csv(str(out_dir / "FLUIDdomain-000000100.csv"), b)
    assert rows == int((b >= 0).sum())
    # (the snapshot's moments are recomputed from the populations; velocities
    # carry the fp32 rounding of momentum sums of O(0.05) populations)
    assert np.all(np.abs(D - d["mom"][0]) <= 3e-7 * np.abs(d["mom"][0]))
    for a, ref in ((U, d["mom"][1]), (V, d["mom"][2]), (W, d["mom"][3])):
        assert np.all(np.abs(a - ref) <= 1.2e-7 * np.abs(ref) + 5e-8)
    assert en.sum() > 0 and (wi > 0).sum() > 0  # cell-list counts and wall indices are filled
    cid, st, x, vel, ft = zf.read_cells_csv(str(out_dir / "AllCellMemb-000000100.csv"), 642)
    assert np.array_equal(cid, np.arange(1, 9)) and np.abs(x - d["x"]).max() < 5e-6
    hist = open(out_dir / "VolumeAreaHistory.dat").read().splitlines()
    assert hist[0].startswith("Iteration#") and len(hist) == 1 + 3 * 8
    # continuing from the checkpoint is the uninterrupted run, within the
    # spread of two uninterrupted runs (the spreading's atomics sum in no
    # fixed order)
    full2 = str(tmp_path / "full2.bin")
    for args in (["--load-state", state, "--out", cont], ["--out", full], ["--out", full2]):
        r = subprocess.run([EXE, "--steps", "200" if "--load-state" not in args else "100"] + args,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    a, c, a2 = read_dump(full), read_dump(cont), read_dump(full2)
    assert a["iter"] == c["iter"] == 200
    assert np.array_equal(a["status"], c["status"])
    for k, floor in (("x", 1e-6), ("mom", 1e-6)):
        spread = np.abs(a[k] - a2[k]).max()
        assert np.abs(a[k] - c[k]).max() <= 10 * spread + floor, (k, spread)

"""Builds the fixtures tests/golden/ref_*.npz from the reference's own code.

Runs oracle/ref/Makefile, which compiles the reference's ZebraflowWT.c where
it lies (main renamed) and runs two harnesses against it:
 * oracle/ref/harness_setup.c: CGSM_ZFISHRBC_DATA_GEN /
   CGSM_FILAMENT_PARAMETERS / CGSM_EQUILIBRIUM_METRICS on the shipped RBC and
   nucleus meshes, and LBM_DOM_SETUP / LBM_BC_SETUP on a small synthetic
   lattice -> ref_setup.npz;
 * oracle/ref/harness_cells.c: one membrane step of the reference's own
   force blocks of main() (CGSM_NODAL_FORCE_ZERO, CGSM_AREA, centroid/area,
   CGSM_LOCAL_FORCES, CGSM_VOLUME_CALC; ZebraflowWT.c:5706-7535) for two
   deformed RBCs with nuclei -> ref_cells.npz (node coordinates, node forces,
   triangle geometry, per-cell area/volume/centroid/global-area/volume terms);
 * oracle/ref/harness_ib.c: one membrane iteration of the reference's own
   blocks of main() (forces, IB interpolation + wall repulsion, nucleus-
   membrane and RBC-RBC repulsion, IB spreading, position update;
   ZebraflowWT.c:5659-12189) on the scene of tests/golden/ib_scene.py ->
   ref_ib.npz (cell coordinates, scene checksums, the state after each stage);
 * the unmodified post-processor PostProWSSandPressure.c, run on input files
   written here (the cylinder wall mesh and node normals of
   tests/golden/ib_scene.py, and a FLUIDdomain csv of its lattice with a
   pressurised swirling flow) -> ref_wss.npz (wall pressure, WSS and validity
   of every wall node, as the post-processor prints them);
 * oracle/ref/harness_output.c: the reference's OUTPUT() writer on a small
   lattice and two cells with seeded values -> ref_output.npz (the inputs and
   the bytes of the fluid, membrane, nucleus, nucleus-edge and volume/area
   files it writes);
 * oracle/ref/harness_step.c in its pressure mode: the same blocks with
   pressure inlet/outlet layers of the reference's waveform codes at both
   ends of the tube (tests/golden/pressure_scene.py) -> ref_pressure.npz;
 * oracle/ref/harness_step.c: five LBM steps of the reference's own
   stream-collide, wall and copy blocks of main() (ZebraflowWT.c:6101-6145,
   :6292-6433, :6601-6626) on a small capped tube with a phase-5 ball ->
   ref_step.npz (lattice, initial populations and body force, populations
   after steps 1 and 5, moments and body force after step 5).
The fixtures keep the inputs and the reference's outputs so that the pins run
where the reference tree is absent.

Usage: python tests/golden/make_ref_golden.py [reference_dir [output_dir]]
(output_dir defaults to tests/golden; tests/test_oracle_ref_pin.py regenerates
the fixtures into a scratch folder and compares them with the committed ones)
"""
import gzip
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = HERE  # where the fixtures go (second argument)
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]  # the package, the oracle, tests/golden


def read_mesh(ref):
    def rd(name, conv):
        lines = gzip.open(os.path.join(ref, name), "rt").read().split("\n")[1:]
        return np.array([conv(v) for ln in lines for v in ln.split()])
    X = rd("ZFISHRBCNODES.dat.gz", float).reshape(-1, 3)
    T = rd("ZFISHRBCTRIANGLES.dat.gz", int).reshape(-1, 3).astype(np.int32)
    XN = rd("NucleusNodes.dat.gz", float).reshape(-1, 3)
    EN = rd("NucleusEdges.dat.gz", int).reshape(-1, 2).astype(np.int32)
    return X, T, XN, EN


def main():
    global OUT
    from oracle.refsrc import reference_dir
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_dir()
    if len(sys.argv) > 2:
        OUT = sys.argv[2]
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), f"REF={ref}"], check=True)
    raw = open(os.path.join(ROOT, "oracle", "_ref", "ref_setup.bin"), "rb").read()
    a = np.frombuffer(raw, np.int32)
    f = np.frombuffer(raw, np.float32)
    p = 0
    ne = int(a[p]); p += 1
    edges = a[p:p + 6 * ne].reshape(ne, 6).copy(); p += 6 * ne
    epar = f[p:p + 5 * ne].reshape(5, ne).copy(); p += 5 * ne
    nen = int(a[p]); p += 1
    epar_n = f[p:p + 3 * nen].reshape(3, nen).copy(); p += 3 * nen
    dommax = int(a[p]); p += 1
    domlist = a[p:p + 3 * dommax].reshape(dommax, 3).copy(); p += 3 * dommax
    bcmax = int(a[p]); p += 1
    bc = a[p:p + 7 * bcmax].reshape(bcmax, 7).copy(); p += 7 * bcmax
    assert p == a.size
    X, T, XN, EN = read_mesh(ref)
    np.savez_compressed(os.path.join(OUT, "ref_setup.npz"), mesh_x=X, mesh_tri=T, nuc_x=XN,
                        nuc_edges=EN, edges=edges, epar=epar, epar_n=epar_n, domlist=domlist,
                        bclist=bc[:, :4], bcnlist=bc[:, 4:])
    print(f"edges {ne}, nucleus edges {nen}, listed points {dommax}, boundary points {bcmax}")

    raw = open(os.path.join(ROOT, "oracle", "_ref", "ref_step.bin"), "rb").read()
    a = np.frombuffer(raw, np.int32)
    f = np.frombuffer(raw, np.float32)
    n, steps = int(a[0]), int(a[1])
    p = 2
    listed = a[p:p + 4 * n].reshape(n, 4).copy(); p += 4 * n
    out = {}
    for key, k in (("f0", 19), ("bf0", 3), ("f1", 19), ("fN", 19), ("D", 1), ("U", 1), ("V", 1),
                   ("W", 1), ("bfN", 3)):
        out[key] = f[p:p + k * n].reshape(k, n).copy().squeeze(); p += k * n
    assert p == a.size
    np.savez_compressed(os.path.join(OUT, "ref_step.npz"), listed=listed, steps=steps, **out)
    print(f"LBM step: {n} listed points, {steps} steps")

    raw = open(os.path.join(ROOT, "oracle", "_ref", "ref_cells.bin"), "rb").read()
    pos = [0]

    def rd(dt, k):
        r = np.frombuffer(raw, dt, k, pos[0]).copy()
        pos[0] += r.itemsize * k
        return r
    nc, nn, nnn, nt = rd(np.int32, 4)
    area_eq = rd(np.float32, nt)
    keys = (("x", np.float64, 3 * nn), ("xn", np.float64, 3 * nnn), ("ftot", np.float32, 3 * nn),
            ("ftot_n", np.float32, 3 * nnn), ("tri_area", np.float32, nt),
            ("tri_normal", np.float32, 3 * nt), ("tri_centroid", np.float32, 3 * nt),
            ("node_normal", np.float32, 3 * nn), ("cell", np.float32, 7), ("status", np.int32, 2))
    per = {k: [] for k, _, _ in keys}
    for _ in range(nc):
        for k, dt, m in keys:
            per[k].append(rd(dt, m))
    simfailure = int(rd(np.int32, 1)[0])
    assert pos[0] == len(raw)
    out = {}
    for k, _, m in keys:
        a = np.stack(per[k])                       # [cell][...]
        if m % 3 == 0 and k not in ("tri_area",):  # [cell][3][n] -> [3][cell][n]
            a = a.reshape(nc, 3, -1).transpose(1, 0, 2)
        out[k] = a
    np.savez_compressed(os.path.join(OUT, "ref_cells.npz"), tri_area_eq=area_eq,
                        simfailure=simfailure, **out)
    print(f"membrane step: {nc} cells, simfailure {simfailure}")
    ib_fixture()
    ib_fixture(nucleus=True)
    loop_fixture()
    wss_fixture()
    output_fixture()
    pressure_fixture()


def pressure_fixture():
    """The reference's own LBM blocks (oracle/ref/harness_step.c, pressure
    mode) with pressure inlet/outlet layers at both ends of the tube, for the
    runs of tests/golden/pressure_scene.py: the lattice and initial state are
    rebuilt from the scene (checked here against what the harness used), so
    the fixture keeps the reference's moments after the last step and the
    populations of the boundary points (walls and inlets)."""
    from golden import pressure_scene as PS
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_step")
    out = {"runs": np.array(PS.RUNS, np.int64)}
    for r, (lo, hi, it0) in enumerate(PS.RUNS):
        path = os.path.join(ROOT, "oracle", "_ref", "ref_pressure.bin")
        subprocess.run([exe, path, "pressure", str(lo), str(hi), str(it0)], check=True, stdout=subprocess.DEVNULL)
        raw = open(path, "rb").read()
        a = np.frombuffer(raw, np.int32)
        f = np.frombuffer(raw, np.float32)
        n, steps, it = int(a[0]), int(a[1]), int(a[2])
        assert steps == PS.STEPS and it == it0
        p = 3
        listed = a[p:p + 4 * n].reshape(n, 4).copy(); p += 4 * n
        arr = {}
        for key, k in (("f0", 19), ("bf0", 3), ("f1", 19), ("fN", 19), ("D", 1), ("U", 1), ("V", 1), ("W", 1),
                       ("bfN", 3)):
            arr[key] = f[p:p + k * n].reshape(k, n).copy().squeeze(); p += k * n
        assert p == a.size
        b = PS.lattice(lo, hi)
        dom = np.argwhere(b >= 0)
        assert np.array_equal(listed[:, :3] - np.array(PS.BOX_LO), dom)
        assert np.array_equal(listed[:, 3], b[tuple(dom.T)])
        f0, bf0 = PS.initial_state(n)
        assert np.array_equal(f0, arr["f0"]) and np.array_equal(bf0, arr["bf0"])
        bc = np.flatnonzero((listed[:, 3] == 0) | (listed[:, 3] >= 1000)).astype(np.int32)
        out[f"run{r}_mom"] = np.stack([arr["D"], arr["U"], arr["V"], arr["W"]])
        out[f"run{r}_bc"] = bc
        out[f"run{r}_fN_bc"] = arr["fN"][:, bc]
        os.remove(path)
    np.savez_compressed(os.path.join(OUT, "ref_pressure.npz"), **out)
    print(f"pressure inlets: {len(PS.RUNS)} runs of {PS.STEPS} steps, {n} listed points")


OUTPUT_FILES = ("FLUIDdomain", "AllCellMemb", "AllCellNucleus", "AllNucEdgeMesh")


def output_fixture():
    """The reference's own OUTPUT() (oracle/ref/harness_output.c) on a small
    lattice and two cells: its inputs and the bytes of the files it writes."""
    import shutil
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), "../_ref/ref_output"], check=True)
    run = os.path.join(ROOT, "oracle", "_ref", "output_run")
    shutil.rmtree(run, ignore_errors=True)
    os.makedirs(run)
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_output"), "inputs.bin"], cwd=run, check=True,
                   stdout=open(os.path.join(run, "output.log"), "w"))
    raw = open(os.path.join(run, "inputs.bin"), "rb").read()
    pos = [0]

    def rd(dt, k):
        r = np.frombuffer(raw, dt, k, pos[0]).copy()
        pos[0] += r.itemsize * k
        return r
    n, nx, ny, nz, i0, j0, k0 = rd(np.int32, 7)
    rec = rd(np.int32, 6 * n).reshape(n, 6)
    fl = {k: rd(np.float32, n) for k in ("D", "U", "V", "W")}
    bf = rd(np.float32, 3 * n).reshape(3, n)
    area0 = rd(np.float32, 504)
    edge_n = rd(np.int32, 2 * 544).reshape(544, 2)
    lmax_n = rd(np.float32, 544)
    cells = {k: [] for k in ("head", "cellf", "x", "vel", "walltri", "wrep", "area", "ftot", "fvol", "outflag",
                             "xn", "veln", "ftotn", "nneigh", "nflag")}
    for _ in range(2):
        cells["head"].append(rd(np.int32, 3))
        cells["cellf"].append(rd(np.float32, 5))
        for k, dt, m in (("x", np.float64, 3 * 504), ("vel", np.float64, 3 * 504), ("walltri", np.int32, 504),
                         ("wrep", np.float32, 3 * 504), ("area", np.float32, 504), ("ftot", np.float32, 3 * 504),
                         ("fvol", np.float32, 3 * 504), ("outflag", np.int32, 504), ("xn", np.float64, 3 * 121),
                         ("veln", np.float64, 3 * 121), ("ftotn", np.float32, 3 * 121), ("nneigh", np.int32, 121),
                         ("nflag", np.int32, 121)):
            cells[k].append(rd(dt, m))
    assert pos[0] == len(raw)
    out = {"n_listed": n, "box": np.array([nx, ny, nz, i0, j0, k0], np.int32), "listed": rec, "bodyforce": bf,
           "area0": area0, "edge_n": edge_n, "lmax_n": lmax_n, **fl}
    for k, v in cells.items():
        a = np.stack(v)
        if a.shape[1] in (3 * 504, 3 * 121):  # [cell][3][n] -> [3][cell][n]
            a = a.reshape(2, 3, -1).transpose(1, 0, 2)
        out["cell_" + k] = a
    sdir = os.path.join(run, "SimulationOutputData")
    for name in OUTPUT_FILES:
        out["file_" + name] = np.frombuffer(open(os.path.join(sdir, name + "-000000000.csv"), "rb").read(), np.uint8)
    out["file_VolumeAreaHistory"] = np.frombuffer(open(os.path.join(sdir, "VolumeAreaHistory.dat"), "rb").read(),
                                                  np.uint8)
    shutil.rmtree(run)
    np.savez_compressed(os.path.join(OUT, "ref_output.npz"), **out)
    print(f"OUTPUT(): {n} listed points, 2 cells, files " +
          ", ".join(f"{k[5:]} {out[k].size} B" for k in out if k.startswith("file_")))


def wss_fixture():
    import shutil
    from golden import ib_scene as S
    from oracle.bind import OracleLBM
    b = S.lattice()
    lbm = OracleLBM(b, wall_mode=1, periodic=(0, 0, 0), tau=1.22, dt=0.5, precision="f32")
    lbm.set_f(S.wss_populations(b))
    lbm.moments_from_f()
    D, U, V, W = [np.asarray(a, np.float32) for a in lbm.moments()]
    xyz, tri, _ = S.wall()
    nrm = S.wall_node_normals(xyz)
    run = os.path.join(ROOT, "oracle", "_ref", "wss_run")
    shutil.rmtree(run, ignore_errors=True)
    for d in ("InputData", "SimulationOutputData", "PostProcessedData"):
        os.makedirs(os.path.join(run, d))
    inp = os.path.join(run, "InputData")
    nw = xyz.shape[1]
    # wall nodes beyond the mesh's own keep the post-processor's zero coordinates:
    # their search windows hold no lattice point, so they come out invalid with zero WSS
    with open(os.path.join(inp, "WallMeshNodeCoord.dat"), "w") as f:
        f.write(f"{nw}\n")
        for m in range(nw):
            f.write("%.9e %.9e %.9e\n" % (xyz[0, m], xyz[1, m], xyz[2, m]))
    with open(os.path.join(inp, "WallMeshNodeNormals.dat"), "w") as f:
        f.write("normals\n\n")
        for m in range(nw):
            f.write("%.9e %.9e %.9e\n" % (nrm[0, m], nrm[1, m], nrm[2, m]))
    with open(os.path.join(inp, "WallMeshCells.dat"), "w") as f:  # cells: only for the VTK output
        f.write("cells\n")
    with open(os.path.join(inp, "WallMeshCellNormals.aa"), "w") as f:
        f.write("normals\n\n")
    open(os.path.join(inp, "WallMeshCellNormals.ab"), "w").close()
    dom = np.argwhere(b >= 0)
    o = np.array(S.REF_ORIGIN)
    with open(os.path.join(run, "SimulationOutputData", "FLUIDdomain-000000000.csv"), "w") as f:
        f.write("X,Y,Z,Bindex,U,V,W,D,Bx,By,Bz,EulNeigh,Windex\n")
        for l, (i, j, k) in enumerate(dom):
            I, J, K = (np.array([i, j, k]) + np.array(S.OFFSET))  # 0-based reference indices
            f.write("%f,%f,%f,%d,%.9e,%.9e,%.9e,%.9e,0,0,0,0,0\n" % (
                o[0] + I * S.DX, o[1] + J * S.DX, o[2] + K * S.DX, b[i, j, k], U[l], V[l], W[l], D[l]))
    # the post-processor stops with "Could not open file" at the next output iteration
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "postpro_wss")], cwd=run, check=True,
                   stdout=open(os.path.join(run, "postpro.log"), "w"))
    txt = open(os.path.join(run, "PostProcessedData", "Wallpressure-000000000.vtk")).read()
    txt = txt[txt.index("POINT_DATA"):]

    def section(after, before, conv):
        a = txt.index("\n", txt.index(after)) + 1
        z = txt.index(before, a) if before else len(txt)
        return np.array([conv(v) for v in txt[a:z].split()[:nw]])
    press = section("LOOKUP_TABLE", "FIELD", float)
    wss = np.stack([section("WSSx 1", "WSSy 1", float), section("WSSy 1", "WSSz 1", float),
                    section("WSSz 1", "Valid 1", float)])
    valid = section("Valid 1", None, int)
    shutil.rmtree(run)  # ~120 MB of text files
    np.savez_compressed(os.path.join(OUT, "ref_wss.npz"), press=press.astype(np.float64),
                        wss=wss.astype(np.float64), valid=valid.astype(np.int32),
                        sum_vel=np.stack([U, V, W, D]).astype(np.float64).sum(axis=1))
    print(f"WSS: {nw} wall nodes, {int(valid.sum())} valid, max |WSS| {np.abs(wss).max():.4g} Pa")


LOOP_STEPS = 100


def loop_fixture():
    """100 iterations of the reference's time loop (LBM every step, cell blocks
    at 50 and 100) on the capped IB scene, by oracle/ref/harness_ib.c."""
    from golden import ib_scene as S
    G = np.load(os.path.join(OUT, "ref_setup.npz"))
    R = np.load(os.path.join(OUT, "ref_ib.npz"))
    x, xn = R["x"], R["xn"]
    b = S.lattice(capped=True)
    f0 = S.populations(b).astype(np.float32)
    n = f0.shape[1]
    wxyz, wtri, wnrm = S.wall()
    from oracle.bind import OracleLBM, OracleWorld
    lbm = OracleLBM(b, wall_mode=1, periodic=(0, 0, 0), precision="f32")
    w = OracleWorld(lbm, None, zf_params(S))
    w.set_wall(wxyz, wtri, wnrm)
    wi, uv = w.wall_index(b.shape)
    nc = x.shape[1]
    hdr = np.array(list(S.OFFSET) + [S.NX, S.NY, S.NZ, wxyz.shape[1], wtri.shape[1], nc, 0, n,
                                     LOOP_STEPS], np.int32)
    scene = os.path.join(ROOT, "oracle", "_ref", "loop_scene.bin")
    with open(scene, "wb") as f:
        for a, dt in ((hdr, np.int32), (b, np.int32), (np.zeros((3, n)), np.float32), (wi, np.int32),
                      (uv, np.float32), (wxyz, np.float32), (wtri, np.int32), (wnrm, np.float32),
                      (x, np.float64), (xn, np.float64), (f0, np.float32)):
            f.write(np.ascontiguousarray(a, dt).tobytes())
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), "../_ref/ref_ib"], check=True)
    out = os.path.join(ROOT, "oracle", "_ref", "ref_loop.bin")
    run = os.path.join(ROOT, "oracle", "_ref", "run")
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_ib"), scene, out], cwd=run, check=True,
                   stdout=open(os.path.join(ROOT, "oracle", "_ref", "ref_loop.log"), "w"))
    raw = open(out, "rb").read()
    pos = [0]

    def rd(dt, shape):
        k = int(np.prod(shape))
        r = np.frombuffer(raw, dt, k, pos[0]).copy().reshape(shape)
        pos[0] += r.itemsize * k
        return r
    f = rd(np.float32, (19, n))
    bf = rd(np.float32, (3, n))
    x_new, xn_new = rd(np.float64, (3, nc, x.shape[2])), rd(np.float64, (3, nc, xn.shape[2]))
    status, simf = rd(np.int32, (nc,)), rd(np.int32, (1,))
    assert pos[0] == len(raw)
    sample = np.arange(0, n, 97, dtype=np.int32)
    nzr = np.flatnonzero(np.any(bf != 0, axis=0)).astype(np.int32)
    np.savez_compressed(os.path.join(OUT, "ref_loop.npz"), steps=LOOP_STEPS, sample=sample,
                        f_sample=f[:, sample], f_sum=f.astype(np.float64).sum(axis=1),
                        bf_idx=nzr, bf_val=bf[:, nzr], x_new=x_new, xn_new=xn_new, status=status,
                        simfailure=simf)
    print(f"time loop: {LOOP_STEPS} steps, {n} listed points, moved up to "
          f"{np.abs(x_new - x).max():.3f} um, simfailure {int(simf[0])}")


def zf_params(S):
    import zebraflow_b200 as zf
    return zf.default_params(nx=S.NX, ny=S.NY, nz=S.NZ, origin=S.ORIGIN, periodic=(0, 0, 0))


def ib_fixture(nucleus=False):
    """The stage-by-stage IB fixture (ref_ib.npz); nucleus: the variant whose
    nuclei reach their membranes, run on the reference build with a 20-row tp
    array (ref_nuc.npz, nucleus-membrane stage only)."""
    from golden import ib_scene as S
    G = np.load(os.path.join(OUT, "ref_setup.npz"))
    mesh = (G["mesh_x"], G["mesh_tri"], G["nuc_x"], G["nuc_edges"])
    if nucleus:
        x, xn = S.place_cells(G["mesh_x"], G["nuc_x"], nucleus_scale=1.0, flatten3=0.92)
    else:
        x, xn = S.place_cells(G["mesh_x"], G["nuc_x"])
    b, p, lbm, oc, w = S.oracle_world(mesh, x, xn, "f32")
    _, U, V, W = lbm.moments()
    vel = np.stack([U, V, W]).astype(np.float32)
    wi, uv = w.wall_index(b.shape)
    wxyz, wtri, wnrm = S.wall()
    nc = x.shape[1]
    hdr = np.array(list(S.OFFSET) + [S.NX, S.NY, S.NZ, wxyz.shape[1], wtri.shape[1], nc, S.ITER,
                                     lbm.n, 0], np.int32)
    scene = os.path.join(ROOT, "oracle", "_ref", "ib_scene.bin")
    with open(scene, "wb") as f:
        for a, dt in ((hdr, np.int32), (b, np.int32), (vel, np.float32), (wi, np.int32),
                      (uv, np.float32), (wxyz, np.float32), (wtri, np.int32), (wnrm, np.float32),
                      (x, np.float64), (xn, np.float64)):
            f.write(np.ascontiguousarray(a, dt).tobytes())
    out = os.path.join(ROOT, "oracle", "_ref", "ref_nuc.bin" if nucleus else "ref_ib.bin")
    if os.path.exists(out):
        os.remove(out)
    if nucleus:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), "../_ref/ref_ib_tp20"],
                       check=True)
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_ib_tp20"), scene, out],
                       cwd=os.path.join(ROOT, "oracle", "_ref", "run"), check=True,
                       stdout=open(os.path.join(ROOT, "oracle", "_ref", "ref_nuc.log"), "w"))
    else:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle", "ref"), "../_ref/ref_ib.bin"],
                       check=True)
    raw = open(out, "rb").read()
    pos = [0]

    def rd(dt, shape):
        k = int(np.prod(shape))
        r = np.frombuffer(raw, dt, k, pos[0]).copy().reshape(shape)
        pos[0] += r.itemsize * k
        return r
    nn, nnn, n = x.shape[2], xn.shape[2], lbm.n
    res = {}
    res["ftot"], res["ftot_n"] = rd(np.float32, (3, nc, nn)), rd(np.float32, (3, nc, nnn))
    res["vel_interp"], res["vel_n_interp"] = rd(np.float64, (3, nc, nn)), rd(np.float64, (3, nc, nnn))
    res["rep_interp"], res["rep_n_interp"] = rd(np.float32, (3, nc, nn)), rd(np.float32, (3, nc, nnn))
    res["rep_nuc"], res["rep_n_nuc"] = rd(np.float32, (3, nc, nn)), rd(np.float32, (3, nc, nnn))
    res["rep_rbc"], res["rep_n_rbc"] = rd(np.float32, (3, nc, nn)), rd(np.float32, (3, nc, nnn))
    bf = rd(np.float32, (3, n))
    res["vel_spread"], res["vel_n_spread"] = rd(np.float64, (3, nc, nn)), rd(np.float64, (3, nc, nnn))
    res["x_new"], res["xn_new"] = rd(np.float64, (3, nc, nn)), rd(np.float64, (3, nc, nnn))
    res["status"] = rd(np.int32, (nc,))
    res["simfailure"] = rd(np.int32, (1,))
    assert pos[0] == len(raw)
    if nucleus:
        np.savez_compressed(os.path.join(OUT, "ref_nuc.npz"), x=x, xn=xn,
                            rep_interp=res["rep_interp"], rep_n_interp=res["rep_n_interp"],
                            rep_nuc=res["rep_nuc"], rep_n_nuc=res["rep_n_nuc"])
        touched = int(np.any(res["rep_nuc"] != res["rep_interp"], axis=0).sum())
        print(f"nucleus-membrane stage: {touched} membrane nodes repelled")
        return
    nzr = np.flatnonzero(np.any(bf != 0, axis=0)).astype(np.int32)  # spread body force, sparse
    np.savez_compressed(os.path.join(OUT, "ref_ib.npz"), x=x, xn=xn, bf_idx=nzr, bf_val=bf[:, nzr],
                        sum_vel=vel.astype(np.float64).sum(axis=1), sum_windex=np.int64(wi.sum()),
                        sum_uvoid=uv.astype(np.float64).sum(), n_listed=n, **res)
    print(f"IB stages: {nc} cells, {n} listed points, {nzr.size} points with spread force, "
          f"simfailure {int(res['simfailure'][0])}")


if __name__ == "__main__":
    main()

"""The reference's file formats (zebraflow_b200/csrc/zf_io.cpp), on the CPU.

The writers are held to the reference's own OUTPUT() (ZebraflowWT.c:282-509):
tests/golden/ref_output.npz keeps the inputs oracle/ref/harness_output.c gave
it and the bytes of the files it wrote; the same values through this
library's writers must give the same bytes.  The readers read those files
back, the shipped meshes and wall meshes, and files in the reference's input
formats written here."""
import gzip
import os

import numpy as np
import pytest

import zebraflow_b200 as zf
from conftest import ROOT
from oracle.refsrc import have_reference, reference_dir

GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def ref():
    return dict(np.load(os.path.join(GOLD, "ref_output.npz")))


def box(ref):
    """b_index, windex [nx][ny][nz] of the harness's box and its origin (um)."""
    nx, ny, nz, i0, j0, k0 = (int(v) for v in ref["box"])
    b = -np.ones((nx, ny, nz), np.int32)
    wi = np.zeros((nx, ny, nz), np.int32)
    rec = ref["listed"]
    i, j, k = rec[:, 0] - i0, rec[:, 1] - j0, rec[:, 2] - k0
    b[i, j, k] = rec[:, 3]
    wi[i, j, k] = rec[:, 5]
    # X = X0 + (i-1) DX with the reference's X0, Y0, Z0 = -1, 29, -27 (ZebraflowWT.c:85-87)
    origin = (-1.0 + (i0 - 1) * 0.5, 29.0 + (j0 - 1) * 0.5, -27.0 + (k0 - 1) * 0.5)
    return b, wi, origin


def cells(ref):
    ids = ref["cell_head"][:, 0]
    status = ref["cell_head"][:, 1]
    regress = ref["cell_head"][:, 2]
    return ids, status, regress


def test_fluid_snapshot_is_the_reference_file(ref, tmp_path):
    b, wi, origin = box(ref)
    out = str(tmp_path / "fluid.csv")
    zf.write_fluid_csv(out, b, ref["D"], ref["U"], ref["V"], ref["W"], ref["bodyforce"],
                       eulneigh=ref["listed"][:, 4], windex=wi, origin=origin)
    assert open(out, "rb").read() == ref["file_FLUIDdomain"].tobytes()


def test_cell_snapshots_are_the_reference_files(ref, tmp_path):
    ids, status, regress = cells(ref)
    area_ratio = (ref["cell_area"] / ref["area0"][None, :]).astype(np.float32)  # float / float, :438
    p = str(tmp_path / "memb.csv")
    zf.write_membrane_csv(p, status, ref["cell_x"], vel=ref["cell_vel"], wall_tri=ref["cell_walltri"],
                          wrep=ref["cell_wrep"], regress=regress, area_ratio=area_ratio, ftot=ref["cell_ftot"],
                          fvol=ref["cell_fvol"], out_flag=ref["cell_outflag"], cell_id=ids)
    assert open(p, "rb").read() == ref["file_AllCellMemb"].tobytes()
    p = str(tmp_path / "nuc.csv")
    zf.write_nucleus_csv(p, status, ref["cell_xn"], vel_n=ref["cell_veln"], ftot_n=ref["cell_ftotn"],
                         neigh=ref["cell_nneigh"], neigh_flag=ref["cell_nflag"], cell_id=ids)
    assert open(p, "rb").read() == ref["file_AllCellNucleus"].tobytes()
    p = str(tmp_path / "edges.csv")
    zf.write_nucleus_edges_csv(p, status, ref["cell_xn"], ref["edge_n"], ref["lmax_n"], cell_id=ids)
    assert open(p, "rb").read() == ref["file_AllNucEdgeMesh"].tobytes()
    p = str(tmp_path / "VolumeAreaHistory.dat")
    cf = np.zeros((2, 8), np.float32)
    cf[:, :5] = ref["cell_cellf"]
    zf.append_volume_area(p, 0, status, cf, regress=regress, cell_id=ids)
    assert open(p, "rb").read() == ref["file_VolumeAreaHistory"].tobytes()
    # appending a later iteration adds rows and no header
    zf.append_volume_area(p, 50, status, cf, regress=regress, cell_id=ids)
    lines = open(p).read().splitlines()
    assert len(lines) == 5 and lines[3].startswith("50,3,") and lines[4].startswith("50,9,")


def test_removed_cells_are_not_written(ref, tmp_path):
    ids, status, regress = cells(ref)
    st = status.copy()
    st[0] = -5000
    p = str(tmp_path / "memb.csv")
    zf.write_membrane_csv(p, st, ref["cell_x"], cell_id=ids)
    lines = open(p).read().splitlines()
    assert len(lines) == 1 + 504 and all(ln.split(",")[3] == "9" for ln in lines[1:])


def test_fluid_snapshot_reads_back(ref, tmp_path):
    b, wi, origin = box(ref)
    p = str(tmp_path / "fluid.csv")
    open(p, "wb").write(ref["file_FLUIDdomain"].tobytes())
    D, U, V, W, bf, en, wir, rows = zf.read_fluid_csv(p, b, origin=origin)
    assert rows == ref["n_listed"]
    # %.7e keeps 8 significant digits: within one float ulp of the written values
    for a, r in ((D, ref["D"]), (U, ref["U"]), (V, ref["V"]), (W, ref["W"]), (bf, ref["bodyforce"])):
        assert np.all(np.abs(a - r) <= 1.2e-7 * np.abs(r) + 1e-30)
    assert np.array_equal(en, ref["listed"][:, 4]) and np.array_equal(wir[b >= 0], wi[b >= 0])
    # the restart's populations: feq of the restored moments
    f = zf.equilibrium_populations(D, U, V, W)
    assert np.allclose(f.sum(axis=0), D, rtol=1e-6)
    assert np.allclose((f * zf.E[:, 2:3]).sum(axis=0), D * W, atol=1e-8)


def test_cell_snapshots_read_back(ref, tmp_path):
    ids, status, regress = cells(ref)
    p = str(tmp_path / "memb.csv")
    open(p, "wb").write(ref["file_AllCellMemb"].tobytes())
    cid, st, x, vel, ft = zf.read_cells_csv(p, 504)
    assert np.array_equal(cid, ids) and np.array_equal(st, status)
    assert np.abs(x - ref["cell_x"]).max() < 5.1e-7 + 2e-6  # %f, read into a float (as fscanf("%f"))
    assert np.all(np.abs(vel - ref["cell_vel"]) <= 1.2e-7 * np.abs(ref["cell_vel"]) + 1e-30)
    assert np.all(np.abs(ft - ref["cell_ftot"]) <= 1.2e-7 * np.abs(ref["cell_ftot"]) + 1e-30)
    p = str(tmp_path / "nuc.csv")
    open(p, "wb").write(ref["file_AllCellNucleus"].tobytes())
    cid, st, xn, veln, ftn = zf.read_cells_csv(p, 121, nucleus=True)
    assert np.array_equal(cid, ids) and xn.shape == (3, 2, 121)
    assert np.abs(xn - ref["cell_xn"]).max() < 5.1e-7 + 2e-6
    with pytest.raises(zf.ZfError):
        zf.read_cells_csv(p, 120, nucleus=True)  # rows are not a multiple of the nodes per cell


def test_bindex_file(tmp_path):
    rng = np.random.default_rng(3)
    dims, origin = (6, 5, 7), (-1.0, 29.0, -27.0)
    b = rng.integers(-1, 3, dims).astype(np.int32)
    p = str(tmp_path / "FLUIDdomainBindex.csv")
    with open(p, "w") as f:  # B_index first, then X, Y, Z (ZebraflowWT.c:2600-2617)
        f.write("Bindex,Points:0,Points:1,Points:2\n")
        for i, j, k in np.argwhere(b >= 0):
            f.write(f"{b[i, j, k]},{origin[0] + 0.5 * i:f},{origin[1] + 0.5 * j:f},{origin[2] + 0.5 * k:f}\n")
    got, rows = zf.read_bindex_csv(p, dims, origin=origin)
    assert rows == int((b >= 0).sum()) and np.array_equal(got, b)
    with open(p, "a") as f:
        f.write(f"1,{origin[0] + 0.5 * 9:f},{origin[1]:f},{origin[2]:f}\n")  # outside the box
    with pytest.raises(zf.ZfError):
        zf.read_bindex_csv(p, dims, origin=origin)


def test_parent_boundary_file(tmp_path):
    rng = np.random.default_rng(4)
    dims, origin = (5, 6, 4), (69.0, 218.5, -27.5)
    b = rng.integers(-1, 3, dims).astype(np.int32)
    p = str(tmp_path / "DAparentBoundary.csv")
    with open(p, "w") as f:  # quoted header, then Bindex, D, U, V, W and the point (ZebraflowWT.c:557-580)
        f.write('"Bindex","D","U","V","W","Points:0","Points:1","Points:2"\n')
        for i, j, k in np.argwhere(b >= 0):
            f.write(f"{b[i, j, k]},1,0,0,0,{origin[0] + 0.5 * i:g},{origin[1] + 0.5 * j:g},{origin[2] + 0.5 * k:g}\n")
    got, rows = zf.read_boundary_csv(p, dims, origin=origin)
    assert rows == int((b >= 0).sum()) and np.array_equal(got, b)
    if have_reference():  # the shipped file: 3008 rows inside its parent segment's box
        q = str(tmp_path / "shipped.csv")
        open(q, "wb").write(gzip.open(os.path.join(reference_dir(), "DAparentBoundary.csv.gz")).read())
        pts = np.loadtxt(q, delimiter=",", skiprows=1)
        lo = pts[:, 5:8].min(axis=0)
        ext = np.rint((pts[:, 5:8].max(axis=0) - lo) / 0.5).astype(int) + 1
        got, rows = zf.read_boundary_csv(q, tuple(ext), origin=tuple(lo))
        assert rows == 3008 and int((got >= 0).sum()) == len(np.unique(pts[:, 5:8], axis=0))


def test_mesh_files(tmp_path):
    s = np.load(os.path.join(GOLD, "ref_setup.npz"))
    X, T, XN, EN = s["mesh_x"], s["mesh_tri"], s["nuc_x"], s["nuc_edges"]
    files = {}
    if have_reference():  # the shipped files themselves
        for name in ("ZFISHRBCNODES", "ZFISHRBCTRIANGLES", "NucleusNodes", "NucleusEdges"):
            p = str(tmp_path / (name + ".dat"))
            open(p, "wb").write(gzip.open(os.path.join(reference_dir(), name + ".dat.gz")).read())
            files[name] = p
    else:  # the same values in their format
        for name, head, a, fmt in (("ZFISHRBCNODES", f"POINTS {len(X)} double", X, "%.17g"),
                                   ("ZFISHRBCTRIANGLES", f"CELLS {len(T)} {4 * len(T)}", T, "%d"),
                                   ("NucleusNodes", f"POINTS {len(XN)} double", XN, "%.17g"),
                                   ("NucleusEdges", f"LINES {len(EN)} {3 * len(EN)}", EN, "%d")):
            p = str(tmp_path / (name + ".dat"))
            np.savetxt(p, a, fmt=fmt, header=head, comments="")
            files[name] = p
    assert np.array_equal(zf.read_mesh_dat(files["ZFISHRBCNODES"], zf.MESH_POINTS), X)
    assert np.array_equal(zf.read_mesh_dat(files["ZFISHRBCTRIANGLES"], zf.MESH_CELLS), T)
    assert np.array_equal(zf.read_mesh_dat(files["NucleusNodes"], zf.MESH_POINTS), XN)
    assert np.array_equal(zf.read_mesh_dat(files["NucleusEdges"], zf.MESH_LINES), EN)
    with pytest.raises(zf.ZfError):
        zf.read_mesh_dat(files["NucleusEdges"], zf.MESH_POINTS)  # wrong header


def write_wall_files(d, xyz, tri, nrm):
    """A wall mesh in the reference's files: 3 points per line, '3 a b c'
    0-based triangles, CELL_DATA normals 3 per line (ZebraflowWT.c:3724-3897)."""
    nw, mt = xyz.shape[1], tri.shape[1]
    paths = [os.path.join(d, n) for n in ("WallMeshNodeCoord.dat", "WallMeshCells.dat", "WallMeshCellNormals.dat")]
    with open(paths[0], "w") as f:
        f.write(f"POINTS {nw} float\n")
        for m in range(0, nw, 3):
            f.write(" ".join("%g %g %g" % tuple(xyz[:, q]) for q in range(m, min(m + 3, nw))) + " \n")
    with open(paths[1], "w") as f:
        f.write(f"POLYGONS {mt} {4 * mt}\n")
        for m in range(mt):
            f.write("3 %d %d %d \n" % tuple(tri[:, m] - 1))
    with open(paths[2], "w") as f:
        f.write(f"CELL_DATA {mt}\nNORMALS Normals float\n")
        for m in range(0, mt, 3):
            f.write(" ".join("%g %g %g" % tuple(nrm[:, q]) for q in range(m, min(m + 3, mt))) + " \n")
    return paths


def test_wall_mesh_files(tmp_path):
    xyz, tri, nrm = zf.gen_wall_tube(11.5, 11.5, 9.0, 16)
    xyz = np.round(xyz, 4).astype(np.float32)
    nrm = np.round(nrm, 5).astype(np.float32)
    paths = write_wall_files(str(tmp_path), xyz, tri, nrm)
    gx, gt, gn = zf.read_wall_mesh(*paths)
    assert np.array_equal(gt, tri)
    assert np.array_equal(gx, np.array([[float("%g" % v) for v in r] for r in xyz], np.float32))
    assert np.abs(gn - nrm).max() < 1e-6


@pytest.mark.skipif(not have_reference(), reason="reference tree not present")
def test_shipped_wall_mesh(tmp_path):
    ref = reference_dir()
    paths = []
    for name in ("DAWallMeshNodeCoord", "DAWallMeshCells", "DAWallMeshCellNormals"):
        p = str(tmp_path / (name + ".dat"))
        open(p, "wb").write(gzip.open(os.path.join(ref, name + ".dat.gz")).read())
        paths.append(p)
    xyz, tri, nrm = zf.read_wall_mesh(*paths)
    lines = open(paths[0]).read().split("\n")
    vals = np.array([float(v) for ln in lines[1:] for v in ln.split()], np.float32).reshape(-1, 3).T
    assert xyz.shape == (3, 29282) and np.array_equal(xyz, vals)
    cel = np.array([int(v) for ln in open(paths[1]).read().split("\n")[1:] for v in ln.split()]).reshape(-1, 4)
    assert tri.shape == (3, 58080) and np.array_equal(tri, (cel[:, 1:] + 1).T)
    assert np.allclose(np.linalg.norm(nrm, axis=0), 1.0, atol=1e-4)


def test_wall_vtk_layout(tmp_path):
    xyz, tri, _ = zf.gen_wall_tube(11.5, 11.5, 9.0, 4)
    nw = xyz.shape[1]
    rng = np.random.default_rng(5)
    press = rng.uniform(50, 150, nw).astype(np.float32)
    wss = rng.normal(0, 0.5, (3, nw)).astype(np.float32)
    valid = (rng.uniform(size=nw) > 0.2).astype(np.int32)
    p = str(tmp_path / "Wallpressure-000000000.vtk")
    zf.write_wall_vtk(p, xyz, tri, press, wss, valid)
    txt = open(p).read()
    # the post-processor's layout (PostProWSSandPressure.c:380-430)
    assert txt.startswith("# vtk DataFile Version 4.0\nvtk output\nASCII\nDATASET POLYDATA\n"
                          f"POINTS {nw} float\n")
    assert f"POLYGONS {tri.shape[1]} {4 * tri.shape[1]}\n" in txt
    assert f"POINT_DATA {nw}\nSCALARS PRESSURE float\nLOOKUP_TABLE default\n" in txt
    body = txt[txt.index("LOOKUP_TABLE default\n") + 21:]
    pv = np.array(body[:body.index("FIELD")].split(), np.float64)
    assert np.allclose(pv, press, atol=5e-7)
    for name, row in (("WSSx", 0), ("WSSy", 1), ("WSSz", 2)):
        seg = txt[txt.index(f"{name} 1 {nw} float\n") + len(f"{name} 1 {nw} float\n"):]
        v = np.array(seg.split()[:nw], np.float64)
        assert np.allclose(v, wss[row], atol=5e-7)
    seg = txt[txt.index(f"Valid 1 {nw} int\n") + len(f"Valid 1 {nw} int\n"):]
    assert np.array_equal(np.array(seg.split(), int), valid)
    first = txt.split("\n")[5].split()
    assert len(first) == 9  # three points per line

// The reference's file formats, host side: readers of its input files and
// writers of the snapshots its OUTPUT() and post-processor write, so that a
// run of this library consumes and produces the same files.
//
//   FLUIDdomainBindex.csv     B_index per lattice point            read  ZebraflowWT.c:2574-2619
//   FLUIDdomain-*.csv         fluid snapshot (13 columns)           write :356-370, read :2649-2700
//   AllCellMemb-*.csv         membrane snapshot (21 columns)        write :429-442, read :5323-5420
//   AllCellNucleus-*.csv      nucleus snapshot (13 columns)         write :446-459, read :5549-5574
//   AllNucEdgeMesh-*.csv      nucleus spring stretch                write :461-504
//   VolumeAreaHistory.dat     per-cell volume, area, centroid       append :345-350
//   mesh .dat (POINTS / CELLS / LINES headers)                      read  :1601-1922
//   wall mesh (POINTS, POLYGONS 0-based, CELL_DATA NORMALS)         read  :3724-3897
//   Wallpressure-*.vtk        wall pressure and WSS (legacy VTK)    write PostProWSSandPressure.c:375-433
//
// Every function works on caller-owned host arrays in the layouts of
// include/zf.h and needs no device.  Numbers are printed with the reference's
// printf formats, so a snapshot written here from the same values is the
// reference's file byte for byte.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/zf.h"
#include "zf_internal.h"

namespace {

using zf::set_error;

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) : f(path ? std::fopen(path, mode) : nullptr) {}
  ~File() {
    if (f) std::fclose(f);
  }
  bool close() {  // true on success
    const bool ok = f && std::fclose(f) == 0;
    f = nullptr;
    return ok;
  }
};

// Whole-file reader with the reference's fscanf semantics for numbers
// separated by commas, blanks or line breaks.
struct Reader {
  std::vector<char> buf;
  size_t pos = 0;
  bool load(const char* path) {
    File in(path, "rb");
    if (!in.f) return false;
    std::fseek(in.f, 0, SEEK_END);
    const long n = std::ftell(in.f);
    std::fseek(in.f, 0, SEEK_SET);
    if (n < 0) return false;
    buf.resize((size_t)n + 1);
    if (n > 0 && std::fread(buf.data(), 1, (size_t)n, in.f) != (size_t)n) return false;
    buf[(size_t)n] = '\0';
    return true;
  }
  bool eof() {
    skip();
    return buf[pos] == '\0';
  }
  void skip() {
    while (buf[pos] == ',' || buf[pos] == ' ' || buf[pos] == '\t' || buf[pos] == '\r' || buf[pos] == '\n')
      ++pos;
  }
  std::string line() {  // the rest of the current line
    const size_t s = pos;
    while (buf[pos] != '\0' && buf[pos] != '\n') ++pos;
    std::string l(buf.data() + s, pos - s);
    if (buf[pos] == '\n') ++pos;
    return l;
  }
  bool num(double& v) {
    skip();
    char* end = nullptr;
    v = std::strtod(buf.data() + pos, &end);
    if (end == buf.data() + pos) return false;
    pos = (size_t)(end - buf.data());
    return true;
  }
  bool f32(float& v) {  // as fscanf("%f"): the decimal rounded to float
    skip();
    char* end = nullptr;
    v = std::strtof(buf.data() + pos, &end);
    if (end == buf.data() + pos) return false;
    pos = (size_t)(end - buf.data());
    return true;
  }
  bool i32(int32_t& v) {
    skip();
    char* end = nullptr;
    const long x = std::strtol(buf.data() + pos, &end, 10);
    if (end == buf.data() + pos) return false;
    pos = (size_t)(end - buf.data());
    v = (int32_t)x;
    return true;
  }
};

int fail_open(const char* fn, const char* path) {
  set_error("%s: cannot open %s (%s)", fn, path ? path : "(null)", std::strerror(errno));
  return ZF_ERR_ARG;
}

int fail_parse(const char* fn, const char* path, const char* what, long long row) {
  set_error("%s: %s: %s at data row %lld", fn, path, what, row);
  return ZF_ERR_ARG;
}

// 0-based lattice index of a coordinate, as the reference's 1-based
// (int)((x - x0)/DX + 1.01) (the reference's X0/DX are double macros)
inline int lat0(float x, double x0, double dx) { return (int)(((double)x - x0) / dx + 1.01) - 1; }

inline float lattice_coord(double x0, double dx, int i) { return (float)(x0 + i * dx); }

}  // namespace

extern "C" {

int zf_read_bindex_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                       int32_t* b_index, int64_t* n_rows) {
  static const char* fn = "zf_read_bindex_csv";
  if (!b_index || !origin || nx <= 0 || ny <= 0 || nz <= 0 || dx <= 0) return ZF_ERR_ARG;
  Reader r;
  if (!r.load(path)) return fail_open(fn, path);
  for (size_t p = 0; p < (size_t)nx * ny * nz; ++p) b_index[p] = -1;  // ZebraflowWT.c:2516
  r.line();                                                            // header
  long long row = 0;
  while (!r.eof()) {
    int32_t b;
    float x, y, z;
    if (!r.i32(b) || !r.f32(x) || !r.f32(y) || !r.f32(z)) return fail_parse(fn, path, "expected B_index,X,Y,Z", row + 1);
    const int i = lat0(x, origin[0], dx), j = lat0(y, origin[1], dx), k = lat0(z, origin[2], dx);
    if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz)
      return fail_parse(fn, path, "point outside the lattice box", row + 1);
    b_index[((size_t)i * ny + j) * nz + k] = b;
    ++row;
  }
  if (n_rows) *n_rows = row;
  return ZF_OK;
}

int zf_read_boundary_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                         int32_t* b_index, int64_t* n_rows) {
  static const char* fn = "zf_read_boundary_csv";
  if (!b_index || !origin || nx <= 0 || ny <= 0 || nz <= 0 || dx <= 0) return ZF_ERR_ARG;
  Reader r;
  if (!r.load(path)) return fail_open(fn, path);
  for (size_t p = 0; p < (size_t)nx * ny * nz; ++p) b_index[p] = -1;  // ZebraflowWT.c:546-555
  r.line();                                                            // header
  long long row = 0;
  while (!r.eof()) {
    int32_t b;
    float d, u, v, w, x, y, z;  // D, U, V, W are read and not kept, as at :563-570
    if (!r.i32(b) || !r.f32(d) || !r.f32(u) || !r.f32(v) || !r.f32(w) || !r.f32(x) || !r.f32(y) || !r.f32(z))
      return fail_parse(fn, path, "expected Bindex,D,U,V,W,Points:0,Points:1,Points:2", row + 1);
    const int i = lat0(x, origin[0], dx), j = lat0(y, origin[1], dx), k = lat0(z, origin[2], dx);
    if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz)
      return fail_parse(fn, path, "point outside the lattice box", row + 1);
    b_index[((size_t)i * ny + j) * nz + k] = b;
    ++row;
  }
  if (n_rows) *n_rows = row;
  return ZF_OK;
}

int zf_write_fluid_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                       const int32_t* b_index, const float* D, const float* U, const float* V, const float* W,
                       const float* bodyforce, const int32_t* eulneigh, const int32_t* windex) {
  static const char* fn = "zf_write_fluid_csv";
  if (!b_index || !origin || !D || !U || !V || !W || !bodyforce || nx <= 0 || ny <= 0 || nz <= 0)
    return ZF_ERR_ARG;
  int64_t n = 0;
  for (size_t p = 0; p < (size_t)nx * ny * nz; ++p) n += b_index[p] >= 0;
  File out(path, "w");
  if (!out.f) return fail_open(fn, path);
  std::fprintf(out.f, "X,Y,Z,Bindex,U,V,W,D,Bx,By,Bz,EulNeigh,Windex\n");
  int64_t l = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const size_t p = ((size_t)i * ny + j) * nz + k;
        if (b_index[p] < 0) continue;
        std::fprintf(out.f, "%f,%f,%f,%d,%.7e,%.7e,%.7e,%.7e,%.7e,%.7e,%.7e,%d,%d\n",
                     lattice_coord(origin[0], dx, i), lattice_coord(origin[1], dx, j),
                     lattice_coord(origin[2], dx, k), b_index[p], U[l], V[l], W[l], D[l], bodyforce[l],
                     bodyforce[n + l], bodyforce[2 * n + l], eulneigh ? eulneigh[l] : 0, windex ? windex[p] : 0);
        ++l;
      }
  if (!out.close()) return fail_open(fn, path);
  return ZF_OK;
}

int zf_read_fluid_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                      const int32_t* b_index, float* D, float* U, float* V, float* W, float* bodyforce,
                      int32_t* eulneigh, int32_t* windex, int64_t* n_rows) {
  static const char* fn = "zf_read_fluid_csv";
  if (!b_index || !origin || nx <= 0 || ny <= 0 || nz <= 0 || dx <= 0) return ZF_ERR_ARG;
  // DOMLIST position of every listed point
  std::vector<int64_t> dom((size_t)nx * ny * nz, -1);
  int64_t n = 0;
  for (size_t p = 0; p < dom.size(); ++p)
    if (b_index[p] >= 0) dom[p] = n++;
  Reader r;
  if (!r.load(path)) return fail_open(fn, path);
  r.line();
  long long row = 0;
  while (!r.eof()) {
    float x, y, z, u, v, w, d, bx, by, bz;
    int32_t b, en, wi;
    if (!r.f32(x) || !r.f32(y) || !r.f32(z) || !r.i32(b) || !r.f32(u) || !r.f32(v) || !r.f32(w) || !r.f32(d) ||
        !r.f32(bx) || !r.f32(by) || !r.f32(bz) || !r.i32(en) || !r.i32(wi))
      return fail_parse(fn, path, "expected 13 columns X,Y,Z,Bindex,U,V,W,D,Bx,By,Bz,EulNeigh,Windex", row + 1);
    ++row;
    if (b < 0) continue;  // only listed points are restored, ZebraflowWT.c:2681
    const int i = lat0(x, origin[0], dx), j = lat0(y, origin[1], dx), k = lat0(z, origin[2], dx);
    if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz)
      return fail_parse(fn, path, "point outside the lattice box", row);
    const size_t p = ((size_t)i * ny + j) * nz + k;
    if (windex) windex[p] = wi;
    const int64_t l = dom[p];
    if (l < 0) return fail_parse(fn, path, "row at a point the lattice does not list", row);
    if (D) D[l] = d;
    if (U) U[l] = u;
    if (V) V[l] = v;
    if (W) W[l] = w;
    if (bodyforce) {
      bodyforce[l] = bx;
      bodyforce[n + l] = by;
      bodyforce[2 * n + l] = bz;
    }
    if (eulneigh) eulneigh[l] = en;
  }
  if (n_rows) *n_rows = row;
  return ZF_OK;
}

int zf_equilibrium_populations(int64_t n, const float* D, const float* U, const float* V, const float* W,
                               float* f) {
  if (n < 0 || !D || !U || !V || !W || !f) return ZF_ERR_ARG;
  // FEQ of the reference's initialisation, ZebraflowWT.c:2561-2570 (EQ_A = 3,
  // EQ_B = 4.5, EQ_C = -1.5; C_LBM = 1), in the reference's direction order
  static const int E[19][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},   {0, 0, -1}, {1, 1, 0},
                               {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0}, {1, 0, 1},  {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1},
                               {0, 1, 1},  {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 0, 0}};
  for (int64_t l = 0; l < n; ++l)
    for (int q = 0; q < 19; ++q) {
      const float w = q < 6 ? 1.f / 18.f : (q < 18 ? 1.f / 36.f : 1.f / 3.f);
      const float cu = U[l] * E[q][0] + V[l] * E[q][1] + W[l] * E[q][2];
      const float uu = U[l] * U[l] + V[l] * V[l] + W[l] * W[l];
      f[(size_t)q * n + l] = (float)(D[l] * w * (1. + 3. * cu + 4.5 * cu * cu + -1.5 * uu));
    }
  return ZF_OK;
}

int zf_write_membrane_csv(const char* path, int n_cells, int n_node, const int32_t* cell_id,
                          const int32_t* status, const double* x, const double* vel, const int32_t* wall_tri,
                          const float* wrep, const int32_t* regress, const float* area_ratio, const float* ftot,
                          const float* fvol, const int32_t* out_flag) {
  static const char* fn = "zf_write_membrane_csv";
  if (n_cells < 0 || n_node <= 0 || !status || !x) return ZF_ERR_ARG;
  File out(path, "w");
  if (!out.f) return fail_open(fn, path);
  std::fprintf(out.f,
               "X,Y,Z,Cell,CellStatus,Vx,Vy,Vz,WallTri,WallRepulfX,WallRepulfY,WallRepulfZ,regressflag,Aratio,"
               "Fx,Fy,Fz,FVx,FVy,FVz,OutNeighFlag\n");
  const size_t nc = (size_t)n_cells, nn = (size_t)n_node;
  auto at = [&](int v, int c, int n) { return ((size_t)v * nc + c) * nn + n; };
  for (int c = 0; c < n_cells; ++c) {
    if (!(status[c] > -5000)) continue;  // removed cells are not written, ZebraflowWT.c:432
    for (int n = 0; n < n_node; ++n) {
      auto f3 = [&](const float* a, int v) { return a ? (double)a[at(v, c, n)] : 0.0; };
      auto d3 = [&](const double* a, int v) { return a ? a[at(v, c, n)] : 0.0; };
      std::fprintf(out.f, "%f,%f,%f,%d,%d,%.7e,%.7e,%.7e,%d,%.7e,%.7e,%.7e,%d,%.7e,%.7e,%.7e,%.7e,%.7e,%.7e,%.7e,%d\n",
                   x[at(0, c, n)], x[at(1, c, n)], x[at(2, c, n)], cell_id ? cell_id[c] : c + 1, status[c],
                   d3(vel, 0), d3(vel, 1), d3(vel, 2), wall_tri ? wall_tri[(size_t)c * nn + n] : 0, f3(wrep, 0),
                   f3(wrep, 1), f3(wrep, 2), regress ? regress[c] : 0,
                   area_ratio ? (double)area_ratio[(size_t)c * nn + n] : 0.0, f3(ftot, 0), f3(ftot, 1),
                   f3(ftot, 2), f3(fvol, 0), f3(fvol, 1), f3(fvol, 2), out_flag ? out_flag[(size_t)c * nn + n] : 0);
    }
  }
  if (!out.close()) return fail_open(fn, path);
  return ZF_OK;
}

int zf_write_nucleus_csv(const char* path, int n_cells, int n_node_n, const int32_t* cell_id,
                         const int32_t* status, const double* xn, const double* vel_n, const float* ftot_n,
                         const int32_t* neigh, const int32_t* neigh_flag) {
  static const char* fn = "zf_write_nucleus_csv";
  if (n_cells < 0 || n_node_n <= 0 || !status || !xn) return ZF_ERR_ARG;
  File out(path, "w");
  if (!out.f) return fail_open(fn, path);
  std::fprintf(out.f, "X,Y,Z,Cell,CellStatus,Vx,Vy,Vz,Fx,Fy,Fz,Neigh,Neighflag\n");
  const size_t nc = (size_t)n_cells, nn = (size_t)n_node_n;
  auto at = [&](int v, int c, int n) { return ((size_t)v * nc + c) * nn + n; };
  for (int c = 0; c < n_cells; ++c) {
    if (!(status[c] > -5000)) continue;  // ZebraflowWT.c:450
    for (int n = 0; n < n_node_n; ++n)
      std::fprintf(out.f, "%f,%f,%f,%d,%d,%.7e,%.7e,%.7e,%.7e,%.7e,%.7e,%d,%d\n", xn[at(0, c, n)], xn[at(1, c, n)],
                   xn[at(2, c, n)], cell_id ? cell_id[c] : c + 1, status[c], vel_n ? vel_n[at(0, c, n)] : 0.0,
                   vel_n ? vel_n[at(1, c, n)] : 0.0, vel_n ? vel_n[at(2, c, n)] : 0.0,
                   ftot_n ? (double)ftot_n[at(0, c, n)] : 0.0, ftot_n ? (double)ftot_n[at(1, c, n)] : 0.0,
                   ftot_n ? (double)ftot_n[at(2, c, n)] : 0.0, neigh ? neigh[(size_t)c * nn + n] : 0,
                   neigh_flag ? neigh_flag[(size_t)c * nn + n] : 0);
  }
  if (!out.close()) return fail_open(fn, path);
  return ZF_OK;
}

int zf_write_nucleus_edges_csv(const char* path, int n_cells, int n_node_n, int n_edge_n, const int32_t* cell_id,
                               const int32_t* status, const double* xn, const int32_t* edge_n, const float* lmax_n) {
  static const char* fn = "zf_write_nucleus_edges_csv";
  if (n_cells < 0 || n_node_n <= 0 || n_edge_n < 0 || !status || !xn || !edge_n || !lmax_n) return ZF_ERR_ARG;
  File out(path, "w");
  if (!out.f) return fail_open(fn, path);
  std::fprintf(out.f, "X,Y,Z,Cell,LX,LY,LZ,Stretch\n");
  const size_t nc = (size_t)n_cells, nn = (size_t)n_node_n;
  for (int c = 0; c < n_cells; ++c) {
    if (!(status[c] > -5000)) continue;  // ZebraflowWT.c:467
    for (int e = 0; e < n_edge_n; ++e) {
      const int n1 = edge_n[2 * e] - 1, n2 = edge_n[2 * e + 1] - 1;
      float p1[3], p2[3], m[3], ev[3];
      for (int v = 0; v < 3; ++v) {  // float locals as :471-482
        p1[v] = (float)xn[((size_t)v * nc + c) * nn + n1];
        p2[v] = (float)xn[((size_t)v * nc + c) * nn + n2];
        m[v] = (float)(0.5 * (p1[v] + p2[v]));
        ev[v] = p1[v] - p2[v];
      }
      const float len = sqrtf(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]);
      const float ratio = (float)(len * 1.e-06 / lmax_n[e]);
      std::fprintf(out.f, "%.7e,%.7e,%.7e,%d,%.7e,%.7e,%.7e,%.7e\n", m[0], m[1], m[2], cell_id ? cell_id[c] : c + 1,
                   ev[0], ev[1], ev[2], ratio);
    }
  }
  if (!out.close()) return fail_open(fn, path);
  return ZF_OK;
}

int zf_append_volume_area(const char* path, int64_t iter, int n_cells, const int32_t* cell_id,
                          const int32_t* status, const float* cell_f, const int32_t* regress) {
  static const char* fn = "zf_append_volume_area";
  if (n_cells < 0 || !status || !cell_f) return ZF_ERR_ARG;
  File out(path, "a");
  if (!out.f) return fail_open(fn, path);
  if (iter == 0) std::fprintf(out.f, "Iteration#,Cell,Vol,Area,CenX,CenY,CenZ,CellState,RegressFlag\n");
  for (int c = 0; c < n_cells; ++c) {
    if (!(status[c] > -5000)) continue;  // ZebraflowWT.c:348
    const float* g = cell_f + 8 * (size_t)c;  // area, volume, centroid x, y, z (zf_get_cell_geometry)
    std::fprintf(out.f, "%d,%d,%.7e,%.7e,%.7e,%.7e,%.7e,%d,%d\n", (int)iter, cell_id ? cell_id[c] : c + 1,
                 (double)g[1], (double)g[0], (double)g[2], (double)g[3], (double)g[4], status[c],
                 regress ? regress[c] : 0);
  }
  if (!out.close()) return fail_open(fn, path);
  return ZF_OK;
}

int zf_read_cells_csv(const char* path, int nucleus, int n_node, int cap_cells, int* n_cells, int32_t* cell_id,
                      int32_t* status, double* x, double* vel, float* ftot) {
  static const char* fn = "zf_read_cells_csv";
  if (!n_cells || n_node <= 0 || cap_cells < 0) return ZF_ERR_ARG;
  Reader r;
  if (!r.load(path)) return fail_open(fn, path);
  r.line();
  // rows of one cell are consecutive, n_node per cell (ZebraflowWT.c:5357-5420)
  struct Row {
    float x[3], v[3], f[3];
    int32_t cell, st;
  };
  std::vector<Row> rows;
  long long row = 0;
  while (!r.eof()) {
    Row w;
    int32_t idum;
    float fdum;
    bool ok = r.f32(w.x[0]) && r.f32(w.x[1]) && r.f32(w.x[2]) && r.i32(w.cell) && r.i32(w.st) && r.f32(w.v[0]) &&
              r.f32(w.v[1]) && r.f32(w.v[2]);
    if (ok && !nucleus) {  // WallTri, WallRepulf xyz, regressflag, Aratio
      ok = r.i32(idum) && r.f32(fdum) && r.f32(fdum) && r.f32(fdum) && r.i32(idum) && r.f32(fdum);
    }
    ok = ok && r.f32(w.f[0]) && r.f32(w.f[1]) && r.f32(w.f[2]);
    if (ok && !nucleus) ok = r.f32(fdum) && r.f32(fdum) && r.f32(fdum) && r.i32(idum);  // FV xyz, OutNeighFlag
    if (ok && nucleus) ok = r.i32(idum) && r.i32(idum);                                    // Neigh, Neighflag
    if (!ok) return fail_parse(fn, path, nucleus ? "expected 13 columns" : "expected 21 columns", row + 1);
    rows.push_back(w);
    ++row;
  }
  if (rows.size() % (size_t)n_node) return fail_parse(fn, path, "row count is not a multiple of the nodes per cell", row);
  const int nc = (int)(rows.size() / (size_t)n_node);
  *n_cells = nc;
  if (!x) return ZF_OK;  // size query
  if (nc > cap_cells) {
    set_error("%s: %s holds %d cells, the buffers %d", fn, path, nc, cap_cells);
    return ZF_ERR_OVERFLOW;
  }
  for (int c = 0; c < nc; ++c)
    for (int n = 0; n < n_node; ++n) {
      const Row& w = rows[(size_t)c * n_node + n];
      if (w.cell != rows[(size_t)c * n_node].cell)
        return fail_parse(fn, path, "a cell's rows are not consecutive", (long long)c * n_node + n + 1);
      if (n == 0) {
        if (cell_id) cell_id[c] = w.cell;
        if (status) status[c] = w.st;
      }
      for (int v = 0; v < 3; ++v) {
        const size_t g = ((size_t)v * nc + c) * n_node + n;
        x[g] = w.x[v];  // %f read into a float, then stored as the reference's double
        if (vel) vel[g] = w.v[v];
        if (ftot) ftot[g] = w.f[v];
      }
    }
  return ZF_OK;
}

int zf_read_mesh_dat(const char* path, int kind, int* n, double* values, int cap) {
  static const char* fn = "zf_read_mesh_dat";
  if (!n || kind < 0 || kind > 2) return ZF_ERR_ARG;
  static const char* heads[3] = {"POINTS", "CELLS", "LINES"};
  const int per[3] = {3, 3, 2};
  Reader r;
  if (!r.load(path)) return fail_open(fn, path);
  const std::string h = r.line();
  int count = 0;
  if (h.compare(0, std::strlen(heads[kind]), heads[kind]) != 0 ||
      std::sscanf(h.c_str() + std::strlen(heads[kind]), "%d", &count) != 1 || count < 0) {
    set_error("%s: %s: expected a '%s n' header, found '%.60s'", fn, path, heads[kind], h.c_str());
    return ZF_ERR_ARG;
  }
  *n = count;
  if (!values) return ZF_OK;
  if (count > cap) {
    set_error("%s: %s holds %d entries, the buffer %d", fn, path, count, cap);
    return ZF_ERR_OVERFLOW;
  }
  for (long long i = 0; i < (long long)count * per[kind]; ++i) {
    double v;
    if (!r.num(v)) return fail_parse(fn, path, "too few values", i / per[kind] + 1);
    values[i] = v;
  }
  return ZF_OK;
}

int zf_read_wall_mesh(const char* nodes_path, const char* cells_path, const char* normals_path, int* n_node_w,
                      int* n_tri_w, float* xyz, int32_t* tri, float* normals, int cap_node, int cap_tri) {
  static const char* fn = "zf_read_wall_mesh";
  if (!n_node_w || !n_tri_w) return ZF_ERR_ARG;
  Reader rn, rc, rm;
  if (!rn.load(nodes_path)) return fail_open(fn, nodes_path);
  if (!rc.load(cells_path)) return fail_open(fn, cells_path);
  if (!rm.load(normals_path)) return fail_open(fn, normals_path);
  int nw = 0, mt = 0, mt2 = 0, mtn = 0;
  std::string h = rn.line();
  if (std::sscanf(h.c_str(), "POINTS %d", &nw) != 1) {
    set_error("%s: %s: expected 'POINTS n float'", fn, nodes_path);
    return ZF_ERR_ARG;
  }
  h = rc.line();
  if (std::sscanf(h.c_str(), "POLYGONS %d %d", &mt, &mt2) != 2) {
    set_error("%s: %s: expected 'POLYGONS n 4n'", fn, cells_path);
    return ZF_ERR_ARG;
  }
  h = rm.line();
  if (std::sscanf(h.c_str(), "CELL_DATA %d", &mtn) != 1 || mtn != mt) {
    set_error("%s: %s: expected 'CELL_DATA %d'", fn, normals_path, mt);
    return ZF_ERR_ARG;
  }
  rm.line();  // NORMALS Normals float
  *n_node_w = nw;
  *n_tri_w = mt;
  if (!xyz || !tri || !normals) return ZF_OK;
  if (nw > cap_node || mt > cap_tri) {
    set_error("%s: the mesh has %d nodes / %d triangles, the buffers %d / %d", fn, nw, mt, cap_node, cap_tri);
    return ZF_ERR_OVERFLOW;
  }
  for (int m = 0; m < nw; ++m)  // three points per line, :3724-3810
    for (int v = 0; v < 3; ++v)
      if (!rn.f32(xyz[(size_t)v * nw + m])) return fail_parse(fn, nodes_path, "too few coordinates", m + 1);
  for (int m = 0; m < mt; ++m) {  // "3 a b c", 0-based; stored +1 as :3826-3835
    int32_t cnt, a, b, c;
    if (!rc.i32(cnt) || !rc.i32(a) || !rc.i32(b) || !rc.i32(c) || cnt != 3)
      return fail_parse(fn, cells_path, "expected '3 a b c'", m + 1);
    if (a < 0 || a >= nw || b < 0 || b >= nw || c < 0 || c >= nw)
      return fail_parse(fn, cells_path, "node index outside the mesh", m + 1);
    tri[m] = a + 1;
    tri[(size_t)mt + m] = b + 1;
    tri[2 * (size_t)mt + m] = c + 1;
  }
  for (int m = 0; m < mt; ++m)
    for (int v = 0; v < 3; ++v)
      if (!rm.f32(normals[(size_t)v * mt + m])) return fail_parse(fn, normals_path, "too few normals", m + 1);
  return ZF_OK;
}

int zf_write_wall_vtk(const char* path, int n_node_w, const float* xyz, int n_tri_w, const int32_t* tri,
                      const float* pressure, const float* wss, const int32_t* valid) {
  static const char* fn = "zf_write_wall_vtk";
  if (n_node_w < 0 || n_tri_w < 0 || !xyz || !tri || !pressure || !wss || !valid) return ZF_ERR_ARG;
  File out(path, "w");
  if (!out.f) return fail_open(fn, path);
  FILE* f = out.f;
  const int nw = n_node_w, mt = n_tri_w;
  std::fprintf(f, "# vtk DataFile Version 4.0\n");
  std::fprintf(f, "vtk output\n");
  std::fprintf(f, "ASCII\n");
  std::fprintf(f, "DATASET POLYDATA\n");
  std::fprintf(f, "POINTS %d float\n", nw);
  for (int m = 0; m < nw; ++m) {
    std::fprintf(f, "%f %f %f ", (double)xyz[m], (double)xyz[(size_t)nw + m], (double)xyz[2 * (size_t)nw + m]);
    if ((m + 1) % 3 == 0) std::fprintf(f, "\n");
  }
  std::fprintf(f, "\n");
  std::fprintf(f, "POLYGONS %d %d\n", mt, mt * 4);
  for (int m = 0; m < mt; ++m)
    std::fprintf(f, "%d %d %d %d\n", 3, tri[m] - 1, tri[(size_t)mt + m] - 1, tri[2 * (size_t)mt + m] - 1);
  std::fprintf(f, "POINT_DATA %d\n", nw);
  std::fprintf(f, "SCALARS PRESSURE float\n");
  std::fprintf(f, "LOOKUP_TABLE default\n");
  auto column = [&](const float* a) {
    for (int m = 0; m < nw; ++m) {
      std::fprintf(f, "%f ", (double)a[m]);
      if ((m + 1) % 6 == 0) std::fprintf(f, "\n");
    }
  };
  column(pressure);
  std::fprintf(f, "FIELD FieldData 4\n");
  static const char* names[3] = {"WSSx", "WSSy", "WSSz"};
  for (int v = 0; v < 3; ++v) {
    std::fprintf(f, "%s 1 %d float\n", names[v], nw);
    column(wss + (size_t)v * nw);
  }
  std::fprintf(f, "Valid 1 %d int\n", nw);
  for (int m = 0; m < nw; ++m) {
    std::fprintf(f, "%d ", valid[m]);
    if ((m + 1) % 6 == 0) std::fprintf(f, "\n");
  }
  if (!out.close()) return fail_open(fn, path);
  return ZF_OK;
}

}  // extern "C"

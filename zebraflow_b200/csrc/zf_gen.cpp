// Reference parameter defaults and the input generators of the benchmark and
// test workloads: voxelised vessels (straight tube, periodic Y-bifurcation) in
// reference B_index codes, icosphere membrane meshes, seeded cell placement and
// the vessels' wall meshes.  The reference reads its zebrafish geometry from
// files (ZebraflowWT.c:2574-2619, :3714-3967, :1601-1922); these generators
// produce the same codes and layouts for synthetic vessels.
//
// Plain host C++ with no CUDA: libzf.so exports these functions as zf_*, and
// the CPU arm's library (oracle/liboracle.so) compiles this same file with
// ZF_SYM renaming them orc_*, so that both arms of a comparison build their
// inputs from one definition without loading the GPU library.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../include/zf.h"

#ifndef ZF_SYM
#define ZF_SYM(name) zf_##name
#endif

namespace {

const int kE18[18][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},   {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                         {1, 1, 0},  {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0}, {1, 0, 1},  {-1, 0, -1},
                         {-1, 0, 1}, {1, 0, -1}, {0, 1, 1},   {0, -1, -1}, {0, -1, 1}, {0, 1, -1}};

// Marks wall points: non-fluid points with a fluid neighbour along one of the
// 18 lattice links (these are the points the reference lists with B_index 0).
void mark_walls(int nx, int ny, int nz, int periodic_z, int32_t* b) {
  auto at = [&](int i, int j, int k) -> int32_t& { return b[((int64_t)i * ny + j) * nz + k]; };
  // first pass decides, second pass writes (a point's own code must not change
  // while its neighbours are still being classified)
  std::vector<uint8_t> is_wall((size_t)nx * ny * nz, 0);
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        if (at(i, j, k) > 0) continue;
        bool wall = false;
        for (int q = 0; q < 18 && !wall; ++q) {
          int ii = i + kE18[q][0], jj = j + kE18[q][1], kk = k + kE18[q][2];
          if (periodic_z) kk = (kk + nz) % nz;
          if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) continue;
          if (at(ii, jj, kk) > 0) wall = true;
        }
        is_wall[((size_t)i * ny + j) * nz + k] = wall;
      }
  for (size_t n = 0; n < is_wall.size(); ++n)
    if (b[n] <= 0) b[n] = is_wall[n] ? 0 : -1;
}

double seg_dist2(double px, double py, double pz, const double* a, const double* b) {
  double d[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double w[3] = {px - a[0], py - a[1], pz - a[2]};
  double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double t = dd > 0 ? (w[0] * d[0] + w[1] * d[1] + w[2] * d[2]) / dd : 0.0;
  t = t < 0 ? 0 : (t > 1 ? 1 : t);
  double r[3] = {w[0] - t * d[0], w[1] - t * d[1], w[2] - t * d[2]};
  return r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
}

uint64_t edge_key(int a, int b) {
  if (a > b) std::swap(a, b);
  return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
}

struct MeshOut {
  std::vector<float> x, y, z;
  std::vector<int32_t> tri;  // 0-based
  std::vector<float> n;      // per triangle, 3 each
};

void orient_and_normals(MeshOut& M, const std::vector<float>& gx, const std::vector<float>& gy,
                        const std::vector<float>& gz) {
  // make each triangle's geometric normal point along the given inward direction
  const size_t mt = M.tri.size() / 3;
  M.n.resize(3 * mt);
  for (size_t t = 0; t < mt; ++t) {
    int* v = &M.tri[3 * t];
    const float ax = M.x[v[1]] - M.x[v[0]], ay = M.y[v[1]] - M.y[v[0]], az = M.z[v[1]] - M.z[v[0]];
    const float bx = M.x[v[2]] - M.x[v[0]], by = M.y[v[2]] - M.y[v[0]], bz = M.z[v[2]] - M.z[v[0]];
    float nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
    if (nx * gx[t] + ny * gy[t] + nz * gz[t] < 0) {
      std::swap(v[1], v[2]);
      nx = -nx;
      ny = -ny;
      nz = -nz;
    }
    const float r = sqrtf(nx * nx + ny * ny + nz * nz);
    M.n[3 * t] = nx / r;
    M.n[3 * t + 1] = ny / r;
    M.n[3 * t + 2] = nz / r;
  }
}

int emit(const MeshOut& M, int* n_node, int* n_tri, float* xyz, int32_t* tri, float* nrm, int cap_node,
         int cap_tri) {
  const int nw = (int)M.x.size(), mt = (int)(M.tri.size() / 3);
  *n_node = nw;
  *n_tri = mt;
  if (!xyz || !tri || !nrm) return ZF_OK;  // size query
  if (nw > cap_node || mt > cap_tri) return ZF_ERR_OVERFLOW;
  for (int i = 0; i < nw; ++i) {
    xyz[i] = M.x[i];
    xyz[nw + i] = M.y[i];
    xyz[2 * nw + i] = M.z[i];
  }
  for (int t = 0; t < mt; ++t)
    for (int a = 0; a < 3; ++a) {
      tri[(size_t)a * mt + t] = M.tri[3 * t + a] + 1;
      nrm[(size_t)a * mt + t] = M.n[3 * t + a];
    }
  return ZF_OK;
}

}  // namespace

extern "C" {

void ZF_SYM(params_default)(zf_params* p) {
  std::memset(p, 0, sizeof *p);
  // ZebraflowWT.c:81-87 (ROI box) and :40-41 (DX, DT)
  p->nx = 249;
  p->ny = 547;
  p->nz = 723;
  p->origin[0] = -1.0;
  p->origin[1] = 29.0;
  p->origin[2] = -27.0;
  p->dx = 0.5;
  p->dt = 0.5;
  // TauPlasma = 0.5 + MU_SCALE*MU = 1.22 (ZebraflowWT.c:62); phase-dependent (ZebraflowWT.c:6110)
  p->tau = 1.22f;
  p->tau_from_phase = 1;
  p->wall_mode = ZF_WALL_REF_EQ;
  p->storage = ZF_STORE_F32;
  p->rho_ref = 1.0f;
  p->stagger = 50;                 // SOLVERSTAGGER, ZebraflowWT.c:151
  p->Es = 3.e-06;                  // ZebraflowWT.c:130
  p->Es_nucleus_ratio = 0.1;       // ZebraflowWT.c:2039
  p->kbend = 1.3856406e-19;        // ZebraflowWT.c:129
  p->kd = 3.6e-05;                 // ZebraflowWT.c:131
  p->ka = 7.7e-05;                 // ZebraflowWT.c:132
  p->kv = 55.;                     // ZebraflowWT.c:133
  p->area0 = 144.916e-012;         // RBC_SURF, ZebraflowWT.c:127
  p->volume0 = 97.5671e-018;       // MCV, ZebraflowWT.c:126
  p->kT = 300 * 1.3806488e-023;    // TEMPERATURE*BOLTZ, ZebraflowWT.c:36-37
  p->e_ratio_eq = 0.3154574132;    // ZebraflowWT.c:134
  p->calib_passes = 51;            // iterrelax loop, ZebraflowWT.c:2339-2346
  p->gamma_p = 1.e-07;             // ZebraflowWT.c:125
  p->unit_mass = 0.5e-6 * 0.5e-6 * 0.5e-6 * 10. * 1000.;  // UNITMASS, ZebraflowWT.c:50-51
  p->bforce_scale = 1. / 3. * 0.5e-6 / (0.5e-6 * 0.5e-6);  // LBM_BFORCE_SCALE, ZebraflowWT.c:65
  p->vel_scale = 1.0;              // VEL_SCALE, ZebraflowWT.c:67
  p->vmax_remove = 5.e-3;          // ZebraflowWT.c:11976
  p->remove_count = 500;           // ZebraflowWT.c:7473
  p->nuc_list_period = 1000;       // ZebraflowWT.c:9527
  p->nuc_list_max = 1004;          // NucMembMAX, ZebraflowWT.c:158
  p->stochastic_round = 1;
  // WALLNODETOCELLNEIGHBORLIST holds 12 entries but its overflow check fires
  // above 24 (ZebraflowWT.c:221, :3911-3934); 24 is the capacity here
  p->wall_list_max = 24;
}

// Straight tube along z: fluid (code 1) where (i-cx)^2+(j-cy)^2 < R^2 in
// lattice units, walls (0) on the first non-fluid layer, solid (-1) beyond.
// With periodic_z the tube wraps in z.
int ZF_SYM(gen_tube)(int nx, int ny, int nz, double cx, double cy, double R, int periodic_z,
                int32_t* b_index) {
  if (!b_index || nx <= 0 || ny <= 0 || nz <= 0 || R <= 0) return ZF_ERR_ARG;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const double r2 = (i - cx) * (i - cx) + (j - cy) * (j - cy);
      const int32_t v = r2 < R * R ? 1 : -1;
      for (int k = 0; k < nz; ++k) b_index[((int64_t)i * ny + j) * nz + k] = v;
    }
  mark_walls(nx, ny, nz, periodic_z, b_index);
  return ZF_OK;
}

// Periodic Y-bifurcation along z: a parent tube of radius Rp on the box axis
// splits, at half-angle `half_angle_deg`, into two daughters of radius Rd
// (in x), runs straight, and merges back into the parent so that the vessel
// is periodic in z.  Lattice units; fluid code 1, walls 0, solid -1.
// Returns the daughter offset and segment lengths through `layout`
// (6 doubles: z_split, z_straight, z_converge, z_merge, offset, unused) if non-NULL.
int ZF_SYM(gen_bifurcation)(int nx, int ny, int nz, double Rp, double Rd, double half_angle_deg,
                       int32_t* b_index, double* layout) {
  if (!b_index || nx <= 0 || ny <= 0 || nz <= 0 || Rp <= 0 || Rd <= 0) return ZF_ERR_ARG;
  const double cx = 0.5 * (nx - 1), cy = 0.5 * (ny - 1);
  const double ta = std::tan(half_angle_deg * M_PI / 180.0);
  double D = 0.8 * (0.5 * (nx - 1) - Rd - 2.0);  // daughter lateral offset
  double Ldiv = D / ta;
  const double Lpar = 0.1 * nz;
  if (2 * Lpar + 2 * Ldiv > 0.9 * nz) {  // short boxes: shrink the offset to fit
    Ldiv = 0.5 * (0.9 * nz - 2 * Lpar);
    D = Ldiv * ta;
  }
  const double z1 = Lpar, z2 = z1 + Ldiv, z4 = nz - Lpar, z3 = z4 - Ldiv;
  if (layout) {
    layout[0] = z1;
    layout[1] = z2;
    layout[2] = z3;
    layout[3] = z4;
    layout[4] = D;
    layout[5] = 0;
  }
  // centreline segments {a, b, radius}; parents extended by one period image
  struct Seg {
    double a[3], b[3], r;
  };
  std::vector<Seg> segs;
  segs.push_back({{cx, cy, z4 - nz}, {cx, cy, z1}, Rp});
  segs.push_back({{cx, cy, z4}, {cx, cy, z1 + nz}, Rp});
  for (int s = -1; s <= 1; s += 2) {
    segs.push_back({{cx, cy, z1}, {cx + s * D, cy, z2}, Rd});
    segs.push_back({{cx + s * D, cy, z2}, {cx + s * D, cy, z3}, Rd});
    segs.push_back({{cx + s * D, cy, z3}, {cx, cy, z4}, Rd});
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        int32_t v = -1;
        for (const Seg& sg : segs) {
          if (seg_dist2(i, j, k, sg.a, sg.b) < sg.r * sg.r) {
            v = 1;
            break;
          }
        }
        b_index[((int64_t)i * ny + j) * nz + k] = v;
      }
  mark_walls(nx, ny, nz, 1, b_index);
  return ZF_OK;
}

// Icosphere: the unit icosahedron subdivided `level` times (each triangle
// into four, midpoints projected to the sphere).  10*4^L+2 nodes and
// 20*4^L triangles, wound counter-clockwise seen from outside (outward
// normals, like the reference mesh).  xyz [n_node][3]; tri [n_tri][3] 1-based.
int ZF_SYM(gen_icosphere)(int level, double* xyz, int32_t* tri) {
  if (level < 0 || level > 6 || !xyz || !tri) return ZF_ERR_ARG;
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<double> V = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t,
                           0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
  std::vector<int> F = {0, 11, 5, 0, 5,  1,  0, 1, 7, 0, 7,  10, 0, 10, 11, 1, 5, 9, 5, 11,
                        4, 11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9,  4,  3,  4,  2, 3, 2, 6, 3,
                        6, 8,  3, 8, 9,  4, 9, 5, 2, 4, 11, 6,  2,  10, 8,  6, 7, 9, 8, 1};
  auto norm = [&](int i) {
    double* p = &V[3 * i];
    const double r = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    p[0] /= r;
    p[1] /= r;
    p[2] /= r;
  };
  for (int i = 0; i < 12; ++i) norm(i);
  for (int L = 0; L < level; ++L) {
    std::unordered_map<uint64_t, int> mid;
    std::vector<int> G;
    auto midpoint = [&](int a, int b) {
      const uint64_t k = edge_key(a, b);
      auto it = mid.find(k);
      if (it != mid.end()) return it->second;
      const int id = (int)(V.size() / 3);
      for (int s = 0; s < 3; ++s) V.push_back(0.5 * (V[3 * a + s] + V[3 * b + s]));
      norm(id);
      mid[k] = id;
      return id;
    };
    for (size_t f = 0; f < F.size(); f += 3) {
      const int a = F[f], b = F[f + 1], c = F[f + 2];
      const int ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
      const int g[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
      G.insert(G.end(), g, g + 12);
    }
    F.swap(G);
  }
  std::memcpy(xyz, V.data(), V.size() * sizeof(double));
  for (size_t f = 0; f < F.size(); ++f) tri[f] = F[f] + 1;
  return ZF_OK;
}

// Seeded placement of n_cells cells in a vessel (B_index codes, lattice
// units): centres uniform over fluid points, orientations uniform (random
// unit quaternion), rejecting a candidate whose ellipsoid (semi-axes
// `axes` um plus `margin` um) overlaps an accepted one on the lattice, or
// any of whose membrane nodes has a non-fluid lattice point within the cube
// of half-width r = max(1, ceil(wall_clear / dx)) around its nearest lattice
// point.  Outputs x [3][n_cells][n_node], xn [3][n_cells][n_node_n] in um.
// Returns the number placed in *placed (fewer than asked when the attempts
// run out).
int ZF_SYM(gen_cells)(const int32_t* b, int nx, int ny, int nz, const double* origin, double dx,
                 int periodic_z, int n_cells, int n_node, const double* rest, int n_node_n,
                 const double* rest_n, const double* axes, double margin, double wall_clear,
                 uint64_t seed, double* x, double* xn, int* placed) {
  if (!b || !origin || !rest || !axes || !x || !placed || n_cells < 0 || dx <= 0) return ZF_ERR_ARG;
  uint64_t st = seed;
  auto next = [&]() {  // splitmix64
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  auto uni = [&]() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); };
  std::vector<int64_t> fluid;
  for (int64_t p = 0; p < (int64_t)nx * ny * nz; ++p)
    if (b[p] > 0) fluid.push_back(p);
  if (fluid.empty()) return ZF_ERR_ARG;
  std::vector<uint8_t> occ((size_t)nx * ny * nz, 0);
  // clear[p] = 1 when every point of the cube of half-width r around p is
  // fluid: the fluid mask eroded by a cube, one axis at a time (a point
  // outside the box counts as non-fluid, except across a periodic z face)
  const int r_clear = std::max(1, (int)std::ceil(wall_clear / dx - 1e-9));
  std::vector<uint8_t> clear((size_t)nx * ny * nz);
  for (int64_t p = 0; p < (int64_t)nx * ny * nz; ++p) clear[p] = b[p] > 0;
  {
    const int64_t stride[3] = {(int64_t)ny * nz, nz, 1};
    const int len[3] = {nx, ny, nz};
    for (int ax = 0; ax < 3; ++ax) {
      const int L = len[ax];
      const bool wrap = ax == 2 && periodic_z;
      const int64_t nlines = (int64_t)nx * ny * nz / L;
#pragma omp parallel
      {
        std::vector<int> bad((size_t)L + 1);
        std::vector<uint8_t> line((size_t)L);
#pragma omp for schedule(static)
        for (int64_t l = 0; l < nlines; ++l) {
          // base point of line l: the index with the axis coordinate zero
          int64_t base;
          if (ax == 0) base = l;                                    // l = j*nz + k
          else if (ax == 1) base = (l / nz) * (int64_t)ny * nz + l % nz;  // l = i*nz + k
          else base = l * nz;                                       // l = i*ny + j
          for (int t = 0; t < L; ++t) line[t] = clear[base + t * stride[ax]];
          bad[0] = 0;  // prefix counts of non-fluid points
          for (int t = 0; t < L; ++t) bad[t + 1] = bad[t] + (line[t] ? 0 : 1);
          const int total = bad[L];
          for (int t = 0; t < L; ++t) {
            int lo = t - r_clear, hi = t + r_clear, cnt;
            if (wrap) {
              if (2 * r_clear + 1 >= L) cnt = total;
              else if (lo < 0) cnt = bad[hi + 1] + (total - bad[L + lo]);
              else if (hi >= L) cnt = (total - bad[lo]) + bad[hi - L + 1];
              else cnt = bad[hi + 1] - bad[lo];
            } else {
              cnt = (lo < 0 || hi >= L) ? 1 : bad[hi + 1] - bad[lo];
            }
            clear[base + t * stride[ax]] = cnt == 0;
          }
        }
      }
    }
  }
  auto at = [&](int i, int j, int k) -> int64_t {
    if (i < 0 || i >= nx || j < 0 || j >= ny) return -1;
    if (k < 0 || k >= nz) {
      if (!periodic_z) return -1;
      k = ((k % nz) + nz) % nz;
    }
    return ((int64_t)i * ny + j) * nz + k;
  };
  const double A[3] = {axes[0] + margin, axes[1] + margin, axes[2] + margin};
  const int reach = (int)std::ceil(std::max(A[0], std::max(A[1], A[2])) / dx) + 1;
  struct Cand {
    double c[3];
    double R[3][3];
  };
  // the whole candidate stream comes from the seed; a candidate is accepted
  // when it fits against the cells accepted before it, so evaluating a batch
  // in parallel against the occupancy at the start of the batch and then
  // re-checking the survivors in order gives the sequential result
  auto fits = [&](const Cand& cd, std::vector<int64_t>* mark) -> bool {
    const double ci = cd.c[0], cj = cd.c[1], ck = cd.c[2];
    const int64_t s0 = at((int)std::lround(ci), (int)std::lround(cj), (int)std::lround(ck));
    if (s0 < 0 || occ[s0]) return false;
    // every membrane node at least r lattice units (Chebyshev) from the wall
    for (int n = 0; n < n_node; ++n) {
      double pos[3];
      for (int a = 0; a < 3; ++a)
        pos[a] = cd.R[a][0] * rest[3 * n] + cd.R[a][1] * rest[3 * n + 1] + cd.R[a][2] * rest[3 * n + 2];
      const int64_t s = at((int)std::lround(ci + pos[0] / dx), (int)std::lround(cj + pos[1] / dx),
                           (int)std::lround(ck + pos[2] / dx));
      if (s < 0 || !clear[s]) return false;
    }
    // lattice points inside the inflated ellipsoid: free?
    for (int di = -reach; di <= reach; ++di)
      for (int dj = -reach; dj <= reach; ++dj)
        for (int dk = -reach; dk <= reach; ++dk) {
          const int i = (int)std::floor(ci) + di, j = (int)std::floor(cj) + dj, k = (int)std::floor(ck) + dk;
          const double v[3] = {(i - ci) * dx, (j - cj) * dx, (k - ck) * dx};
          double q[3];
          for (int a = 0; a < 3; ++a) q[a] = cd.R[0][a] * v[0] + cd.R[1][a] * v[1] + cd.R[2][a] * v[2];
          const double e = q[0] * q[0] / (A[0] * A[0]) + q[1] * q[1] / (A[1] * A[1]) + q[2] * q[2] / (A[2] * A[2]);
          if (e > 1.0) continue;
          const int64_t s = at(i, j, k);
          if (s < 0 || occ[s]) return false;
          if (mark) mark->push_back(s);
        }
    return true;
  };
  int n_ok = 0;
  const int64_t max_tries = 12000LL * n_cells + 1000;
  const int64_t batch = 4096;
  std::vector<Cand> cand((size_t)batch);
  std::vector<uint8_t> pass((size_t)batch);
  std::vector<int64_t> mark;
  for (int64_t tries = 0; n_ok < n_cells && tries < max_tries; tries += batch) {
    const int64_t nb = std::min(batch, max_tries - tries);
    for (int64_t t = 0; t < nb; ++t) {
      Cand& cd = cand[(size_t)t];
      const int64_t p = fluid[(size_t)(uni() * fluid.size()) % fluid.size()];
      cd.c[0] = (double)(p / ((int64_t)ny * nz)) + uni() - 0.5;
      cd.c[1] = (double)((p / nz) % ny) + uni() - 0.5;
      cd.c[2] = (double)(p % nz) + uni() - 0.5;
      // uniform rotation (Shoemake)
      const double u1 = uni(), u2 = uni(), u3 = uni();
      const double qw = std::sqrt(1 - u1) * std::sin(2 * M_PI * u2), qx = std::sqrt(1 - u1) * std::cos(2 * M_PI * u2),
                   qy = std::sqrt(u1) * std::sin(2 * M_PI * u3), qz = std::sqrt(u1) * std::cos(2 * M_PI * u3);
      const double R[3][3] = {{1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)},
                              {2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)},
                              {2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)}};
      std::memcpy(cd.R, R, sizeof(R));
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < nb; ++t) pass[(size_t)t] = fits(cand[(size_t)t], nullptr);
    for (int64_t t = 0; t < nb && n_ok < n_cells; ++t) {
      if (!pass[(size_t)t]) continue;
      const Cand& cd = cand[(size_t)t];
      mark.clear();
      if (!fits(cd, &mark)) continue;
      for (int64_t s : mark) occ[s] = 1;
      const double c0[3] = {origin[0] + cd.c[0] * dx, origin[1] + cd.c[1] * dx, origin[2] + cd.c[2] * dx};
      for (int n = 0; n < n_node; ++n)
        for (int a = 0; a < 3; ++a)
          x[((size_t)a * n_cells + n_ok) * n_node + n] =
              c0[a] + cd.R[a][0] * rest[3 * n] + cd.R[a][1] * rest[3 * n + 1] + cd.R[a][2] * rest[3 * n + 2];
      if (xn && rest_n)
        for (int n = 0; n < n_node_n; ++n)
          for (int a = 0; a < 3; ++a)
            xn[((size_t)a * n_cells + n_ok) * n_node_n + n] =
                c0[a] + cd.R[a][0] * rest_n[3 * n] + cd.R[a][1] * rest_n[3 * n + 1] + cd.R[a][2] * rest_n[3 * n + 2];
      ++n_ok;
    }
  }
  *placed = n_ok;
  return ZF_OK;
}

// Cylinder wall of radius R (lattice units) around the lattice axis (cx, cy),
// along z over nz lattice spacings, in um with the lattice origin/spacing;
// rings every `h` lattice units, `nseg` segments around; inward normals.
// The band that would close the periodic seam is left open.  With NULL
// outputs only the sizes are returned.
int ZF_SYM(gen_wall_tube)(double cx, double cy, double R, int nz, double h, int nseg,
                     const double* origin, double dx, int* n_node, int* n_tri, float* xyz,
                     int32_t* tri, float* nrm, int cap_node, int cap_tri) {
  if (R <= 0 || nz <= 0 || h <= 0 || nseg < 3 || !origin || dx <= 0) return ZF_ERR_ARG;
  MeshOut M;
  const int nring = (int)std::floor(nz / h);
  for (int r = 0; r < nring; ++r)
    for (int s = 0; s < nseg; ++s) {
      const double th = 2 * M_PI * (s + 0.5 * (r & 1)) / nseg;
      M.x.push_back((float)(origin[0] + (cx + R * std::cos(th)) * dx));
      M.y.push_back((float)(origin[1] + (cy + R * std::sin(th)) * dx));
      M.z.push_back((float)(origin[2] + r * h * dx));
    }
  std::vector<float> gx, gy, gz;
  for (int r = 0; r + 1 < nring; ++r)
    for (int s = 0; s < nseg; ++s) {
      const int a = r * nseg + s, b = r * nseg + (s + 1) % nseg;
      const int c2 = (r + 1) * nseg + s, d = (r + 1) * nseg + (s + 1) % nseg;
      const int tris[2][3] = {{a, b, c2}, {b, d, c2}};
      for (auto& t : tris) {
        M.tri.insert(M.tri.end(), t, t + 3);
        const float mx = (M.x[t[0]] + M.x[t[1]] + M.x[t[2]]) / 3.f - (float)(origin[0] + cx * dx);
        const float my = (M.y[t[0]] + M.y[t[1]] + M.y[t[2]]) / 3.f - (float)(origin[1] + cy * dx);
        gx.push_back(-mx);
        gy.push_back(-my);
        gz.push_back(0.f);
      }
    }
  orient_and_normals(M, gx, gy, gz);
  return emit(M, n_node, n_tri, xyz, tri, nrm, cap_node, cap_tri);
}

// Wall of the periodic Y-bifurcation of zf_gen_bifurcation (same arguments):
// the zero set of the signed distance to the vessel (union of capsules),
// extracted by marching tetrahedra on the lattice, vertices shared between
// neighbouring cubes, inward normals.  The periodic seam cubes are skipped.
int ZF_SYM(gen_wall_bifurcation)(int nx, int ny, int nz, double Rp, double Rd, double half_angle_deg,
                            const double* origin, double dx, int* n_node, int* n_tri, float* xyz,
                            int32_t* tri, float* nrm, int cap_node, int cap_tri) {
  if (!origin || dx <= 0 || nx <= 1 || ny <= 1 || nz <= 1) return ZF_ERR_ARG;
  const double cxa = 0.5 * (nx - 1), cya = 0.5 * (ny - 1);
  const double ta = std::tan(half_angle_deg * M_PI / 180.0);
  double D = 0.8 * (0.5 * (nx - 1) - Rd - 2.0), Ldiv = D / ta;
  const double Lpar = 0.1 * nz;
  if (2 * Lpar + 2 * Ldiv > 0.9 * nz) {
    Ldiv = 0.5 * (0.9 * nz - 2 * Lpar);
    D = Ldiv * ta;
  }
  const double z1 = Lpar, z2 = z1 + Ldiv, z4 = nz - Lpar, z3 = z4 - Ldiv;
  struct Seg {
    double a[3], b[3], r;
  };
  std::vector<Seg> segs = {{{cxa, cya, z4 - nz}, {cxa, cya, z1}, Rp},
                           {{cxa, cya, z4}, {cxa, cya, z1 + nz}, Rp}};
  for (int s = -1; s <= 1; s += 2) {
    segs.push_back({{cxa, cya, z1}, {cxa + s * D, cya, z2}, Rd});
    segs.push_back({{cxa + s * D, cya, z2}, {cxa + s * D, cya, z3}, Rd});
    segs.push_back({{cxa + s * D, cya, z3}, {cxa, cya, z4}, Rd});
  }
  auto sdf = [&](double x, double y, double z) {  // < 0 inside the lumen
    double best = 1e30;
    for (const Seg& g : segs) {
      double d[3] = {g.b[0] - g.a[0], g.b[1] - g.a[1], g.b[2] - g.a[2]};
      double w[3] = {x - g.a[0], y - g.a[1], z - g.a[2]};
      double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      double t = dd > 0 ? (w[0] * d[0] + w[1] * d[1] + w[2] * d[2]) / dd : 0.0;
      t = t < 0 ? 0 : (t > 1 ? 1 : t);
      double r[3] = {w[0] - t * d[0], w[1] - t * d[1], w[2] - t * d[2]};
      best = std::min(best, std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) - g.r);
    }
    return best;
  };
  // signed distance at lattice points
  std::vector<float> phi((size_t)nx * ny * nz);
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) phi[((size_t)i * ny + j) * nz + k] = (float)sdf(i, j, k);
  auto P = [&](int i, int j, int k) { return phi[((size_t)i * ny + j) * nz + k]; };
  MeshOut M;
  std::unordered_map<uint64_t, int> vid;  // lattice edge (min point, max point) -> vertex
  auto vertex = [&](const int* p, const int* q) -> int {
    uint64_t a = ((uint64_t)p[0] * ny + p[1]) * nz + p[2], b = ((uint64_t)q[0] * ny + q[1]) * nz + q[2];
    if (a > b) std::swap(a, b);
    const uint64_t key = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull + (a << 6) + (a >> 2));
    auto it = vid.find(key);
    if (it != vid.end()) return it->second;
    const double fp = P(p[0], p[1], p[2]), fq = P(q[0], q[1], q[2]);
    const double t = fp / (fp - fq);
    const int id = (int)M.x.size();
    M.x.push_back((float)(origin[0] + (p[0] + t * (q[0] - p[0])) * dx));
    M.y.push_back((float)(origin[1] + (p[1] + t * (q[1] - p[1])) * dx));
    M.z.push_back((float)(origin[2] + (p[2] + t * (q[2] - p[2])) * dx));
    vid[key] = id;
    return id;
  };
  std::vector<float> gx, gy, gz;
  // Kuhn split of a cube into 6 tetrahedra along the main diagonal 0-7
  static const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  static const int tets[6][4] = {{0, 1, 3, 7}, {0, 3, 2, 7}, {0, 2, 6, 7},
                                 {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 5, 1, 7}};
  for (int i = 0; i + 1 < nx; ++i)
    for (int j = 0; j + 1 < ny; ++j)
      for (int k = 0; k + 1 < nz; ++k) {
        float f[8];
        bool neg = false, pos = false;
        for (int v = 0; v < 8; ++v) {
          f[v] = P(i + corner[v][0], j + corner[v][1], k + corner[v][2]);
          (f[v] < 0 ? neg : pos) = true;
        }
        if (!neg || !pos) continue;
        for (const auto& T : tets) {
          int in[4], out[4], ni = 0, no = 0;
          for (int v = 0; v < 4; ++v) (f[T[v]] < 0 ? in[ni++] : out[no++]) = T[v];
          if (ni == 0 || no == 0) continue;
          auto pt = [&](int v, int* o3) {
            o3[0] = i + corner[v][0];
            o3[1] = j + corner[v][1];
            o3[2] = k + corner[v][2];
          };
          auto V = [&](int a, int b) {
            int pa[3], pb[3];
            pt(a, pa);
            pt(b, pb);
            return vertex(pa, pb);
          };
          std::vector<std::array<int, 3>> ts;
          if (ni == 1) ts.push_back({V(in[0], out[0]), V(in[0], out[1]), V(in[0], out[2])});
          else if (ni == 3) ts.push_back({V(out[0], in[0]), V(out[0], in[1]), V(out[0], in[2])});
          else {
            const int a = V(in[0], out[0]), b = V(in[0], out[1]), c2 = V(in[1], out[1]),
                      d = V(in[1], out[0]);
            ts.push_back({a, b, c2});
            ts.push_back({a, c2, d});
          }
          for (auto& t : ts) {
            if (t[0] == t[1] || t[1] == t[2] || t[0] == t[2]) continue;
            M.tri.insert(M.tri.end(), t.begin(), t.end());
            // inward = -grad(phi) at the triangle centroid (central differences)
            const double mx = ((M.x[t[0]] + M.x[t[1]] + M.x[t[2]]) / 3.0 - origin[0]) / dx;
            const double my = ((M.y[t[0]] + M.y[t[1]] + M.y[t[2]]) / 3.0 - origin[1]) / dx;
            const double mz = ((M.z[t[0]] + M.z[t[1]] + M.z[t[2]]) / 3.0 - origin[2]) / dx;
            const double e = 0.25;
            gx.push_back((float)-(sdf(mx + e, my, mz) - sdf(mx - e, my, mz)));
            gy.push_back((float)-(sdf(mx, my + e, mz) - sdf(mx, my - e, mz)));
            gz.push_back((float)-(sdf(mx, my, mz + e) - sdf(mx, my, mz - e)));
          }
        }
      }
  orient_and_normals(M, gx, gy, gz);
  return emit(M, n_node, n_tri, xyz, tri, nrm, cap_node, cap_tri);
}

}  // extern "C"

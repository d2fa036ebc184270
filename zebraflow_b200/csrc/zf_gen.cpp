// Input generators for the benchmark and test workloads: voxelised vessels
// (straight tube, periodic Y-bifurcation/confluence) in reference B_index
// codes, icosphere membrane meshes, seeded cell placement and a cylinder wall
// mesh.  The reference reads its zebrafish geometry from files
// (ZebraflowWT.c:2574-2619, :3714-3967, :1601-1922); these generators produce
// the same codes and layouts for synthetic vessels.
#include <cmath>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "zf_internal.h"

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

}  // namespace

extern "C" {

// Straight tube along z: fluid (code 1) where (i-cx)^2+(j-cy)^2 < R^2 in
// lattice units, walls (0) on the first non-fluid layer, solid (-1) beyond.
// With periodic_z the tube wraps in z.
int zf_gen_tube(int nx, int ny, int nz, double cx, double cy, double R, int periodic_z,
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
int zf_gen_bifurcation(int nx, int ny, int nz, double Rp, double Rd, double half_angle_deg,
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

}  // extern "C"

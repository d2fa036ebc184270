// Vessel wall meshes: generators for the synthetic vessels and the host
// set-up of the wall data the IB kernels read.
//
// Reference behaviour restated in zf_set_wall (ZebraflowWT.c):
//  - W_index: for every wall-mesh node in order, the lattice points of its
//    +-4 window take it as their nearest wall node when strictly closer than
//    what they hold (Wdistance starts at 5000), :3715-3822
//  - WALLNODETOCELLNEIGHBORLIST: triangles around each wall node, :3899-3935
//  - WALL_CENTROID: :4648-4663
//  - extraluminal "void" velocity at non-fluid points with W_index > 0:
//    normal of the nearest adjacent triangle times a ramp of the wall
//    distance (0 below 0.7 um, 1 above 3 um) times 1e-3 um/us, :4788-4852.
//    The reference measures that nearest triangle from stale coordinates
//    (xp, yp, zp are not set inside the loop); here it is measured from the
//    lattice point itself.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "zf_internal.h"

namespace zf {

// Minimum-image difference along a periodic axis of length L (L <= 0: none).
static inline double mind(double d, double L) {
  if (L <= 0) return d;
  return d - L * std::floor(d / L + 0.5);
}

int wall_build(zf_ctx* c, int nw, const float* xyz, int mt, const int32_t* tri1,
               const float* nrm, WallHost& W) {
  const zf_params& P = c->p;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const double X0 = P.origin[0], Y0 = P.origin[1], Z0 = P.origin[2], DX = P.dx;
  const double Lz = P.periodic[2] ? nz * DX : 0.0;
  W.nw = nw;
  W.mt = mt;
  W.xyz.assign(xyz, xyz + 3 * (size_t)nw);
  W.nrm.assign(nrm, nrm + 3 * (size_t)mt);
  W.tri.resize(3 * (size_t)mt);  // input [3][mt] (WALLCELLNODE layout) -> [mt][3]
  for (int m = 0; m < mt; ++m)
    for (int v = 0; v < 3; ++v) {
      const int32_t id = tri1[(size_t)v * mt + m];
      if (id < 1 || id > nw) {
        set_error("zf_set_wall: triangle node %d out of range 1..%d", id, nw);
        return ZF_ERR_ARG;
      }
      W.tri[3 * (size_t)m + v] = id - 1;
    }
  // node -> triangle lists in triangle order, ZebraflowWT.c:3907-3932
  const int cap = P.wall_list_max;
  W.cap = cap;
  W.ntri.assign((size_t)nw * (cap + 1), 0);
  for (int m = 0; m < mt; ++m)
    for (int v = 0; v < 3; ++v) {
      const int n = W.tri[3 * (size_t)m + (size_t)v];
      int32_t* L = &W.ntri[(size_t)n * (cap + 1)];
      if (L[0] >= cap) {
        c->status.list_overflows++;
        continue;
      }
      L[0] += 1;
      L[L[0]] = m;
    }
  // centroids (float sums over 3, as :4658)
  W.cen.resize(3 * (size_t)mt);
  for (int m = 0; m < mt; ++m)
    for (int a = 0; a < 3; ++a) {
      const float s = xyz[(size_t)a * nw + W.tri[3 * m]] + xyz[(size_t)a * nw + W.tri[3 * m + 1]] +
                      xyz[(size_t)a * nw + W.tri[3 * m + 2]];
      W.cen[(size_t)a * mt + m] = (float)(s / 3.);
    }
  // candidate points of each node's list, contiguous, in the order searched
  W.cand_off.assign((size_t)nw + 1, 0);
  for (int n = 0; n < nw; ++n) W.cand_off[n + 1] = W.cand_off[n] + 4 * W.ntri[(size_t)n * (cap + 1)];
  W.cand.resize((size_t)W.cand_off[nw]);
  for (int n = 0; n < nw; ++n) {
    const int32_t* L = &W.ntri[(size_t)n * (cap + 1)];
    float4* out = W.cand.data() + W.cand_off[n];
    for (int l = 1; l <= L[0]; ++l) {
      const int t = L[l];
      float tid;
      std::memcpy(&tid, &t, sizeof tid);
      for (int v = 0; v < 3; ++v) {
        const int q = W.tri[3 * (size_t)t + v];
        *out++ = make_float4(xyz[q], xyz[(size_t)nw + q], xyz[2 * (size_t)nw + q], tid);
      }
      *out++ = make_float4(W.cen[t], W.cen[(size_t)mt + t], W.cen[2 * (size_t)mt + t], tid);
    }
  }
  // node normals: triangle normals weighted by triangle area, normalised
  W.nnrm.assign(3 * (size_t)nw, 0.f);
  {
    std::vector<double> acc(3 * (size_t)nw, 0.0);
    for (int m = 0; m < mt; ++m) {
      double e1[3], e2[3];
      for (int a = 0; a < 3; ++a) {
        e1[a] = (double)xyz[(size_t)a * nw + W.tri[3 * m + 1]] - xyz[(size_t)a * nw + W.tri[3 * m]];
        e2[a] = (double)xyz[(size_t)a * nw + W.tri[3 * m + 2]] - xyz[(size_t)a * nw + W.tri[3 * m]];
      }
      const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                   cz = e1[0] * e2[1] - e1[1] * e2[0];
      const double area = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
      for (int v = 0; v < 3; ++v)
        for (int a = 0; a < 3; ++a) acc[(size_t)a * nw + W.tri[3 * m + v]] += area * nrm[(size_t)a * mt + m];
    }
    for (int n = 0; n < nw; ++n) {
      const double x = acc[n], y = acc[(size_t)nw + n], z = acc[2 * (size_t)nw + n];
      const double l = std::sqrt(x * x + y * y + z * z);
      if (l > 0)
        for (int a = 0; a < 3; ++a) W.nnrm[(size_t)a * nw + n] = (float)(acc[(size_t)a * nw + n] / l);
    }
  }
  // bounding radius of each node's candidates (the vertices and centroids of
  // its listed triangles): lets a search skip a node whose candidates are all
  // farther than a distance already reached
  W.rad.assign(nw, 0.f);
  for (int n = 0; n < nw; ++n) {
    const int32_t* L = &W.ntri[(size_t)n * (cap + 1)];
    double r2 = 0.0;
    for (int l = 1; l <= L[0]; ++l) {
      const int t = L[l];
      for (int v = 0; v < 4; ++v) {
        double d2 = 0.0;
        for (int a = 0; a < 3; ++a) {
          const double q = v < 3 ? xyz[(size_t)a * nw + W.tri[3 * (size_t)t + v]] : W.cen[(size_t)a * mt + t];
          const double e = q - xyz[(size_t)a * nw + n];
          d2 += e * e;
        }
        r2 = std::max(r2, d2);
      }
    }
    W.rad[n] = (float)(std::sqrt(r2) * (1.0 + 1e-6) + 1e-5);
  }
  // W_index / Wdistance over the lattice box
  const int64_t npts = (int64_t)nx * ny * nz;
  W.windex.assign(npts, 0);
  W.wdist.assign(npts, 5000.f);
  for (int m = 0; m < nw; ++m) {
    const float xc = xyz[m], yc = xyz[(size_t)nw + m], zc = xyz[2 * (size_t)nw + m];
    const int i = (int)std::floor((xc - X0) / DX + 0.01), j = (int)std::floor((yc - Y0) / DX + 0.01),
              k = (int)std::floor((zc - Z0) / DX + 0.01);
    const int i1 = std::max(i - 4, 0), i2 = std::min(i + 4, nx - 1);
    const int j1 = std::max(j - 4, 0), j2 = std::min(j + 4, ny - 1);
    const int k1 = Lz > 0 ? k - 4 : std::max(k - 4, 0), k2 = Lz > 0 ? k + 4 : std::min(k + 4, nz - 1);
    for (int ii = i1; ii <= i2; ++ii)
      for (int jj = j1; jj <= j2; ++jj)
        for (int kk = k1; kk <= k2; ++kk) {
          const int kw = ((kk % nz) + nz) % nz;
          const float dx = (float)(X0 + ii * DX) - xc, dy = (float)(Y0 + jj * DX) - yc;
          const float dz = (float)mind((Z0 + kw * DX) - zc, Lz);
          const float d = sqrtf(dx * dx + dy * dy + dz * dz);
          const int64_t p = ((int64_t)ii * ny + jj) * nz + kw;
          if (d < W.wdist[p]) {
            W.wdist[p] = d;
            W.windex[p] = m + 1;  // 1-based as the reference; 0 = none
          }
        }
  }
  // void velocity at non-fluid points near the wall
  W.uvoid.clear();
  for (int64_t p = 0; p < npts; ++p) {
    const int m1 = W.windex[p];
    if (m1 <= 0 || c->b_index[p] > 0) continue;
    const int i = (int)(p / ((int64_t)ny * nz)), j = (int)((p / nz) % ny), k = (int)(p % nz);
    const float xp = (float)(X0 + i * DX), yp = (float)(Y0 + j * DX), zp = (float)(Z0 + k * DX);
    const int32_t* L = &W.ntri[(size_t)(m1 - 1) * (cap + 1)];
    float best = 5000.f;
    int tw = -1;
    for (int l = 1; l <= L[0]; ++l) {
      const int t = L[l];
      for (int v = 0; v < 4; ++v) {
        float px, py, pz;
        if (v < 3) {
          const int n = W.tri[3 * (size_t)t + v];
          px = xyz[n];
          py = xyz[(size_t)nw + n];
          pz = xyz[2 * (size_t)nw + n];
        } else {
          px = W.cen[t];
          py = W.cen[(size_t)mt + t];
          pz = W.cen[2 * (size_t)mt + t];
        }
        const float dx = xp - px, dy = yp - py, dz = (float)mind(zp - pz, Lz);
        const float d = sqrtf(dx * dx + dy * dy + dz * dz);
        if (d < best) {
          best = d;
          tw = t;
        }
      }
    }
    if (tw < 0) continue;
    const float wd = W.wdist[p];
    const float w1 = wd <= 0.7f ? 0.f : (wd <= 3.f ? (wd - 0.7f) / (3.f - 0.7f) : 1.f);
    if (w1 == 0.f) continue;
    const float s = (float)(w1 * 1.e-03 / P.vel_scale);
    VoidPoint vp;
    vp.p = p;
    for (int a = 0; a < 3; ++a) vp.u[a] = s * nrm[(size_t)a * mt + tw];
    W.uvoid.push_back(vp);
  }
  return ZF_OK;
}

}  // namespace zf

// ---- generators ---------------------------------------------------------------

namespace {

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

// Cylinder wall of radius R (lattice units) around the lattice axis (cx, cy),
// along z over nz lattice spacings, in um with the lattice origin/spacing;
// rings every `h` lattice units, `nseg` segments around; inward normals.
// The band that would close the periodic seam is left open.  With NULL
// outputs only the sizes are returned.
int zf_gen_wall_tube(double cx, double cy, double R, int nz, double h, int nseg,
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
int zf_gen_wall_bifurcation(int nx, int ny, int nz, double Rp, double Rd, double half_angle_deg,
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

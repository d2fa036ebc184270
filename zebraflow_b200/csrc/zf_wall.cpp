// Vessel wall meshes: the host set-up of the wall data the IB kernels read.
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

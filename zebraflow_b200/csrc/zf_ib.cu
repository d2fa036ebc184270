// Immersed-boundary coupling and cell interactions, one membrane step.
//
//   k_ib_interp     velocity interpolation (Peskin cosine delta, spherical
//                   support of 2 lattice units, not renormalised) of the fluid
//                   velocity, or of the void velocity at non-fluid points near
//                   the wall, plus nearest-wall-triangle search and wall
//                   repulsion                       ZebraflowWT.c:8690-9142, :9149-9430
//   k_bin_*         cell list: each triangle centroid binned to its nearest
//                   listed lattice point within 1 um (the reference's Eulerian
//                   lists EulNeigh, :5857-5902), as a CSR over lattice slots
//   k_nuc_memb      nucleus-membrane repulsion over per-node triangle lists
//                   rebuilt every nuc_list_period iterations  :9516-9730
//   k_rbc_rbc       membrane node vs. facing triangles of any cell (16 sub-
//                   triangle centroids)                :9911-10053
//   k_ib_spread     force spreading with the same delta into BODYFORCE
//                                                      :10737-10870, :10874-10990
//   k_update        explicit Euler position update and the speed check that
//                   removes a cell                     :11965-12031
// Positions and node velocities are fp64 as in the reference; distances and
// weights are fp32 on fp32 copies of the positions, as the reference's float
// locals.  Sums of distances that pick a nearest triangle use non-contracted
// fp32 operations so that ties resolve as on the CPU.
#include <algorithm>
#include <climits>

#include "zf_internal.h"

namespace zf {

namespace {

// warps per block of the queue-based search kernels
constexpr int kRepWarps = 4;

__device__ __forceinline__ float dist3(float dx, float dy, float dz) {
  return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}
__device__ __forceinline__ float wrapd(float d, float L) {
  if (L > 0.f) {
    if (d > 0.5f * L) d -= L;
    else if (d < -0.5f * L) d += L;
  }
  return d;
}

// 0-based lattice index of a coordinate as the reference computes its 1-based
// one: (int)((x - x0)/DX + 1.01) - 1, with floor for coordinates below x0.
__device__ __forceinline__ int lat_index(float x, double x0, double dx) {
  return (int)floor(((double)x - x0) / dx + 1.01) - 1;
}
__device__ __forceinline__ int wrapk(const IbArgs& a, int k) {
  return a.per_z ? ((k % a.nz) + a.nz) % a.nz : k;
}

// slot of lattice point (i,j,k), k already wrapped; -1 when no tile holds it
__device__ __forceinline__ int64_t slot_of(const IbArgs& a, int i, int j, int k) {
  const int t = a.tile_map[((k >> 2) * a.nty + (j >> 2)) * a.ntx + (i >> 2)];
  if (t < 0) return -1;
  return (int64_t)t * ZF_TC + (i & 3) + 4 * (j & 3) + 16 * (k & 3);
}

// The Peskin stencil of a node (ZebraflowWT.c:8963-8996 interpolation,
// :10806-10866 spreading): of the reference's +-4 window only the 4 lattice
// points b..b+3 per axis around the node can lie within the support radius
// 2 DX (StencilWidth*DX).  The cosine delta is a product of one factor per
// axis, so the factors are formed once per axis point -- 12 cosines per node
// instead of 3 per stencil point -- each as the reference forms it: the
// offset d = x_lattice - x_node in float, the cosine of PI |d| / (2 DX) with
// its argument in double (PI is a double literal there), and the product
// (1 + cx)(1 + cy)(1 + cz) / 64 in double.  The distance test keeps the
// reference's float sqrtf of the summed float squares.
constexpr double kPId = 3.14159265358979;  // PI, ZebraflowWT.c:34

struct StencilAxis {
  int b;        // first lattice index along the axis
  unsigned ok;  // bit m: point b + m lies in the box and in the node's +-4 window
  float s[4];   // d^2
  float c[4];   // cosf(PI |d| / (2 DX))
};

// lo, hi: the box's index range along the axis; i0: the node's lattice index
__device__ __forceinline__ void stencil_axis(StencilAxis& ax, float xp, double x0, double dx, int lo, int hi,
                                             int i0) {
  ax.b = (int)floor(((double)xp - x0) / dx) - 1;
  ax.ok = 0u;
  const double h2 = 2.0 * dx;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int i = ax.b + m;
    if (i >= lo && i <= hi && i >= i0 - 4 && i <= i0 + 4) ax.ok |= 1u << m;
    const float d = (float)(x0 + i * dx) - xp;
    ax.s[m] = __fmul_rn(d, d);
    ax.c[m] = cosf((float)(kPId * (double)fabsf(d) / h2));
  }
}

// entry m of a 4-array held in registers (m not a compile-time constant)
__device__ __forceinline__ float sel4(const float (&v)[4], int m) {
  return m < 2 ? (m == 0 ? v[0] : v[1]) : (m == 2 ? v[2] : v[3]);
}

// Walks the stencil points of a node in the reference's i, j, k order and
// calls fn(i, j, k, w) for those within the support radius, w > 0 in double:
// (1 + cx)(1 + cy)(1 + cz) / 64, the three factors multiplied left to right.
template <class Fn>
__device__ __forceinline__ void stencil_walk(const StencilAxis& X, const StencilAxis& Y, const StencilAxis& Z,
                                             float h2, Fn&& fn) {
  for (int mi = 0; mi < 4; ++mi) {
    if (!((X.ok >> mi) & 1u)) continue;
    const float sx = sel4(X.s, mi);
    const double fx = 1.0 + (double)sel4(X.c, mi);
    for (int mj = 0; mj < 4; ++mj) {
      if (!((Y.ok >> mj) & 1u)) continue;
      const float sxy = __fadd_rn(sx, sel4(Y.s, mj));
      const double fxy = fx * (1.0 + (double)sel4(Y.c, mj));
#pragma unroll
      for (int mk = 0; mk < 4; ++mk) {
        if (!((Z.ok >> mk) & 1u)) continue;
        if (!(sqrtf(__fadd_rn(sxy, Z.s[mk])) <= h2)) continue;
        const double w = fxy * (1.0 + (double)Z.c[mk]) / 64.0;
        if (w > 0.0) fn(X.b + mi, Y.b + mj, Z.b + mk, w);
      }
    }
  }
}

__device__ __forceinline__ void node_stencil(const IbArgs& a, float xp, float yp, float zp, StencilAxis& X,
                                             StencilAxis& Y, StencilAxis& Z) {
  const int i0 = lat_index(xp, a.X0, a.DX), j0 = lat_index(yp, a.Y0, a.DX), k0 = lat_index(zp, a.Z0, a.DX);
  stencil_axis(X, xp, a.X0, a.DX, 0, a.nx - 1, i0);
  stencil_axis(Y, yp, a.Y0, a.DX, 0, a.ny - 1, j0);
  stencil_axis(Z, zp, a.Z0, a.DX, a.kmin, a.kmax, k0);
}

struct NodeRef {
  double* x;      // [3][nc][n] positions
  int n;          // nodes per cell of this kind
};

__device__ __forceinline__ void node_pos(const double* x, int nc, int n, int cell, int node,
                                         float LZ, double Z0, float& xp, float& yp, float& zp) {
  xp = (float)x[((size_t)0 * nc + cell) * n + node];
  yp = (float)x[((size_t)1 * nc + cell) * n + node];
  double z = x[((size_t)2 * nc + cell) * n + node];
  if (LZ > 0.f) z -= (double)LZ * floor((z - (double)Z0) / (double)LZ);
  zp = (float)z;
}

}  // namespace

// One thread per node: membrane nodes of all cells, then nucleus nodes.
__global__ void k_ib_interp(IbArgs a, CellArgs c) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  const int64_t nmem = (int64_t)nc * c.nn;
  const bool nuc = gid >= nmem;
  if (gid >= nmem + (int64_t)nc * c.nnn) return;
  const int n = nuc ? c.nnn : c.nn;
  const int64_t lid = nuc ? gid - nmem : gid;
  const int cell = (int)(lid / n), node = (int)(lid % n);
  if (a.wall_tri) a.wall_tri[gid] = -1;  // the wall search that follows sets it
  if (c.status[cell] <= 0) return;
  const double* X = nuc ? c.xn : c.x;
  float xp, yp, zp;
  node_pos(X, nc, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
  const float h2 = 2.f * a.DX;
  StencilAxis SX, SY, SZ;
  node_stencil(a, xp, yp, zp, SX, SY, SZ);
  if (SZ.b + 3 < a.own_k0 || SZ.b >= a.own_k1) return;  // no owned plane in reach

  // velocity interpolation over the 4x4x4 stencil points, in the reference's
  // i, j, k order; fluid points give U, V, W, non-fluid points with a wall
  // index the void velocity (on a slab of a split lattice: the owned planes
  // only, the other slabs add the rest)
  double vx = 0.0, vy = 0.0, vz = 0.0;
  stencil_walk(SX, SY, SZ, h2, [&](int i, int j, int k, double w) {
    if (k < a.own_k0 || k >= a.own_k1) return;
    const int64_t s = slot_of(a, i, j, wrapk(a, k));
    if (s < 0) return;
    const uint8_t cd = a.code[s];
    const bool fluid = zf_code_fluid(cd) || zf_code_pressure(cd);  // 0 < B_index < 4998
    if (!fluid && a.windex[s] <= 0) return;
    float u, v, ww;
    if (fluid) {
      u = a.mom[a.ns + s];
      v = a.mom[2 * a.ns + s];
      ww = a.mom[3 * a.ns + s];
    } else {
      u = a.uvoid[s];
      v = a.uvoid[a.ns_all + s];
      ww = a.uvoid[2 * a.ns_all + s];
    }
    vx += w * (double)(a.vel_scale * u);
    vy += w * (double)(a.vel_scale * v);
    vz += w * (double)(a.vel_scale * ww);
  });
  double* V = nuc ? c.vel_n : c.vel;
  V[((size_t)0 * nc + cell) * n + node] += vx;
  V[((size_t)1 * nc + cell) * n + node] += vy;
  V[((size_t)2 * nc + cell) * n + node] += vz;
}

// Nearest wall triangle over the +-4 window in the reference scan order
// (ZebraflowWT.c:8998-9053) and the wall repulsion (:9055-9077), one thread
// per node as k_ib_interp.  The first candidate point (vertex or centroid of a
// triangle listed at a wall node) that reaches the window's minimum decides,
// so lists that cannot reach it change nothing: a wall node met again (same
// candidates) is skipped, and so is one whose candidates all lie farther than
// a distance some candidate of the window already reached
// (|node - m| - rad[m] > bound).  Lanes walk their windows in lock-step and
// queue the lists that remain; a batch scans 32 lists, one per lane, each
// giving its first minimum, and the owner folds them in its scan order with a
// strict <, which is the reference's running minimum taken list by list.
__device__ __forceinline__ void wall_list_min(const IbArgs& a, int nodewall, float xp, float yp, float zp,
                                              float& best, int& tbest) {
  // the node's candidates, stored contiguously in list order: for each listed
  // triangle its 3 vertices and its centroid (x, y, z, triangle id)
  const int32_t c0 = a.wcand_off[nodewall - 1], c1 = a.wcand_off[nodewall];
  for (int i = c0; i < c1; ++i) {
    const float4 p = a.wcand[i];
    const float d = dist3(xp - p.x, yp - p.y, wrapd(zp - p.z, a.LZ));
    if (d < best) {
      best = d;
      tbest = __float_as_int(p.w);
    }
  }
}

__global__ void __launch_bounds__(kRepWarps * 32) k_ib_wall(IbArgs a, CellArgs c) {
  __shared__ int sq_m[kRepWarps][64];
  __shared__ unsigned char sq_l[kRepWarps][64];
  __shared__ float sq_d[kRepWarps][32];
  __shared__ int sq_t[kRepWarps][32];
  const unsigned FULL = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  const int64_t nmem = (int64_t)nc * c.nn;
  const bool nuc = gid >= nmem;
  bool active = gid < nmem + (int64_t)nc * c.nnn;
  const int n = nuc ? c.nnn : c.nn;
  const int64_t lid = nuc ? gid - nmem : gid;
  int cell = 0, node = 0;
  if (active) {
    cell = (int)(lid / n);
    node = (int)(lid % n);
    active = c.status[cell] > 0;
  }
  float xp = 0.f, yp = 0.f, zp = 0.f;
  int i0 = 0, j0 = 0, k0 = 0, i1 = 0, i2 = -1, j1 = 0, j2 = -1, k1 = 0, k2 = -1;
  if (active) {
    node_pos(nuc ? c.xn : c.x, nc, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
    i0 = lat_index(xp, a.X0, a.DX);
    j0 = lat_index(yp, a.Y0, a.DX);
    k0 = lat_index(zp, a.Z0, a.DX);
    if (k0 < a.own_k0 || k0 >= a.own_k1) active = false;  // another slab's node
    i1 = max(i0 - 4, 0);
    i2 = min(i0 + 4, a.nx - 1);
    j1 = max(j0 - 4, 0);
    j2 = min(j0 + 4, a.ny - 1);
    k1 = max(k0 - 4, a.kmin);
    k2 = min(k0 + 4, a.kmax);
    // skip the walk when no tile of the window holds a point with W_index > 0
    bool any = false;
    for (int ti = i1 >> 2; ti <= (i2 >> 2) && !any; ++ti)
      for (int tj = j1 >> 2; tj <= (j2 >> 2) && !any; ++tj)
        for (int k = k1; k <= k2 && !any; ++k) {
          if (k != k1 && (k & 3) != 0) continue;  // first point of each z tile
          const int kw = wrapk(a, k);
          const int t = a.tile_map[((kw >> 2) * a.nty + tj) * a.ntx + ti];
          if (t >= 0 && a.tile_wall[t]) any = true;
        }
    active = any;
  }
  // an upper bound of the window minimum: the node's own lattice point's list
  float bound = 1.5f;
  if (active && i0 >= i1 && i0 <= i2 && j0 >= j1 && j0 <= j2 && k0 >= k1 && k0 <= k2) {
    const int64_t s = slot_of(a, i0, j0, wrapk(a, k0));
    if (s >= 0 && a.windex[s] > 0) {
      int unused = -1;
      wall_list_min(a, a.windex[s], xp, yp, zp, bound, unused);
    }
  }
  // walk of the window: columns (i, j), runs of z points inside one tile
  int ci = i1, cj = j1, ck = k1, r = 0, rn = -1;
  int64_t s0 = 0;
  auto next_run = [&]() -> bool {
    while (true) {
      if (ck > k2) {
        ck = k1;
        if (++cj > j2) {
          cj = j1;
          if (++ci > i2) return false;
        }
      }
      const int kw = wrapk(a, ck);
      int run = min(k2 - ck, 3 - (kw & 3));
      if (a.per_z) run = min(run, a.nz - 1 - kw);
      ck += run + 1;
      const int t = a.tile_map[((kw >> 2) * a.nty + (cj >> 2)) * a.ntx + (ci >> 2)];
      if (t < 0 || !a.tile_wall[t]) continue;
      s0 = (int64_t)t * ZF_TC + (ci & 3) + 4 * (cj & 3) + 16 * (kw & 3);
      r = 0;
      rn = run;
      return true;
    }
  };
  bool done = !(active && i1 <= i2 && j1 <= j2 && k1 <= k2);
  if (!done) done = !next_run();
  float mindis = 1.5f;
  int triwall = -1, last = 0, qn = 0;
  const unsigned below = (1u << lane) - 1u;
  auto batch = [&](int nb) {
    __syncwarp();
    const int my = lane < nb ? sq_m[w][lane] : 0;
    const int owner = lane < nb ? (int)sq_l[w][lane] : 0;
    const float ox = __shfl_sync(FULL, xp, owner), oy = __shfl_sync(FULL, yp, owner),
                oz = __shfl_sync(FULL, zp, owner);
    float d = 3.0e38f;
    int t = -1;
    if (my > 0) wall_list_min(a, my, ox, oy, oz, d, t);
    sq_d[w][lane] = d;
    sq_t[w][lane] = t;
    __syncwarp();
    for (int q = 0; q < nb; ++q)
      if (sq_l[w][q] == lane && sq_d[w][q] < mindis) {
        mindis = sq_d[w][q];
        triwall = sq_t[w][q];
      }
    __syncwarp();
  };
  while (__any_sync(FULL, !done)) {
    int item = 0;
    if (!done) {
      const float4 wn = a.wnode[s0 + 16 * r];
      if (wn.w >= 0.f) {
        const float dm = dist3(xp - wn.x, yp - wn.y, wrapd(zp - wn.z, a.LZ));
        if (!(dm - wn.w > fminf(bound, mindis) + 1e-4f)) {
          const int nodewall = a.windex[s0 + 16 * r];
          if (nodewall != last) {
            last = nodewall;
            item = nodewall;
          }
        }
      }
      if (++r > rn) done = !next_run();
    }
    const unsigned bal = __ballot_sync(FULL, item > 0);
    if (item > 0) {
      const int pos = qn + __popc(bal & below);
      sq_m[w][pos] = item;
      sq_l[w][pos] = (unsigned char)lane;
    }
    qn += __popc(bal);
    if (qn >= 32) {
      batch(32);
      const int rem = qn - 32;
      int tm = 0, tl = 0;
      if (lane < rem) {
        tm = sq_m[w][32 + lane];
        tl = sq_l[w][32 + lane];
      }
      __syncwarp();
      if (lane < rem) {
        sq_m[w][lane] = tm;
        sq_l[w][lane] = (unsigned char)tl;
      }
      qn = rem;
    }
  }
  if (qn > 0) batch(qn);
  if (!active) return;
  if (triwall < 0) return;
  if (a.wall_tri) a.wall_tri[gid] = triwall;  // for the adjoint
  // signed distance to the plane of the wall triangle, repulsion, :9055-9077
  const int w1 = a.wtri[3 * triwall];
  const float n0 = a.wnrm[triwall], n1 = a.wnrm[a.mt + triwall], n2 = a.wnrm[2 * a.mt + triwall];
  const float ddx = xp - a.wxyz[w1], ddy = yp - a.wxyz[a.nw + w1],
              ddz = wrapd(zp - a.wxyz[2 * a.nw + w1], a.LZ);
  const float dist = __fadd_rn(__fadd_rn(__fmul_rn(ddx, n0), __fmul_rn(ddy, n1)), __fmul_rn(ddz, n2));
  if (dist < 0.25f && fabsf(dist) < 1.0f) {
    float repulf = (float)((0.25 - (double)dist) / 1.0);
    if (dist < -0.75f) repulf = 1.f;
    // nucleus nodes add to the membrane array at their own index, as the
    // reference does (ZebraflowWT.c:9415-9430 write NODE_WALLREPUL[v][caps][node])
    float* R = c.wrep;
    const int tn = node;
    if (nuc && tn >= c.nn) return;
    atomicAdd(&R[((size_t)0 * nc + cell) * c.nn + tn], (float)((double)repulf * 1.e-04 * n0));
    atomicAdd(&R[((size_t)1 * nc + cell) * c.nn + tn], (float)((double)repulf * 1.e-04 * n1));
    atomicAdd(&R[((size_t)2 * nc + cell) * c.nn + tn], (float)((double)repulf * 1.e-04 * n2));
  }
}

// ---- cell list of triangle centroids ----------------------------------------

// bin key of a population slot: the tile's 64 points with z fastest, so the
// points of one (x, y) column of a tile have consecutive keys
__device__ __forceinline__ int64_t bin_key(int64_t s) {
  const int c = (int)(s & 63);
  return (s & ~(int64_t)63) | (((c >> 4) & 3) + 4 * ((c >> 2) & 3) + 16 * (c & 3));
}

// bin of each triangle: the nearest listed lattice point within 1 um of its
// centroid inside the reference window (:5857-5902), or -1.  Only points
// within 2 lattice units per axis can lie within 1 um (2 DX), and the first
// minimum of the reference scan is the first minimum of any sub-scan in the
// same order that holds every point within 1 um, so the scan covers +-2.
__global__ void k_bin_assign(IbArgs a, CellArgs c, int32_t* tri_bin, int32_t* counts) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  if (g >= (int64_t)nc * c.nt) return;
  const int cell = (int)(g / c.nt), t = (int)(g % c.nt);
  tri_bin[g] = -1;
  if (c.status[cell] > 0) {
    const float xp = c.tri_c[((size_t)0 * nc + cell) * c.nt + t];
    const float yp = c.tri_c[((size_t)1 * nc + cell) * c.nt + t];
    const float zraw = c.tri_c[((size_t)2 * nc + cell) * c.nt + t];
    float zp = zraw;
    bool in = true;
    if (a.LZ > 0.f) zp = (float)((double)zp - (double)a.LZ * floor(((double)zp - a.Z0) / a.LZ));
    else in = !(zp < a.Z0 || zp > a.Z0 + (a.nz - 1) * a.DX);
    float mindis = 5000.f;
    int64_t best = -1;
    if (in) {
      const int i0 = lat_index(xp, a.X0, a.DX), j0 = lat_index(yp, a.Y0, a.DX),
                k0 = lat_index(zp, a.Z0, a.DX);
      const int i1 = max(i0 - 2, 0), i2 = min(i0 + 2, a.nx - 1);
      const int j1 = max(j0 - 2, 0), j2 = min(j0 + 2, a.ny - 1);
      const int k1 = a.per_z ? k0 - 2 : max(k0 - 2, 2), k2 = a.per_z ? k0 + 2 : min(k0 + 2, a.nz - 4);
      auto listed = [&](int i, int j, int k) -> int64_t {
        const int kw = a.per_z ? ((k % a.nz) + a.nz) % a.nz : k;
        const int64_t s = slot_of(a, i, j, kw);
        return (s < 0 || s >= a.ns || a.code[s] == 0) ? (int64_t)-1 : s;
      };
      auto scan = [&](int ia, int ib, int ja, int jb, int ka, int kb) {
        for (int i = ia; i <= ib; ++i)
          for (int j = ja; j <= jb; ++j)
            for (int k = ka; k <= kb; ++k) {
              const int64_t s = listed(i, j, k);  // listed points only
              if (s < 0) continue;
              const float xc = (float)((double)a.X0 + i * (double)a.DX);
              const float yc = (float)((double)a.Y0 + j * (double)a.DX);
              const float zc = (float)((double)a.Z0 + k * (double)a.DX);
              const float d = dist3(xc - xp, yc - yp, zc - zp);
              if (d < mindis) {
                mindis = d;
                best = s;
              }
            }
      };
      // the lattice point nearest the centroid: when it is listed, every
      // point as near or nearer (ties included) is one of its 27 neighbours,
      // so the first minimum of the window scan lies among them
      const int ic = (int)floor(((double)xp - a.X0) / a.DX + 0.5), jc = (int)floor(((double)yp - a.Y0) / a.DX + 0.5),
                kc = (int)floor(((double)zp - a.Z0) / a.DX + 0.5);
      if (ic >= i1 && ic <= i2 && jc >= j1 && jc <= j2 && kc >= k1 && kc <= k2 && listed(ic, jc, kc) >= 0)
        scan(max(ic - 1, i1), min(ic + 1, i2), max(jc - 1, j1), min(jc + 1, j2), max(kc - 1, k1), min(kc + 1, k2));
      else
        scan(i1, i2, j1, j2, k1, k2);
    }
    if (best >= 0 && mindis < 1.f) {
      const int64_t key = bin_key(best);
      tri_bin[g] = (int32_t)key;
      atomicAdd(&counts[key], 1);
    }
  }
}

// exclusive scan of counts[0..n) into off[0..n], three passes
__global__ void k_scan_blocks(const int32_t* in, int64_t n, int32_t* out, int32_t* bsum) {
  __shared__ int32_t sh[1024];
  const int64_t i = (int64_t)blockIdx.x * 1024 + threadIdx.x;
  int32_t v = i < n ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int32_t t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = sh[threadIdx.x] - v;
  if (threadIdx.x == 1023) bsum[blockIdx.x] = sh[1023];
}
// exclusive scan of the nb block sums in place, *total their sum: one block
// of 1024 threads, 1024 sums per round (warp scans, then a scan of the 32
// warp totals), the running total carried between rounds
__global__ void __launch_bounds__(1024) k_scan_sums(int32_t* bsum, int nb, int32_t* total) {
  __shared__ int32_t s_w[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t carry = 0;
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + (int)threadIdx.x;
    const int32_t v = i < nb ? bsum[i] : 0;
    int32_t x = v;  // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
      int32_t t = s_w[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      s_w[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const int32_t before = carry + (w > 0 ? s_w[w - 1] : 0) + x - v;
    if (i < nb) bsum[i] = before;
    carry += s_w[31];
    __syncthreads();  // s_w is rewritten by the next round
  }
  if (threadIdx.x == 0) *total = carry;
}
__global__ void k_scan_add(int32_t* out, int64_t n, const int32_t* bsum) {
  const int64_t i = (int64_t)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += bsum[blockIdx.x];
}

__global__ void k_bin_fill(CellArgs c, const int32_t* tri_bin, const int32_t* off, int32_t* cursor,
                           int32_t* bin_tri, uint8_t* bin_kk) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)c.n_cells * c.nt) return;
  const int32_t b = tri_bin[g];
  if (b < 0) return;
  const int pos = atomicAdd(&cursor[b], 1);
  bin_tri[off[b] + pos] = (int32_t)g;
  bin_kk[off[b] + pos] = (uint8_t)(b & 63);
}

// deterministic order inside each bin (ascending global triangle id)
__global__ void k_bin_sort(const int32_t* off, int64_t ns, int32_t* bin_tri) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const int b0 = off[s], b1 = off[s + 1];
  for (int i = b0 + 1; i < b1; ++i) {
    const int32_t v = bin_tri[i];
    int j = i - 1;
    while (j >= b0 && bin_tri[j] > v) {
      bin_tri[j + 1] = bin_tri[j];
      --j;
    }
    bin_tri[j + 1] = v;
  }
}

// The w word of a bin record holds the entry's key inside its tile (low 8
// bits) and the bounding radius rounded up to 2^-20 um (high 24 bits).
__device__ __forceinline__ float rec_pack(int kk, float rb) {
  const unsigned q = min((unsigned)ceilf(rb * 1048576.f), 0xffffffu);
  return __uint_as_float((q << 8) | (unsigned)kk);
}
__device__ __forceinline__ int rec_kk(float w) { return (int)(__float_as_uint(w) & 0xffu); }
__device__ __forceinline__ float rec_rb(float w) { return (float)(__float_as_uint(w) >> 8) * (1.f / 1048576.f); }

// per bin entry: centroid and bounding radius, normal and triangle id (one
// 32-byte record), and the three vertices (fp32 of the fp64 positions, with their node ids), so the
// repulsion search reads one contiguous range of records per run of bins and
// evaluates a triangle from its own record.  The radius bounds the distance from the centroid to any point of the
// triangle (the vertices, as float), with a margin for float rounding.
__global__ void k_bin_records(IbArgs a, CellArgs c, const int32_t* total) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= *total) return;
  const int nc = c.n_cells;
  const int g = a.bin_tri[e];
  const int m = g / c.nt, tri = g - m * c.nt;
  const float cx = c.tri_c[((size_t)0 * nc + m) * c.nt + tri];
  const float cy = c.tri_c[((size_t)1 * nc + m) * c.nt + tri];
  const float cz = c.tri_c[((size_t)2 * nc + m) * c.nt + tri];
  float r2 = 0.f;
  for (int v = 0; v < 3; ++v) {
    const int n = c.tri[3 * tri + v];
    const float dx = (float)c.x[((size_t)0 * nc + m) * c.nn + n] - cx;
    const float dy = (float)c.x[((size_t)1 * nc + m) * c.nn + n] - cy;
    const float dz = (float)c.x[((size_t)2 * nc + m) * c.nn + n] - cz;
    r2 = fmaxf(r2, dx * dx + dy * dy + dz * dz);
  }
  a.bin_rec[2 * e] = make_float4(cx, cy, cz, rec_pack(a.bin_kk[e], sqrtf(r2) * 1.0001f + 1e-3f));
  const int64_t stride = (int64_t)nc * c.nt;
  for (int v = 0; v < 3; ++v) {
    const int n = c.tri[3 * tri + v];
    a.bin_v[v * stride + e] = make_float4((float)c.x[((size_t)0 * nc + m) * c.nn + n],
                                          (float)c.x[((size_t)1 * nc + m) * c.nn + n],
                                          (float)c.x[((size_t)2 * nc + m) * c.nn + n], __int_as_float(n));
  }
  a.bin_rec[2 * e + 1] = make_float4(c.tri_nrm[((size_t)0 * nc + m) * c.nt + tri],
                           c.tri_nrm[((size_t)1 * nc + m) * c.nt + tri],
                           c.tri_nrm[((size_t)2 * nc + m) * c.nt + tri], __int_as_float(g));
}

// ---- nucleus-membrane repulsion --------------------------------------------

__global__ void k_nuc_memb(IbArgs a, CellArgs c, int rebuild, unsigned long long* overflow) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  if (gid >= (int64_t)nc * c.nnn) return;
  const int cell = (int)(gid / c.nnn), node = (int)(gid % c.nnn);
  if (c.status[cell] <= 0) return;
  const float xc = (float)c.xn[((size_t)0 * nc + cell) * c.nnn + node];
  const float yc = (float)c.xn[((size_t)1 * nc + cell) * c.nnn + node];
  const float zc = (float)c.xn[((size_t)2 * nc + cell) * c.nnn + node];
  const float* TC = c.tri_c;
  const size_t tb = (size_t)cell * c.nt;
  uint16_t* list = a.nuc_list + (size_t)gid * a.nuc_cap;
  if (rebuild) {  // own triangles with centroid within 0.5 um, :9530-9590
    int l = 0;
    for (int m = 0; m < c.nt; ++m) {
      const float d = dist3(xc - TC[(size_t)0 * nc * c.nt + tb + m], yc - TC[(size_t)1 * nc * c.nt + tb + m],
                            zc - TC[(size_t)2 * nc * c.nt + tb + m]);
      if (d < 0.5f) {
        if (l < a.nuc_cap) list[l++] = (uint16_t)m;
        else atomicAdd(overflow, 1ull);
      }
    }
    a.nuc_cnt[gid] = l;
  }
  if (a.own_k0 > -(1 << 30)) {  // a slab of a split lattice: the slab of the node's lattice point pushes
    float px, py, pz;
    node_pos(c.xn, nc, c.nnn, cell, node, a.LZ, a.Z0, px, py, pz);
    const int k0 = lat_index(pz, a.Z0, a.DX);
    if (k0 < a.own_k0 || k0 >= a.own_k1) return;
  }
  const int cnt = a.nuc_cnt[gid];
  for (int l = 0; l < cnt; ++l) {
    const int tri = list[l];
    const float px = TC[(size_t)0 * nc * c.nt + tb + tri], py = TC[(size_t)1 * nc * c.nt + tb + tri],
                pz = TC[(size_t)2 * nc * c.nt + tb + tri];
    if (!(dist3(xc - px, yc - py, zc - pz) < 1.f)) continue;
    const int n1 = c.tri[3 * tri], n2 = c.tri[3 * tri + 1], n3 = c.tri[3 * tri + 2];
    const float e1v[3] = {c.tri_nrm[((size_t)0 * nc + cell) * c.nt + tri],
                          c.tri_nrm[((size_t)1 * nc + cell) * c.nt + tri],
                          c.tri_nrm[((size_t)2 * nc + cell) * c.nt + tri]};
    float p1[3], p2[3], p3[3];
    for (int v = 0; v < 3; ++v) {
      p1[v] = (float)c.x[((size_t)v * nc + cell) * c.nn + n1];
      p2[v] = (float)c.x[((size_t)v * nc + cell) * c.nn + n2];
      p3[v] = (float)c.x[((size_t)v * nc + cell) * c.nn + n3];
    }
    // 19 sample points of the triangle, :9638-9687
    float tp[20][3];
    for (int v = 0; v < 3; ++v) {
      float ep[10];
      ep[1] = (p1[v] + p2[v]) / 2.f;
      ep[2] = (p2[v] + p3[v]) / 2.f;
      ep[3] = (p3[v] + p1[v]) / 2.f;
      ep[4] = (p1[v] + ep[1]) / 2.f;
      ep[5] = (ep[1] + p2[v]) / 2.f;
      ep[6] = (p2[v] + ep[2]) / 2.f;
      ep[7] = (ep[2] + p3[v]) / 2.f;
      ep[8] = (p3[v] + ep[3]) / 2.f;
      ep[9] = (ep[3] + p1[v]) / 2.f;
      tp[1][v] = (p1[v] + p2[v] + p3[v]) / 3.f;
      tp[2][v] = (ep[3] + p1[v] + ep[1]) / 3.f;
      tp[3][v] = (ep[1] + p2[v] + ep[2]) / 3.f;
      tp[4][v] = (ep[2] + p3[v] + ep[3]) / 3.f;
      tp[5][v] = (ep[1] + ep[3]) / 2.f;
      tp[6][v] = (ep[1] + ep[2]) / 2.f;
      tp[7][v] = (ep[2] + ep[3]) / 2.f;
      tp[8][v] = (p1[v] + tp[2][v]) / 2.f;
      tp[9][v] = (ep[1] + tp[2][v]) / 2.f;
      tp[10][v] = (ep[3] + tp[2][v]) / 2.f;
      tp[11][v] = (ep[1] + tp[3][v]) / 2.f;
      tp[12][v] = (p2[v] + tp[3][v]) / 2.f;
      tp[13][v] = (ep[2] + tp[3][v]) / 2.f;
      tp[14][v] = (ep[3] + tp[4][v]) / 2.f;
      tp[15][v] = (ep[2] + tp[4][v]) / 2.f;
      tp[16][v] = (p3[v] + tp[4][v]) / 2.f;
      tp[17][v] = (ep[1] + tp[1][v]) / 2.f;
      tp[18][v] = (ep[2] + tp[1][v]) / 2.f;
      tp[19][v] = (ep[3] + tp[1][v]) / 2.f;
    }
    for (int v = 1; v <= 19; ++v) {
      const float d = dist3(tp[v][0] - xc, tp[v][1] - yc, tp[v][2] - zc);
      if (d <= 0.2f) {
        float repulf = (float)((0.2 - (double)d) / 0.2);
        repulf = (float)((double)repulf * 4.1666667e-07);
        for (int i = 0; i < 3; ++i) {
          const float f = (float)((double)(repulf * e1v[i]) / 3.);
          atomicAdd(&c.wrep[((size_t)i * nc + cell) * c.nn + n1], f);
          atomicAdd(&c.wrep[((size_t)i * nc + cell) * c.nn + n2], f);
          atomicAdd(&c.wrep[((size_t)i * nc + cell) * c.nn + n3], f);
        }
      }
    }
  }
}

// ---- cell-cell repulsion ------------------------------------------------------

// Warps work on a queue: every lane walks its node's bins in the reference
// scan order and tests each entry with the cheap filters (centroid within
// 2 um, ZebraflowWT.c:9978; a sub-centroid possibly within 1 um; facing
// normals; not a triangle of the node itself).  Entries that pass go to a
// per-warp queue in shared memory; each full batch of 32 is evaluated one
// entry per lane (the 16 sub-centroids), and each owner adds its entries'
// results in its own scan order, so the sums are deterministic.

__device__ __forceinline__ void rbc_entry(const IbArgs& a, const CellArgs& c, int e, const float4 cr,
                                          float xc, float yc, float zc, float& tx, float& ty, float& tz) {
  const int64_t stride = (int64_t)c.n_cells * c.nt;
  const float4 v1 = a.bin_v[e], v2 = a.bin_v[stride + e], v3 = a.bin_v[2 * stride + e];
  const float dzc = wrapd(cr.z - zc, a.LZ);
  const float shift = (cr.z - zc) - dzc;  // periodic image of the other cell
  // the 15 points of the subdivided triangle, then the 16 sub-triangle
  // centroids one at a time (ZebraflowWT.c:9981-10027)
  float tp[16][3];
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    const float off = v == 2 ? shift : 0.f;
    tp[1][v] = (v == 0 ? v1.x : v == 1 ? v1.y : v1.z) - off;
    tp[2][v] = (v == 0 ? v2.x : v == 1 ? v2.y : v2.z) - off;
    tp[3][v] = (v == 0 ? v3.x : v == 1 ? v3.y : v3.z) - off;
    tp[4][v] = 0.5f * (tp[1][v] + tp[2][v]);
    tp[5][v] = 0.5f * (tp[2][v] + tp[3][v]);
    tp[6][v] = 0.5f * (tp[1][v] + tp[3][v]);
    tp[7][v] = 0.5f * (tp[1][v] + tp[4][v]);
    tp[8][v] = 0.5f * (tp[2][v] + tp[4][v]);
    tp[9][v] = 0.5f * (tp[2][v] + tp[5][v]);
    tp[10][v] = 0.5f * (tp[5][v] + tp[3][v]);
    tp[11][v] = 0.5f * (tp[3][v] + tp[6][v]);
    tp[12][v] = 0.5f * (tp[6][v] + tp[1][v]);
    tp[13][v] = 0.5f * (tp[4][v] + tp[6][v]);
    tp[14][v] = 0.5f * (tp[4][v] + tp[5][v]);
    tp[15][v] = 0.5f * (tp[5][v] + tp[6][v]);
  }
  // sub-triangle v = 1..16: corners (kSubA, kSubB, kSubC)[v-1]
  constexpr int kSubA[16] = {1, 7, 7, 4, 4, 8, 8, 12, 13, 13, 14, 14, 6, 15, 15, 11};
  constexpr int kSubB[16] = {7, 13, 4, 14, 8, 9, 2, 13, 15, 14, 5, 9, 15, 10, 5, 10};
  constexpr int kSubC[16] = {12, 12, 13, 13, 14, 14, 9, 6, 6, 15, 15, 5, 11, 11, 10, 3};
  // (the reference divides by 3 and by d; multiplying by 1/3 and by 1/d
  // differs in the last bit only, far below the forces' fp32 resolution)
  tx = ty = tz = 0.f;
#pragma unroll
  for (int v = 0; v < 16; ++v) {  // ZebraflowWT.c:10028-10042
    const float third = 1.f / 3.f;
    const float cx = (tp[kSubA[v]][0] + tp[kSubB[v]][0] + tp[kSubC[v]][0]) * third;
    const float cy = (tp[kSubA[v]][1] + tp[kSubB[v]][1] + tp[kSubC[v]][1]) * third;
    const float cz = (tp[kSubA[v]][2] + tp[kSubB[v]][2] + tp[kSubC[v]][2]) * third;
    const float dx = cx - xc, dy = cy - yc, dz = cz - zc;
    // dist3 without its square root unless the squared distance is below 1
    // (the square root is correctly rounded, so d < 1 implies d2 < 1; the
    // second test keeps the reference's d < 1 exactly)
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (d2 < 1.0f) {
      const float d = sqrtf(d2);
      if (d < 1.0f) {
        const float s = -8.333e-07f * (1.f - d) / d;
        tx += s * dx;
        ty += s * dy;
        tz += s * dz;
      }
    }
  }
}

__global__ void __launch_bounds__(kRepWarps * 32) k_rbc_rbc(IbArgs a, CellArgs c) {
  __shared__ int sq_e[kRepWarps][64];
  __shared__ unsigned char sq_l[kRepWarps][64];
  __shared__ float sq_r[kRepWarps][32][3];
  const unsigned FULL = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  bool active = gid < (int64_t)nc * c.nn;
  int cell = 0, node = 0;
  if (active) {
    cell = (int)(gid / c.nn);
    node = (int)(gid % c.nn);
    active = c.status[cell] > 0;
  }
  float xc = 0.f, yc = 0.f, zc = 0.f, e1x = 0.f, e1y = 0.f, e1z = 0.f;
  int i1 = 0, i2 = -1, j1 = 0, j2 = -1, k1 = 0, k2 = -1;
  if (active) {
    node_pos(c.x, nc, c.nn, cell, node, a.LZ, a.Z0, xc, yc, zc);
    e1x = c.node_normal[((size_t)0 * nc + cell) * c.nn + node];
    e1y = c.node_normal[((size_t)1 * nc + cell) * c.nn + node];
    e1z = c.node_normal[((size_t)2 * nc + cell) * c.nn + node];
    const int i0 = lat_index(xc, a.X0, a.DX), j0 = lat_index(yc, a.Y0, a.DX),
              k0 = lat_index(zc, a.Z0, a.DX);
    if (k0 < a.own_k0 || k0 >= a.own_k1) active = false;  // another slab's node
    i1 = max(i0 - 4, 0);
    i2 = min(i0 + 4, a.nx - 1);
    j1 = max(j0 - 4, 0);
    j2 = min(j0 + 4, a.ny - 1);
    k1 = a.per_z ? k0 - 4 : max(k0 - 4, 2);
    k2 = a.per_z ? k0 + 4 : min(k0 + 4, a.nz - 4);
  }
  const int64_t n_pop_tiles = a.ns / ZF_TC;
  // walk of the +-4 window: columns (i, j), runs of z points inside one tile
  int ci = i1, cj = j1, ck = k1, e = 0, e_end = 0;
  auto next_run = [&]() -> bool {
    while (true) {
      if (ck > k2) {
        ck = k1;
        if (++cj > j2) {
          cj = j1;
          if (++ci > i2) return false;
        }
      }
      const int kw = a.per_z ? ((ck % a.nz) + a.nz) % a.nz : ck;
      int run = min(k2 - ck, 3 - (kw & 3));
      if (a.per_z) run = min(run, a.nz - 1 - kw);
      ck += run + 1;
      const int t = a.tile_map[((kw >> 2) * a.nty + (cj >> 2)) * a.ntx + (ci >> 2)];
      if (t < 0 || t >= n_pop_tiles) continue;
      const int64_t key = (int64_t)t * ZF_TC + 16 * (ci & 3) + 4 * (cj & 3) + (kw & 3);
      e = a.bin_off[key];
      e_end = a.bin_off[key + run + 1];
      if (e < e_end) return true;
    }
  };
  bool done = !(active && i1 <= i2 && j1 <= j2 && k1 <= k2);
  if (!done) done = !next_run();
  float rx = 0.f, ry = 0.f, rz = 0.f;
  int qn = 0;
  const unsigned below = (1u << lane) - 1u;
  auto batch = [&](int n) {
    __syncwarp();
    const int my = lane < n ? sq_e[w][lane] : -1;
    const int owner = lane < n ? (int)sq_l[w][lane] : 0;
    const float ox = __shfl_sync(FULL, xc, owner), oy = __shfl_sync(FULL, yc, owner),
                oz = __shfl_sync(FULL, zc, owner);
    float tx = 0.f, ty = 0.f, tz = 0.f;
    if (my >= 0) rbc_entry(a, c, my, a.bin_rec[2 * my], ox, oy, oz, tx, ty, tz);
    sq_r[w][lane][0] = tx;
    sq_r[w][lane][1] = ty;
    sq_r[w][lane][2] = tz;
    __syncwarp();
    for (int q = 0; q < n; ++q)
      if (sq_l[w][q] == lane) {
        rx += sq_r[w][q][0];
        ry += sq_r[w][q][1];
        rz += sq_r[w][q][2];
      }
    __syncwarp();
  };
  while (__any_sync(FULL, !done)) {
    int item = -1;
    if (!done) {
      const float4 cr = a.bin_rec[2 * e];
      const float dzc = wrapd(cr.z - zc, a.LZ);
      const float dcen = dist3(xc - cr.x, yc - cr.y, -dzc);
      if (dcen < 2.f && !(dcen - rec_rb(cr.w) > 1.f)) {
        const float4 nr = a.bin_rec[2 * e + 1];
        if (e1x * nr.x + e1y * nr.y + e1z * nr.z < 0.f) {
          const int g = __float_as_int(nr.w);
          const int m = g / c.nt;
          bool own = false;
          if (m == cell) {
            const int tri = g - m * c.nt;
            own = c.tri[3 * tri] == node || c.tri[3 * tri + 1] == node || c.tri[3 * tri + 2] == node;
          }
          if (!own) item = e;
        }
      }
      if (++e >= e_end) done = !next_run();
    }
    const unsigned bal = __ballot_sync(FULL, item >= 0);
    if (item >= 0) {
      const int pos = qn + __popc(bal & below);
      sq_e[w][pos] = item;
      sq_l[w][pos] = (unsigned char)lane;
    }
    qn += __popc(bal);
    if (qn >= 32) {
      batch(32);
      const int rem = qn - 32;
      int te = 0, tl = 0;
      if (lane < rem) {
        te = sq_e[w][32 + lane];
        tl = sq_l[w][32 + lane];
      }
      __syncwarp();
      if (lane < rem) {
        sq_e[w][lane] = te;
        sq_l[w][lane] = (unsigned char)tl;
      }
      qn = rem;
    }
  }
  if (qn > 0) batch(qn);
  if (!active) return;
  c.wrep[((size_t)0 * nc + cell) * c.nn + node] += rx;
  c.wrep[((size_t)1 * nc + cell) * c.nn + node] += ry;
  c.wrep[((size_t)2 * nc + cell) * c.nn + node] += rz;
}

// ---- tile-cooperative searches ------------------------------------------------
//
// Nodes are grouped by the lattice tile of their nearest lattice point
// (lat_index, clamped into the box; z wrapped when periodic).  The +-4 window
// of every node of a tile then lies inside the 3x3x3 tiles around it, so a
// warp that takes a tile finds all its nodes' candidates (bin records of the
// cell list, W_index points) in those 27 tiles, which stay in L1 while it
// walks the tile's nodes.  Each test applies the node's own window exactly,
// so the candidates are the reference's.  Needs the z tiles to wrap with the
// lattice when z is periodic (nz a multiple of 4, at least three tiles);
// other periodic boxes use k_rbc_rbc and k_ib_wall.

constexpr int kTileThreads = 256;
constexpr int kTileWarps = kTileThreads / 32;

__device__ __forceinline__ int node_grid_tile(const IbArgs& a, float xp, float yp, float zp) {
  const int i0 = min(max(lat_index(xp, a.X0, a.DX), 0), a.nx - 1);
  const int j0 = min(max(lat_index(yp, a.Y0, a.DX), 0), a.ny - 1);
  const int k0 = lat_index(zp, a.Z0, a.DX);
  const int kw = a.per_z ? ((k0 % a.nz) + a.nz) % a.nz : min(max(k0, 0), a.nz - 1);
  return ((kw >> 2) * a.nty + (j0 >> 2)) * a.ntx + (i0 >> 2);
}

// node gid: membrane nodes of all cells, then nucleus nodes (as k_ib_interp)
__device__ __forceinline__ bool node_of(const CellArgs& c, int64_t gid, bool& nuc, int& cell, int& node) {
  const int64_t nmem = (int64_t)c.n_cells * c.nn;
  nuc = gid >= nmem;
  const int n = nuc ? c.nnn : c.nn;
  const int64_t lid = nuc ? gid - nmem : gid;
  cell = (int)(lid / n);
  node = (int)(lid % n);
  return c.status[cell] > 0;
}

__global__ void k_node_tiles(IbArgs a, CellArgs c) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  if (gid >= (int64_t)nc * (c.nn + c.nnn)) return;
  bool nuc;
  int cell, node;
  if (!node_of(c, gid, nuc, cell, node)) {
    a.node_gt[gid] = -1;
    return;
  }
  float xp, yp, zp;
  node_pos(nuc ? c.xn : c.x, nc, nuc ? c.nnn : c.nn, cell, node, a.LZ, a.Z0, xp, yp, zp);
  const int gt = node_grid_tile(a, xp, yp, zp);
  a.node_gt[gid] = gt;
  atomicAdd(&a.node_cnt[gt], 1);
}

__global__ void k_node_fill(IbArgs a, CellArgs c) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)c.n_cells * (c.nn + c.nnn)) return;
  const int gt = a.node_gt[gid];
  if (gt < 0) return;
  const int pos = atomicAdd(&a.node_cnt[gt], 1);
  a.node_sorted[a.node_off[gt] + pos] = (int32_t)gid;
  if (pos == 0) a.tile_list[atomicAdd(&a.tile_ctr[0], 1)] = gt;
}

// One warp per tile (taken from a work counter), no block-level barriers: the
// tile's nodes are handled one after another by the warp, and what the 27
// neighbour tiles hold is read from global memory, where it stays in L1 while
// the warp walks the tile's nodes.
__device__ __forceinline__ int warp_next_tile(int32_t* ctr, int lane) {
  int li = 0;
  if (lane == 0) li = atomicAdd(ctr, 1);
  return __shfl_sync(0xffffffffu, li, 0);
}

// neighbour r = (dz+1)*9 + (dy+1)*3 + (dx+1) of grid tile (tx, ty, tz): its
// tile id in the lattice view, -1 when outside the box or absent
__device__ __forceinline__ int neighbour_tile(const IbArgs& a, int tx, int ty, int tz, int r, int& X, int& Y,
                                              int& Z) {
  X = tx + r % 3 - 1;
  Y = ty + (r / 3) % 3 - 1;
  Z = tz + r / 9 - 1;
  if (X < 0 || X >= a.ntx || Y < 0 || Y >= a.nty) return -1;
  if (a.per_z) {
    if (Z < 0) Z += a.ntz;
    else if (Z >= a.ntz) Z -= a.ntz;
  } else if (Z < 0 || Z >= a.ntz) {
    return -1;
  }
  return a.tile_map[((int64_t)Z * a.nty + Y) * a.ntx + X];
}

// RBC-RBC repulsion (ZebraflowWT.c:9911-10053), one block per lattice tile of
// nodes.  The block stages up to kRgNodes membrane nodes of the tile, takes
// their bounding box, and walks the bin entries of the 27 tiles around it (the
// +-4 window of any node of the tile lies inside them) in their stored order,
// keeping in shared memory the triangles that some node of the box could
// reach: a sub-centroid lies within 3/4 of the bounding radius of the
// centroid, so a triangle whose centroid is farther than 1 um + 3/4 of that
// radius from the box (plus a margin for rounding) contributes to none of
// them.  Each warp then takes nodes one at a time and its lanes test the kept
// triangles against the node with the reference's conditions (bin inside the
// node's window, centroid within 2 um, facing normals, not one of the node's
// own triangles) and a disk bound (the 16 sub-centroids lie within 3/4 of the bounding radius
// of the centroid, in the triangle's plane); survivors queue up and are
// evaluated 32 at a time, one per lane (the 16 sub-centroids).  Each node's
// contributions are met in the same order whatever else the block holds, and
// lane sums meet in a fixed butterfly.
constexpr int kRgThreads = 256;
constexpr int kRgWarps = kRgThreads / 32;
constexpr int kRgNodes = 256;   // nodes staged per chunk (one per thread)
constexpr int kRgCand = 1024;   // candidate triangles held per pass

struct RgShared {
  float4 cand_c[kRgCand];   // centroid, then the squared reach bound (1 um + 3/4 radius, with margin)
  float4 cand_n[kRgCand];   // normal, global triangle id (int bits)
  int cand_w[kRgCand];      // the record's w word (in-tile key, bounding radius)
  int cand_e[kRgCand];      // bin entry (vertices in bin_v)
  int cand_xy[kRgCand];     // one-hot bin column: bit x, bit 12 + y (x, y relative to the 12^3 block)
  int cand_z[kRgCand];      // one-hot bin z: bit z
  float4 node_p[kRgNodes];  // position (z wrapped into the box), node normal |e| in w
  float4 node_n[kRgNodes];  // normal; cell id in w (int bits, -1: inactive)
  int node_wxy[kRgNodes];   // window columns: x bits 0..11, y bits 12..23
  int node_wz[kRgNodes];    // window z bits
  int node_id[kRgNodes];    // node index in its cell
  float acc[kRgNodes][3];
  int q[kRgWarps][64];
  int rng[28];              // prefix of entry counts over the 27 tiles
  int rst[27];              // first entry of each tile
  int rrel[27];             // tile offset in the 12^3 block: x | y << 8 | z << 16 (in units of 4 points)
  float bb[6];              // node box: min x, y, z, max x, y, z
  int wsum[kRgWarps];
  int wsum2[2][kRgWarps];   // per warp: kept records of a staging round (two rounds alternate)
  int li, nn, node_next;
};

__device__ __forceinline__ int onehot_range(int lo, int hi) {  // bits lo..hi of 12, clamped
  lo = max(lo, 0);
  hi = min(hi, 11);
  return lo > hi ? 0 : (int)(((2u << hi) - 1u) & ~((1u << lo) - 1u));
}

__global__ void __launch_bounds__(kRgThreads, 3) k_rbc_group(IbArgs a, CellArgs c) {
  extern __shared__ __align__(16) unsigned char rg_raw[];
  RgShared& S = *reinterpret_cast<RgShared*>(rg_raw);
  const unsigned FULL = 0xffffffffu;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nc = c.n_cells;
  const int64_t nmem = (int64_t)nc * c.nn;
  const int64_t n_pop_tiles = a.ns / ZF_TC;
  const int nlist = a.tile_ctr[0];
  for (;;) {
    if (tid == 0) S.li = atomicAdd(&a.tile_ctr[1], 1);
    __syncthreads();
    const int li = S.li;
    if (li >= nlist) break;
    const int gt = a.tile_list[li];
    const int tx = gt % a.ntx, ty = (gt / a.ntx) % a.nty, tz = gt / (a.ntx * a.nty);
    const int ox = (tx - 1) * 4, oy = (ty - 1) * 4, oz = (tz - 1) * 4;
    if (tid < 27) {
      int X, Y, Z;
      const int t = neighbour_tile(a, tx, ty, tz, tid, X, Y, Z);
      int e0 = 0, len = 0;
      if (t >= 0 && t < n_pop_tiles) {
        e0 = a.bin_off[(int64_t)t * ZF_TC];
        len = a.bin_off[(int64_t)t * ZF_TC + ZF_TC] - e0;
      }
      S.rst[tid] = e0;
      S.rng[tid + 1] = len;  // counts, scanned below
      S.rrel[tid] = (tid % 3) | (((tid / 3) % 3) << 8) | ((tid / 9) << 16);
    }
    __syncthreads();
    if (tid == 0) {
      S.rng[0] = 0;
      for (int r = 0; r < 27; ++r) S.rng[r + 1] += S.rng[r];
    }
    const int n0 = a.node_off[gt], n1 = a.node_off[gt + 1];
    for (int c0 = n0; c0 < n1; c0 += kRgNodes) {
      const int cnt = min(kRgNodes, n1 - c0);
      __syncthreads();
      // stage the chunk's membrane nodes and their box
      float px = 0.f, py = 0.f, pz = 0.f;
      bool live = false;
      if (tid < cnt) {
        const int64_t gid = a.node_sorted[c0 + tid];
        int cell = -1, node = 0;
        if (gid < nmem) {
          cell = (int)(gid / c.nn);
          node = (int)(gid % c.nn);
          if (c.status[cell] <= 0) cell = -1;
        }
        int wxy = 0, wz = 0;
        float ex = 0.f, ey = 0.f, ez = 0.f;
        if (cell >= 0) {
          node_pos(c.x, nc, c.nn, cell, node, a.LZ, a.Z0, px, py, pz);
          ex = c.node_normal[((size_t)0 * nc + cell) * c.nn + node];
          ey = c.node_normal[((size_t)1 * nc + cell) * c.nn + node];
          ez = c.node_normal[((size_t)2 * nc + cell) * c.nn + node];
          const int i0 = lat_index(px, a.X0, a.DX), j0 = lat_index(py, a.Y0, a.DX), k0 = lat_index(pz, a.Z0, a.DX);
          const int i1 = max(i0 - 4, 0), i2 = min(i0 + 4, a.nx - 1);
          const int j1 = max(j0 - 4, 0), j2 = min(j0 + 4, a.ny - 1);
          if (k0 < a.own_k0 || k0 >= a.own_k1) cell = -1;  // another slab's node
          // z unwrapped around the node's tile: window k and the block share one frame
          const int kw = a.per_z ? ((k0 % a.nz) + a.nz) % a.nz : k0;
          const int k1 = a.per_z ? kw - 4 : max(k0 - 4, 2), k2 = a.per_z ? kw + 4 : min(k0 + 4, a.nz - 4);
          wxy = onehot_range(i1 - ox, i2 - ox) | (onehot_range(j1 - oy, j2 - oy) << 12);
          wz = onehot_range(k1 - oz, k2 - oz);
          live = cell >= 0 && (wxy & 0xfff) && (wxy >> 12) && wz;
          if (!live) cell = -1;
        }
        S.node_p[tid] = make_float4(px, py, pz, sqrtf(ex * ex + ey * ey + ez * ez));
        S.node_n[tid] = make_float4(ex, ey, ez, __int_as_float(cell));
        S.node_wxy[tid] = wxy;
        S.node_wz[tid] = wz;
        S.node_id[tid] = node;
        S.acc[tid][0] = S.acc[tid][1] = S.acc[tid][2] = 0.f;
      }
      // box of the live nodes (warp reductions, then one warp over the warps)
      float mn[3] = {live ? px : 3e38f, live ? py : 3e38f, live ? pz : 3e38f};
      float mx[3] = {live ? px : -3e38f, live ? py : -3e38f, live ? pz : -3e38f};
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          mn[d] = fminf(mn[d], __shfl_xor_sync(FULL, mn[d], o));
          mx[d] = fmaxf(mx[d], __shfl_xor_sync(FULL, mx[d], o));
        }
      const int nlive = __popc(__ballot_sync(FULL, live));
      __shared__ float s_wb[kRgWarps][6];
      if (lane == 0) {
        for (int d = 0; d < 3; ++d) {
          s_wb[warp][d] = mn[d];
          s_wb[warp][3 + d] = mx[d];
        }
        S.wsum[warp] = nlive;
      }
      __syncthreads();
      if (tid < 6) {
        float v = s_wb[0][tid];
        for (int w = 1; w < kRgWarps; ++w) v = tid < 3 ? fminf(v, s_wb[w][tid]) : fmaxf(v, s_wb[w][tid]);
        S.bb[tid] = v;
      }
      if (tid == 0) {
        int t = 0;
        for (int w = 0; w < kRgWarps; ++w) t += S.wsum[w];
        S.nn = t;
      }
      __syncthreads();
      if (S.nn == 0) continue;
      const float hx = 0.5f * (S.bb[3] - S.bb[0]), hy = 0.5f * (S.bb[4] - S.bb[1]), hz = 0.5f * (S.bb[5] - S.bb[2]);
      const float mxc = S.bb[0] + hx, myc = S.bb[1] + hy, mzc = S.bb[2] + hz;
      const int total = S.rng[27];
      int ncl = 0;  // kept records held (the same in every thread)

      // the kept triangles, tested against the staged nodes
      auto process = [&]() {
        if (tid == 0) S.node_next = 0;
        __syncthreads();
        const int ncand = ncl;
        int* queue = S.q[warp];
        // nodes go to the warps as they free up (their costs differ widely)
        for (;;) {
          int t = 0;
          if (lane == 0) t = atomicAdd(&S.node_next, 1);
          t = __shfl_sync(FULL, t, 0);
          if (t >= cnt) break;
          const float4 np = S.node_p[t], nn4 = S.node_n[t];
          const int cell = __float_as_int(nn4.w);
          if (cell < 0) continue;
          const float xc = np.x, yc = np.y, zc = np.z;
          const float e1x = nn4.x, e1y = nn4.y, e1z = nn4.z;
          const int wxy = S.node_wxy[t], wz = S.node_wz[t], node = S.node_id[t];
          const int g_own = cell * c.nt;
          float rx = 0.f, ry = 0.f, rz = 0.f;
          int qn = 0;
          auto flush = [&](int nb) {
            __syncwarp();
            if (lane < nb) {
              const int e = queue[lane];
              float tx2, ty2, tz2;
              rbc_entry(a, c, e, a.bin_rec[2 * e], xc, yc, zc, tx2, ty2, tz2);
              rx += tx2;
              ry += ty2;
              rz += tz2;
            }
            const int rem = qn - nb;
            const int tq = lane < rem ? queue[nb + lane] : 0;
            __syncwarp();
            if (lane < rem) queue[lane] = tq;
            __syncwarp();
            qn = rem;
          };
          for (int k0 = 0; k0 < ncand; k0 += 32) {
            const int k = k0 + lane;
            bool pass = false;
            int e = 0;
            if (k < ncand) {
              const float4 cc = S.cand_c[k];
              const float dzc = wrapd(cc.z - zc, a.LZ);
              const float ddx = xc - cc.x, ddy = yc - cc.y;
              if (ddx * ddx + ddy * ddy + dzc * dzc <= cc.w) {
                const int cxy = S.cand_xy[k];
                if ((cxy & wxy) == cxy && (S.cand_z[k] & wz)) {
                  const float rw = __int_as_float(S.cand_w[k]);
                  const float dcen = dist3(ddx, ddy, -dzc);
                  const float4 nr = S.cand_n[k];
                  if (dcen < 2.f && !(dcen - rec_rb(rw) > 1.f) && e1x * nr.x + e1y * nr.y + e1z * nr.z < 0.f) {
                    const float pd = (cc.x - xc) * nr.x + (cc.y - yc) * nr.y + dzc * nr.z;
                    const float qd = fmaxf(sqrtf(fmaxf(dcen * dcen - pd * pd, 0.f)) - 0.75f * rec_rb(rw), 0.f);
                    const int tri = __float_as_int(nr.w) - g_own;  // not the node's own triangle
                    pass = pd * pd + qd * qd <= 1.004f &&
                           !((unsigned)tri < (unsigned)c.nt &&
                             (c.tri[3 * tri] == node || c.tri[3 * tri + 1] == node || c.tri[3 * tri + 2] == node));
                    e = S.cand_e[k];
                  }
                }
              }
            }
            const unsigned bal = __ballot_sync(FULL, pass);
            if (pass) queue[qn + __popc(bal & ((1u << lane) - 1u))] = e;
            qn += __popc(bal);
            if (qn >= 32) flush(32);
          }
          while (qn > 0) flush(min(qn, 32));
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            rx += __shfl_xor_sync(FULL, rx, o);
            ry += __shfl_xor_sync(FULL, ry, o);
            rz += __shfl_xor_sync(FULL, rz, o);
          }
          if (lane == 0) {
            S.acc[t][0] += rx;
            S.acc[t][1] += ry;
            S.acc[t][2] += rz;
          }
        }
        __syncthreads();  // the list is free for the next records
        ncl = 0;
      };

      // one barrier per round: each warp's count goes to one of two arrays in
      // turn, and every thread sums them itself, so records keep their order.
      // A thread's record of the next round (centroid and normal words, one
      // 32-byte sector) is loaded while the current round is filtered.
      auto fetch = [&](int f, int& e, int& r, float4& cr, float4& nr) {
        e = 0;
        r = 0;
        cr = nr = make_float4(0.f, 0.f, 0.f, 0.f);
        if (f < total) {
#pragma unroll
          for (int stp = 16; stp > 0; stp >>= 1)
            if (r + stp < 27 && f >= S.rng[r + stp]) r += stp;
          e = S.rst[r] + (f - S.rng[r]);
          cr = a.bin_rec[2 * e];
          nr = a.bin_rec[2 * e + 1];
        }
      };
      int f0 = 0, par = 0;
      while (f0 < total) {
        if (ncl + kRgThreads > kRgCand) process();  // outside the rounds: no prefetch is live
        int e_nx, r_nx;
        float4 cr_nx, nr_nx;
        fetch(f0 + tid, e_nx, r_nx, cr_nx, nr_nx);
        for (; f0 < total && ncl + kRgThreads <= kRgCand; f0 += kRgThreads, par ^= 1) {
          const int f = f0 + tid, e = e_nx, r = r_nx;
          const float4 cr = cr_nx, nr = nr_nx;
          fetch(f + kRgThreads, e_nx, r_nx, cr_nx, nr_nx);
          bool keep = false;
          if (f < total) {
            const float rb = rec_rb(cr.w);
            const float dx = fmaxf(fabsf(cr.x - mxc) - hx, 0.f), dy = fmaxf(fabsf(cr.y - myc) - hy, 0.f);
            const float dz = fmaxf(fabsf(wrapd(cr.z - mzc, a.LZ)) - hz, 0.f);
            const float lim = 1.0021f + 0.75f * rb;
            keep = dx * dx + dy * dy + dz * dz <= lim * lim * 1.0001f;
          }
          const unsigned bal = __ballot_sync(FULL, keep);
          if (lane == 0) S.wsum2[par][warp] = __popc(bal);
          __syncthreads();
          int base = ncl, kept = 0;
          for (int w = 0; w < kRgWarps; ++w) {
            const int n = S.wsum2[par][w];
            if (w < warp) base += n;
            kept += n;
          }
          if (keep) {
            const int pos = base + __popc(bal & ((1u << lane) - 1u));
            const float rb = rec_rb(cr.w);
            const float lim = 1.0021f + 0.75f * rb;
            S.cand_c[pos] = make_float4(cr.x, cr.y, cr.z, lim * lim * 1.0001f);
            S.cand_n[pos] = nr;
            S.cand_w[pos] = __float_as_int(cr.w);
            S.cand_e[pos] = e;
            const int kk = rec_kk(cr.w), rel = S.rrel[r];
            const int bi = (rel & 0xff) * 4 + (kk >> 4), bj = ((rel >> 8) & 0xff) * 4 + ((kk >> 2) & 3),
                      bk = (rel >> 16) * 4 + (kk & 3);
            S.cand_xy[pos] = (1 << bi) | (1 << (12 + bj));
            S.cand_z[pos] = 1 << bk;
          }
          ncl += kept;
        }
      }
      if (ncl > 0) process();
      // the chunk's sums into NODE_WALLREPUL (one writer per node)
      if (tid < cnt) {
        const int cell = __float_as_int(S.node_n[tid].w);
        if (cell >= 0) {
          const int node = S.node_id[tid];
          c.wrep[((size_t)0 * nc + cell) * c.nn + node] += S.acc[tid][0];
          c.wrep[((size_t)1 * nc + cell) * c.nn + node] += S.acc[tid][1];
          c.wrep[((size_t)2 * nc + cell) * c.nn + node] += S.acc[tid][2];
        }
      }
    }
    __syncthreads();
  }
}

// Wall nodes that can hold a node's nearest wall triangle, per lattice point
// p of a tile near the wall (ZebraflowWT.c:8998-9077).  A node whose lattice
// index is p lies in the box B = [p - 0.01, p + 0.99] DX per axis (as
// lat_index rounds; 0.51 DX half-width here for rounding).  Its search scans
// the lists of the wall nodes in p's window in scan order and keeps the first
// candidate (triangle vertex or centroid) strictly nearer than the running
// minimum, which starts at 1.5 um.  With U = min over the window's candidates
// c of max over B of |x - c|, the minimum is at most min(U, 1.5), so a list
// whose candidates are all farther from B than that holds neither the winner
// nor a tie with it; a list met again adds nothing.  What remains is the
// distinct wall nodes, in order of first appearance, whose lists come within
// min(U, 1.5) + 1e-3 of B: at most kWallRel of them (more: -1, and the node
// walks its window instead).  One thread per point, one block of 64 per grid
// tile; the count pass writes counts, the fill pass the lists.
constexpr int kWallRel = 192;
template <bool kFill>
__global__ void k_wall_rel(IbArgs a, int32_t* __restrict__ cnt, int32_t* __restrict__ clipped,
                           const int32_t* __restrict__ off, int32_t* __restrict__ out) {
  const int64_t gt = blockIdx.x;
  const int t = a.tile_map[gt];
  if (t < 0) return;
  const int tx = (int)(gt % a.ntx), ty = (int)((gt / a.ntx) % a.nty), tz = (int)(gt / ((int64_t)a.ntx * a.nty));
  const int cl = threadIdx.x;
  const int i = tx * 4 + (cl & 3), j = ty * 4 + ((cl >> 2) & 3), k = tz * 4 + (cl >> 4);
  const int64_t s = (int64_t)t * ZF_TC + cl;
  // windows of this tile reach the 27 tiles around it only
  int near = 0;
  if (cl < 27) {
    int X, Y, Z;
    const int tn = neighbour_tile(a, tx, ty, tz, cl, X, Y, Z);
    near = tn >= 0 && a.tile_wall[tn];
  }
  if (!__syncthreads_or(near)) {
    if (!kFill) cnt[s] = clipped[s] = 0;
    return;
  }
  // the fill pass writes exactly the count pass's entries, and only there
  const int nfill = kFill ? cnt[s] : 0;
  if (kFill && nfill <= 0) return;
  const int i1 = max(i - 4, 0), i2 = min(i + 4, a.nx - 1);
  const int j1 = max(j - 4, 0), j2 = min(j + 4, a.ny - 1);
  const int k1 = max(k - 4, a.kmin), k2 = min(k + 4, a.kmax);
  const float DXf = (float)a.DX;
  const float cx = (float)(a.X0 + (i + 0.49) * a.DX), cy = (float)(a.Y0 + (j + 0.49) * a.DX),
              cz = (float)(a.Z0 + (k + 0.49) * a.DX);
  const float h = 0.51f * DXf;
  auto box_min = [&](float x, float y, float z) {
    const float dx = fmaxf(fabsf(x - cx) - h, 0.f), dy = fmaxf(fabsf(y - cy) - h, 0.f),
                dz = fmaxf(fabsf(wrapd(z - cz, a.LZ)) - h, 0.f);
    return sqrtf(dx * dx + dy * dy + dz * dz);
  };
  auto box_max = [&](float x, float y, float z) {
    const float dx = fabsf(x - cx) + h, dy = fabsf(y - cy) + h, dz = fabsf(wrapd(z - cz, a.LZ)) + h;
    return sqrtf(dx * dx + dy * dy + dz * dz);
  };
  const float cap = 1.51f;
  float U = 3.0e38f;
  int last = 0;
  for (int ii = i1; ii <= i2; ++ii)
    for (int jj = j1; jj <= j2; ++jj)
      for (int kk = k1; kk <= k2; ++kk) {
        const int64_t sw = slot_of(a, ii, jj, wrapk(a, kk));
        if (sw < 0) continue;
        const int m = a.windex[sw];
        if (m <= 0 || m == last) continue;
        last = m;
        const float4 wn = a.wnode[sw];
        if (box_min(wn.x, wn.y, wn.z) - wn.w > cap) continue;  // cannot bring U below 1.5
        for (int e = a.wcand_off[m - 1]; e < a.wcand_off[m]; ++e) {
          const float4 p = a.wcand[e];
          U = fminf(U, box_max(p.x, p.y, p.z));
        }
      }
  const float thr = fminf(U, 1.5f) + 1e-3f;
  int seen[kWallRel];
  int n = 0;
  const int base = kFill ? off[s] : 0;
  last = 0;
  for (int ii = i1; ii <= i2; ++ii)
    for (int jj = j1; jj <= j2; ++jj)
      for (int kk = k1; kk <= k2; ++kk) {
        const int64_t sw = slot_of(a, ii, jj, wrapk(a, kk));
        if (sw < 0) continue;
        const int m = a.windex[sw];
        if (m <= 0 || m == last) continue;
        last = m;
        const float4 wn = a.wnode[sw];
        if (box_min(wn.x, wn.y, wn.z) - wn.w > thr) continue;
        float lbm = 3.0e38f;
        for (int e = a.wcand_off[m - 1]; e < a.wcand_off[m]; ++e) {
          const float4 p = a.wcand[e];
          lbm = fminf(lbm, box_min(p.x, p.y, p.z));
        }
        if (lbm > thr) continue;
        bool dup = false;
        for (int q = 0; q < min(n, kWallRel); ++q) dup |= seen[q] == m;
        if (dup) continue;
        if (n < kWallRel) {
          seen[n] = m;
          if (kFill && n < nfill) out[base + n] = m;
        }
        ++n;
      }
  if (!kFill) {
    cnt[s] = n > kWallRel ? -1 : n;
    clipped[s] = n > kWallRel ? 0 : n;
  }
}

__device__ __forceinline__ void wall_repel(const IbArgs& a, const CellArgs& c, int64_t gid, int cell, int node,
                                           float xp, float yp, float zp, int triwall) {
  // signed distance to the plane of the wall triangle, repulsion, :9055-9077
  if (a.wall_tri) a.wall_tri[gid] = triwall;  // for the adjoint
  const int nc = c.n_cells;
  const int w1 = a.wtri[3 * triwall];
  const float n0 = a.wnrm[triwall], n1 = a.wnrm[a.mt + triwall], n2 = a.wnrm[2 * a.mt + triwall];
  const float ddx = xp - a.wxyz[w1], ddy = yp - a.wxyz[a.nw + w1], ddz = wrapd(zp - a.wxyz[2 * a.nw + w1], a.LZ);
  const float dist = __fadd_rn(__fadd_rn(__fmul_rn(ddx, n0), __fmul_rn(ddy, n1)), __fmul_rn(ddz, n2));
  if (dist < 0.25f && fabsf(dist) < 1.0f && node < c.nn) {
    float repulf = (float)((0.25 - (double)dist) / 1.0);
    if (dist < -0.75f) repulf = 1.f;
    // nucleus nodes add to the membrane array at their own index, as the
    // reference does (ZebraflowWT.c:9415-9430 write NODE_WALLREPUL[v][caps][node])
    atomicAdd(&c.wrep[((size_t)0 * nc + cell) * c.nn + node], (float)((double)repulf * 1.e-04 * n0));
    atomicAdd(&c.wrep[((size_t)1 * nc + cell) * c.nn + node], (float)((double)repulf * 1.e-04 * n1));
    atomicAdd(&c.wrep[((size_t)2 * nc + cell) * c.nn + node], (float)((double)repulf * 1.e-04 * n2));
  }
}

// Nearest wall triangle and wall repulsion (as k_ib_wall), first pass: one
// thread per node.  A node whose lattice point has wall-node lists
// (k_wall_rel) is queued at the back of `walk` for k_wall_lists; no list means
// no triangle.  Nodes whose point has no lists (too many, or outside the IB
// view) are queued at the front for k_wall_walk.  ctr: [0] front count,
// [2] back count.
__global__ void k_wall_nodes(IbArgs a, CellArgs c, int32_t* __restrict__ walk, int32_t* __restrict__ ctr) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ntot = (int64_t)c.n_cells * (c.nn + c.nnn);
  if (gid >= ntot) return;
  bool nuc;
  int cell, node;
  if (!node_of(c, gid, nuc, cell, node)) return;
  const int n = nuc ? c.nnn : c.nn;
  float xp, yp, zp;
  node_pos(nuc ? c.xn : c.x, c.n_cells, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
  const int i0 = lat_index(xp, a.X0, a.DX), j0 = lat_index(yp, a.Y0, a.DX), k0 = lat_index(zp, a.Z0, a.DX);
  if (k0 < a.own_k0 || k0 >= a.own_k1) return;  // another slab's node
  if (max(i0 - 4, 0) > min(i0 + 4, a.nx - 1) || max(j0 - 4, 0) > min(j0 + 4, a.ny - 1) ||
      max(k0 - 4, a.kmin) > min(k0 + 4, a.kmax))
    return;  // empty window
  int rel = -1;
  int64_t s0 = -1;
  if (a.wrel_cnt && i0 >= 0 && i0 < a.nx && j0 >= 0 && j0 < a.ny) {
    const int kw0 = wrapk(a, k0);
    if (kw0 >= 0 && kw0 < a.nz) {
      s0 = slot_of(a, i0, j0, kw0);
      if (s0 >= 0) rel = a.wrel_cnt[s0];
    }
  }
  if (rel < 0) walk[atomicAdd(&ctr[0], 1)] = (int32_t)gid;
  else if (rel > 0) walk[ntot - 1 - atomicAdd(&ctr[2], 1)] = (int32_t)gid;
}

// The queued nodes with wall-node lists, a warp per node: each lane scans
// whole lists (lane l takes list l of every 32), keeping its first strict
// minimum below 1.5 um and that candidate's position in the node's scan; the
// warp then takes the smallest distance, ties to the earliest position -- the
// first candidate in scan order that reaches the minimum, which is what the
// reference's running minimum (strict <) ends on.
__global__ void __launch_bounds__(kTileThreads) k_wall_lists(IbArgs a, CellArgs c, const int32_t* __restrict__ walk,
                                                            const int32_t* __restrict__ ctr, int32_t* __restrict__ work) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t ntot = (int64_t)c.n_cells * (c.nn + c.nnn);
  const int nq = ctr[2];
  for (int li = warp_next_tile(work, lane); li < nq; li = warp_next_tile(work, lane)) {
    const int64_t gid = walk[ntot - 1 - li];
    bool nuc;
    int cell, node;
    node_of(c, gid, nuc, cell, node);
    const int n = nuc ? c.nnn : c.nn;
    float xp, yp, zp;
    node_pos(nuc ? c.xn : c.x, c.n_cells, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
    const int i0 = lat_index(xp, a.X0, a.DX), j0 = lat_index(yp, a.Y0, a.DX), k0 = lat_index(zp, a.Z0, a.DX);
    const int64_t s0 = slot_of(a, i0, j0, wrapk(a, k0));
    const int rel = a.wrel_cnt[s0];
    const int32_t* lists = a.wrel + a.wrel_off[s0];
    // lane l scans list r0 + l of each chunk of 32 lists, in order; a
    // candidate's position in the node's scan is the lists' running count
    // before its list (a warp scan) plus its place in the list
    float best = 1.5f;
    int bpos = INT_MAX, tbest = -1, pos0 = 0;
    for (int r0 = 0; r0 < rel; r0 += 32) {
      int32_t c0 = 0, len = 0;
      if (r0 + lane < rel) {
        const int m = lists[r0 + lane];
        c0 = a.wcand_off[m - 1];
        len = a.wcand_off[m] - c0;
      }
      int incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      const int before = pos0 + incl - len;
#pragma unroll 4
      for (int i = 0; i < len; ++i) {
        const float4 p = a.wcand[c0 + i];
        const float d = dist3(xp - p.x, yp - p.y, wrapd(zp - p.z, a.LZ));
        if (d < best) {
          best = d;
          bpos = before + i;
          tbest = __float_as_int(p.w);
        }
      }
      pos0 += __shfl_sync(FULL, incl, 31);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(FULL, best, o);
      const int op = __shfl_xor_sync(FULL, bpos, o), ot = __shfl_xor_sync(FULL, tbest, o);
      if (ob < best || (ob == best && op < bpos)) {
        best = ob;
        bpos = op;
        tbest = ot;
      }
    }
    if (lane == 0 && tbest >= 0) wall_repel(a, c, gid, cell, node, xp, yp, zp, tbest);
  }
}

// Second pass for the queued nodes: a warp per node walks its window 32
// points at a time in the reference scan order (i, j, k).  A first pass finds
// the window's nearest wall node; the first minimum of its list bounds the
// window minimum from above.  The second pass skips a point that repeats the
// previous point's wall node or whose wall node cannot reach the bound, and
// queues the other lists in scan order; they are scanned 32 at a time, one
// per lane, and folded in queue order: the lowest lane holding the batch
// minimum is the first candidate in scan order, and it replaces the running
// minimum only when strictly smaller.
__global__ void __launch_bounds__(kTileThreads) k_wall_walk(IbArgs a, CellArgs c, const int32_t* __restrict__ walk,
                                                           const int32_t* __restrict__ walk_n,
                                                           int32_t* __restrict__ ctr) {
  __shared__ int s_q[kTileWarps][64];
  const unsigned FULL = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nc = c.n_cells;
  const int nwalk = *walk_n;
  int* queue = s_q[warp];
  for (int li = warp_next_tile(ctr, lane); li < nwalk; li = warp_next_tile(ctr, lane)) {
    const int64_t gid = walk[li];
    bool nuc;
    int cell, node;
    if (!node_of(c, gid, nuc, cell, node)) continue;
    const int n = nuc ? c.nnn : c.nn;
    float xp, yp, zp;
    node_pos(nuc ? c.xn : c.x, nc, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
    const int gt = node_grid_tile(a, xp, yp, zp);
    const int tx = gt % a.ntx, ty = (gt / a.ntx) % a.nty, tz = gt / (a.ntx * a.nty);
    // lane r < 27: tile id of neighbour r when it holds W_index points
    int rt = -1;
    if (lane < 27) {
      int X, Y, Z;
      const int t = neighbour_tile(a, tx, ty, tz, lane, X, Y, Z);
      if (t >= 0 && a.tile_wall[t]) rt = t;
    }
    if (!__any_sync(FULL, rt >= 0)) continue;
    const int i0 = lat_index(xp, a.X0, a.DX), j0 = lat_index(yp, a.Y0, a.DX), k0 = lat_index(zp, a.Z0, a.DX);
    const int i1 = max(i0 - 4, 0), i2 = min(i0 + 4, a.nx - 1);
    const int j1 = max(j0 - 4, 0), j2 = min(j0 + 4, a.ny - 1);
    const int k1 = max(k0 - 4, a.kmin), k2 = min(k0 + 4, a.kmax);
    if (i1 > i2 || j1 > j2 || k1 > k2) continue;
    float mindis = 1.5f;
    int triwall = -1;
    const int ni = i2 - i1 + 1, nj = j2 - j1 + 1, nk = k2 - k1 + 1;
    const int k1w = wrapk(a, k1);
    const int npts = ni * nj * nk;
    // lane l starts at window point l and steps 32 points in mixed radix;
    // (i, j, dk) with the wrapped z index kw = k1w + dk (minus nz past the end)
    const int sk = 32 % nk, sj = (32 / nk) % nj, si = 32 / (nk * nj);
    const int pi0 = i1 + lane / (nj * nk), pj0 = j1 + (lane / nk) % nj, pk0 = lane % nk;
    auto step = [&](int& i, int& j, int& dk) {
      dk += sk;
      int cy = 0;
      if (dk >= nk) {
        dk -= nk;
        cy = 1;
      }
      j += sj + cy;
      cy = 0;
      if (j > j2) {
        j -= nj;
        cy = 1;
      }
      i += si + cy;
    };
    // slot of window point (i, j, dk) in the IB view, -1 outside the wall tiles
    auto slot = [&](int i, int j, int dk) -> int64_t {
      int kw = k1w + dk;
      if (kw >= a.nz) kw -= a.nz;
      int lz = (kw >> 2) - tz + 1;
      if (lz < 0) lz += a.ntz;
      else if (lz > 2) lz -= a.ntz;
      const int r = (lz * 3 + ((j >> 2) - ty + 1)) * 3 + ((i >> 2) - tx + 1);
      const int t = __shfl_sync(FULL, rt, r);  // every lane calls slot()
      return t < 0 ? (int64_t)-1 : (int64_t)t * ZF_TC + (i & 3) + 4 * (j & 3) + 16 * (kw & 3);
    };
    // bound: the first minimum of one list of the window bounds the window
    // minimum from above (1.5 is the reference's starting value); take the
    // nearest wall node among those of the 8 lattice points around the node
    float bound = 1.5f;
    {
      float dbest = 3.0e38f;
      int mbest = 0;
      const int ci = (int)floor(((double)xp - a.X0) / a.DX) + (lane & 1);
      const int cj = (int)floor(((double)yp - a.Y0) / a.DX) + ((lane >> 1) & 1);
      const int ck = (int)floor(((double)zp - a.Z0) / a.DX) + ((lane >> 2) & 1);
      const bool in = lane < 8 && ci >= i1 && ci <= i2 && cj >= j1 && cj <= j2 && ck >= k1 && ck <= k2;
      // every lane calls slot(); lanes outside pass a window point
      const int64_t sc = slot(in ? ci : i1, in ? cj : j1, in ? ck - k1 : 0);
      if (in && sc >= 0) {
        const int wi = a.windex[sc];
        const float4 wn = a.wnode[sc];
        if (wi > 0) {
          dbest = dist3(xp - wn.x, yp - wn.y, wrapd(zp - wn.z, a.LZ));
          mbest = wi;
        }
      }
      float dmin = dbest;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dmin = fminf(dmin, __shfl_xor_sync(FULL, dmin, o));
      const unsigned at = __ballot_sync(FULL, dbest == dmin && mbest > 0);
      if (at) {
        const int m = __shfl_sync(FULL, mbest, __ffs(at) - 1);
        int unused = -1;
        wall_list_min(a, m, xp, yp, zp, bound, unused);
      }
    }
    int last = 0, qn = 0;
    auto flush = [&](int nb) {
      __syncwarp();
      float d = 3.0e38f;
      int t = -1;
      if (lane < nb) wall_list_min(a, queue[lane], xp, yp, zp, d, t);
      float dmin = d;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dmin = fminf(dmin, __shfl_xor_sync(FULL, dmin, o));
      const unsigned at = __ballot_sync(FULL, d == dmin && t >= 0);
      if (at && dmin < mindis) {
        mindis = dmin;
        triwall = __shfl_sync(FULL, t, __ffs(at) - 1);
      }
      const int rem = qn - nb;
      const int tq = lane < rem ? queue[nb + lane] : 0;
      __syncwarp();
      if (lane < rem) queue[lane] = tq;
      __syncwarp();
      qn = rem;
    };
    {
      int i = pi0, j = pj0, dk = pk0;
      for (int p0 = 0; p0 < npts; p0 += 32) {
        int wi = 0;
        float4 wn = make_float4(0.f, 0.f, 0.f, -1.f);
        const int64_t s = slot(i, j, dk);
        if (p0 + lane < npts && s >= 0) {
          wi = a.windex[s];
          wn = a.wnode[s];
        }
        step(i, j, dk);
        int prev = __shfl_up_sync(FULL, wi, 1);
        if (lane == 0) prev = last;
        last = __shfl_sync(FULL, wi, 31);
        bool want = false;
        if (wi > 0 && wi != prev) {
          const float dm = dist3(xp - wn.x, yp - wn.y, wrapd(zp - wn.z, a.LZ));
          want = !(dm - wn.w > fminf(bound, mindis) + 1e-4f);
        }
        const unsigned bal = __ballot_sync(FULL, want);
        if (want) queue[qn + __popc(bal & ((1u << lane) - 1u))] = wi;
        qn += __popc(bal);
        while (qn >= 32) flush(32);
      }
      while (qn > 0) flush(min(qn, 32));
    }
    if (triwall >= 0 && lane == 0) wall_repel(a, c, gid, cell, node, xp, yp, zp, triwall);
  }
}

// ---- spreading ----------------------------------------------------------------

__global__ void k_ib_spread(IbArgs a, CellArgs c, int spread_walls) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  const int64_t nmem = (int64_t)nc * c.nn;
  const bool nuc = gid >= nmem;
  if (gid >= nmem + (int64_t)nc * c.nnn) return;
  const int n = nuc ? c.nnn : c.nn;
  const int64_t lid = nuc ? gid - nmem : gid;
  const int cell = (int)(lid / n), node = (int)(lid % n);
  if (c.status[cell] <= 0) return;
  const double* X = nuc ? c.xn : c.x;
  double* V = nuc ? c.vel_n : c.vel;
  const float* R = nuc ? c.wrep_n : c.wrep;
  const float* FT = nuc ? c.ftot_n : c.ftot;
  float Ff[3];
  for (int v = 0; v < 3; ++v) {  // :10749-10754
    const size_t g = ((size_t)v * nc + cell) * n + node;
    V[g] += (double)R[g];
    Ff[v] = (float)((double)a.gamma_p * (double)R[g] + (double)FT[g]);
  }
  float xp, yp, zp;
  node_pos(X, nc, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
  const float h2 = 2.f * a.DX;
  StencilAxis SX, SY, SZ;
  node_stencil(a, xp, yp, zp, SX, SY, SZ);
  stencil_walk(SX, SY, SZ, h2, [&](int i, int j, int k, double w) {
    if (k < a.own_k0 || k >= a.own_k1) return;  // another slab's plane
    const int64_t s = slot_of(a, i, j, wrapk(a, k));
    if (s < 0 || s >= a.ns) return;
    const uint8_t cd = a.code[s];
    if (!(zf_code_fluid(cd) || (spread_walls && (cd == ZF_CODE_WALL || zf_code_pressure(cd))))) return;
    for (int v = 0; v < 3; ++v) atomicAdd(&a.force[v * a.ns + s], (float)(w * (double)Ff[v] * a.force_scale));
  });
}

// k_ib_spread per lattice tile of nodes (node-tile lists): a block takes a
// tile, adds its nodes' stencil contributions into shared memory over the
// 12x12x12 points of the tile's 3x3x3 neighbourhood (a node's stencil stays
// inside it), then adds each touched point to BODYFORCE once.  Neighbouring
// nodes share most stencil points, so the global float atomics drop several
// times.  The nodes' own updates (NODE_VEL += NODE_WALLREPUL, :10749-10754)
// happen once per node in the first pass.  A contribution outside the
// neighbourhood (not expected) goes straight to BODYFORCE.
constexpr int kSpreadNodes = 128;  // nodes staged per pass
// five blocks per SM (48 registers): the block waits on its shared-memory
// atomics and barriers, and more resident blocks hide that
__global__ void __launch_bounds__(256, 5) k_spread_tiles(IbArgs a, CellArgs c, int spread_walls) {
  __shared__ float acc[3][1728];
  __shared__ float s_f[3][kSpreadNodes];
  __shared__ StencilAxis s_ax[3][kSpreadNodes];  // per staged node: its stencil along x, y, z
  __shared__ int s_li;
  const int nc = c.n_cells;
  const int nlist = a.tile_ctr[0];
  const float h2 = 2.f * a.DX;
  for (;;) {
    if (threadIdx.x == 0) s_li = atomicAdd(&a.tile_ctr[3], 1);
    __syncthreads();
    const int li = s_li;
    if (li >= nlist) break;
    float* accf = &acc[0][0];
    for (int e = threadIdx.x; e < 3 * 1728; e += blockDim.x) accf[e] = 0.f;
    const int gt = a.tile_list[li];
    const int tx = gt % a.ntx, ty = (gt / a.ntx) % a.nty, tz = gt / (a.ntx * a.nty);
    const int ox = (tx - 1) * 4, oy = (ty - 1) * 4, oz = (tz - 1) * 4;
    const int n0 = a.node_off[gt], n1 = a.node_off[gt + 1];
    for (int c0 = n0; c0 < n1; c0 += kSpreadNodes) {
      const int cnt = min(kSpreadNodes, n1 - c0);
      __syncthreads();  // the previous chunk's items are done with the staged nodes
      if ((int)threadIdx.x < cnt) {
        const int t = threadIdx.x;
        bool nuc;
        int cell, node;
        s_ax[0][t].ok = 0u;  // inactive node: no stencil point
        if (node_of(c, a.node_sorted[c0 + t], nuc, cell, node)) {
          const int n = nuc ? c.nnn : c.nn;
          double* V = nuc ? c.vel_n : c.vel;
          const float* R = nuc ? c.wrep_n : c.wrep;
          const float* FT = nuc ? c.ftot_n : c.ftot;
          for (int v = 0; v < 3; ++v) {  // :10749-10754
            const size_t g = ((size_t)v * nc + cell) * n + node;
            V[g] += (double)R[g];
            s_f[v][t] = (float)((double)a.gamma_p * (double)R[g] + (double)FT[g]);
          }
          float xp, yp, zp;
          node_pos(nuc ? c.xn : c.x, nc, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
          StencilAxis X, Y, Z;
          node_stencil(a, xp, yp, zp, X, Y, Z);
          s_ax[0][t] = X;
          s_ax[1][t] = Y;
          s_ax[2][t] = Z;
        }
      }
      __syncthreads();
      // one item per (node, x, y) column of its stencil, walking z
      for (int it = threadIdx.x; it < cnt * 16; it += blockDim.x) {
        const int t = it >> 4, mi = (it >> 2) & 3, mj = it & 3;
        const StencilAxis& X = s_ax[0][t];
        const StencilAxis& Y = s_ax[1][t];
        const StencilAxis& Z = s_ax[2][t];
        if (!((X.ok >> mi) & (Y.ok >> mj) & 1u)) continue;
        const int i = X.b + mi, j = Y.b + mj;
        const float sxy = __fadd_rn(X.s[mi], Y.s[mj]);
        const double fxy = (1.0 + (double)X.c[mi]) * (1.0 + (double)Y.c[mj]);
        const float f0 = s_f[0][t], f1 = s_f[1][t], f2 = s_f[2][t];
        for (int mk = 0; mk < 4; ++mk) {
          if (!((Z.ok >> mk) & 1u)) continue;
          if (!(sqrtf(__fadd_rn(sxy, Z.s[mk])) <= h2)) continue;
          const double w = fxy * (1.0 + (double)Z.c[mk]) / 64.0;
          if (!(w > 0.0)) continue;
          const int k = Z.b + mk;
          if (k < a.own_k0 || k >= a.own_k1) continue;  // another slab's plane
          const int64_t sl = slot_of(a, i, j, wrapk(a, k));
          if (sl < 0 || sl >= a.ns) continue;
          const uint8_t cd = a.code[sl];
          if (!(zf_code_fluid(cd) || (spread_walls && (cd == ZF_CODE_WALL || zf_code_pressure(cd))))) continue;
          const int di = i - ox, dj = j - oy;
          int dk = k - oz;
          if (a.per_z) dk = ((dk % a.nz) + a.nz) % a.nz;
          const bool in = di >= 0 && di < 12 && dj >= 0 && dj < 12 && dk >= 0 && dk < 12;
          const float v0 = (float)(w * (double)f0 * a.force_scale), v1 = (float)(w * (double)f1 * a.force_scale),
                      v2 = (float)(w * (double)f2 * a.force_scale);
          if (in) {
            const int r = (dk * 12 + dj) * 12 + di;
            atomicAdd(&acc[0][r], v0);
            atomicAdd(&acc[1][r], v1);
            atomicAdd(&acc[2][r], v2);
          } else {
            atomicAdd(&a.force[sl], v0);
            atomicAdd(&a.force[a.ns + sl], v1);
            atomicAdd(&a.force[2 * a.ns + sl], v2);
          }
        }
      }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < 1728; r += blockDim.x) {
      const float fx = acc[0][r], fy = acc[1][r], fz = acc[2][r];
      if (fx == 0.f && fy == 0.f && fz == 0.f) continue;
      const int i = ox + r % 12, j = oy + (r / 12) % 12;
      int k = oz + r / 144;
      if (a.per_z) k = ((k % a.nz) + a.nz) % a.nz;
      if (i < 0 || i >= a.nx || j < 0 || j >= a.ny || k < 0 || k >= a.nz) continue;
      const int64_t sl = slot_of(a, i, j, k);
      if (sl < 0 || sl >= a.ns) continue;
      atomicAdd(&a.force[sl], fx);
      atomicAdd(&a.force[a.ns + sl], fy);
      atomicAdd(&a.force[2 * a.ns + sl], fz);
    }
    __syncthreads();
  }
}

// ---- position update ------------------------------------------------------------

__global__ void k_update(IbArgs a, CellArgs c) {
  const int cell = blockIdx.x;
  if (c.status[cell] <= 0) return;
  const int nc = c.n_cells;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < c.nnn; i += blockDim.x)  // nucleus first, :11969-11973
    for (int v = 0; v < 3; ++v) {
      const size_t g = ((size_t)v * nc + cell) * c.nnn + i;
      c.xn[g] += c.vel_n[g] * a.dt_stagger;
    }
  for (int i = threadIdx.x; i < c.nn; i += blockDim.x) {  // speed check, :11975-11981
    const double vx = c.vel[((size_t)0 * nc + cell) * c.nn + i];
    const double vy = c.vel[((size_t)1 * nc + cell) * c.nn + i];
    const double vz = c.vel[((size_t)2 * nc + cell) * c.nn + i];
    const float sp = sqrtf((float)(vx * vx + vy * vy + vz * vz));
    if (sp > a.vmax_remove || isnan(sp) || isinf(sp)) bad = 1;
  }
  __syncthreads();
  if (!bad) {
    for (int i = threadIdx.x; i < c.nn; i += blockDim.x)
      for (int v = 0; v < 3; ++v) {
        const size_t g = ((size_t)v * nc + cell) * c.nn + i;
        c.x[g] += c.vel[g] * a.dt_stagger;
      }
    return;
  }
  // removal: every node to the null position, :12007-12030
  for (int i = threadIdx.x; i < c.nn; i += blockDim.x)
    for (int v = 0; v < 3; ++v) {
      const size_t g = ((size_t)v * nc + cell) * c.nn + i;
      c.x[g] = -5000.0;
      c.vel[g] = 0.0;
      c.ftot[g] = 0.f;
      c.wrep[g] = 0.f;
    }
  for (int i = threadIdx.x; i < c.nnn; i += blockDim.x)
    for (int v = 0; v < 3; ++v) {
      const size_t g = ((size_t)v * nc + cell) * c.nnn + i;
      c.xn[g] = -5000.0;
      c.vel_n[g] = 0.0;
      c.ftot_n[g] = 0.f;
    }
  if (threadIdx.x == 0) {
    c.status[cell] = -5000;
    atomicAdd(&c.counters[1], 1ull);
  }
}

// ---- launchers --------------------------------------------------------------------

// ---- wall shear stress ----------------------------------------------------------

// One thread per wall-mesh node: the reference's post-processor
// (PostProWSSandPressure.c:275-369).  Lattice coordinates X0 + i DX and the
// 1-based index (int)((x - X0)/DX + 1.01) are kept; windows are +-3 with the
// reference's one-sided clamps (i from 3, j and k from 1, 1-based).  Moments
// (a.mom) must hold the current populations' D, U, V, W.
__device__ __forceinline__ void wss_window(int ii, int n, int lo, bool wrap, int& i1, int& i2) {
  // ii, lo 0-based; n points along the axis
  i1 = ii - 3;
  i2 = ii + 3;
  if (wrap) return;
  if (i2 > n - 1) i2 = n - 1;
  else if (i1 < lo) i1 = lo;
}

// probe one DX along the node normal and the Peskin stencil around it, in the
// reference's order (:320-356); fn(slot, weight) for every fluid point in 2 DX
template <class Fn>
__device__ __forceinline__ void wss_stencil(const IbArgs& a, float xm, float ym, float zm, float n0, float n1,
                                            float n2, Fn&& fn) {
  const float xp = (float)((double)xm + a.DX * (double)n0);
  const float yp = (float)((double)ym + a.DX * (double)n1);
  const float zp = (float)((double)zm + a.DX * (double)n2);
  auto lat1 = [&](float x, double x0) { return (int)(((double)x - x0) / a.DX + 1.01) - 1; };
  int i1, i2, j1, j2, k1, k2;
  wss_window(lat1(xp, a.X0), a.nx, 2, false, i1, i2);
  wss_window(lat1(yp, a.Y0), a.ny, 0, false, j1, j2);
  wss_window(lat1(zp, a.Z0), a.nz, 0, a.per_z, k1, k2);
  for (int i = i1; i <= i2; ++i)
    for (int j = j1; j <= j2; ++j)
      for (int k = k1; k <= k2; ++k) {
        const float dx = xp - (float)(a.X0 + i * a.DX), dy = yp - (float)(a.Y0 + j * a.DX);
        const float dz = wrapd(zp - (float)(a.Z0 + k * a.DX), a.LZ);
        const float d = dist3(dx, dy, dz);
        if (!((double)d <= 2 * a.DX)) continue;
        if (i < 0 || i >= a.nx || j < 0 || j >= a.ny) continue;
        int kk = k;
        if (kk < 0 || kk >= a.nz) {
          if (!a.per_z) continue;
          kk = ((kk % a.nz) + a.nz) % a.nz;
        }
        const int64_t s = slot_of(a, i, j, kk);
        if (s < 0 || s >= a.ns) continue;
        const uint8_t cd = a.code[s];
        if (!(zf_code_fluid(cd) || zf_code_pressure(cd))) continue;  // 0.11 < B_index < 4997
        const float w =
            (float)((1. + cosf((float)(kPId * fabsf(dx) / 2 / a.DX))) *
                    (1. + cosf((float)(kPId * fabsf(dy) / 2 / a.DX))) *
                    (1. + cosf((float)(kPId * fabsf(dz) / 2 / a.DX))) / 64.);
        fn(s, w);
      }
}

// WSS = -0.0012 Pa.s (u - (u.n) n) / (DX 1e-6 m)   (:358-368)
__device__ __forceinline__ void wss_of(const IbArgs& a, float UU, float VV, float WW, float n0, float n1,
                                       float n2, float& W0, float& W1, float& W2) {
  const float vn = UU * n0 + VV * n1 + WW * n2;
  const float vt0 = UU - vn * n0, vt1 = VV - vn * n1, vt2 = WW - vn * n2;
  W0 = (float)(-0.0012 * (double)vt0 / a.DX / 1.e-06);
  W1 = (float)(-0.0012 * (double)vt1 / a.DX / 1.e-06);
  W2 = (float)(-0.0012 * (double)vt2 / a.DX / 1.e-06);
}

__global__ void k_wss(IbArgs a, const float* __restrict__ nrm, float pgauge, float* __restrict__ wss,
                      float* __restrict__ press, int32_t* __restrict__ valid) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nw) return;
  const float xm = a.wxyz[m], ym = a.wxyz[a.nw + m], zm = a.wxyz[2 * a.nw + m];
  const float n0 = nrm[m], n1 = nrm[a.nw + m], n2 = nrm[2 * a.nw + m];
  const bool wz = a.per_z;
  auto lat1 = [&](float x, double x0) { return (int)(((double)x - x0) / a.DX + 1.01) - 1; };
  auto point_slot = [&](int i, int j, int k) -> int64_t {  // k may lie outside when wrapping
    if (i < 0 || i >= a.nx || j < 0 || j >= a.ny) return -1;
    if (k < 0 || k >= a.nz) {
      if (!wz) return -1;
      k = ((k % a.nz) + a.nz) % a.nz;
    }
    return slot_of(a, i, j, k);
  };
  // wall pressure at the nearest listed point within 1.42 DX (:276-318)
  {
    int i1, i2, j1, j2, k1, k2;
    wss_window(lat1(xm, a.X0), a.nx, 2, false, i1, i2);
    wss_window(lat1(ym, a.Y0), a.ny, 0, false, j1, j2);
    wss_window(lat1(zm, a.Z0), a.nz, 0, wz, k1, k2);
    float mindis = (float)(1.42 * a.DX);
    int64_t best = -1;
    for (int i = i1; i <= i2; ++i)
      for (int j = j1; j <= j2; ++j)
        for (int k = k1; k <= k2; ++k) {
          const int64_t s = point_slot(i, j, k);
          if (s < 0 || s >= a.ns || a.code[s] == ZF_CODE_SOLID) continue;  // B_index >= 0
          const float dx = xm - (float)(a.X0 + i * a.DX), dy = ym - (float)(a.Y0 + j * a.DX);
          const float dz = wrapd(zm - (float)(a.Z0 + k * a.DX), a.LZ);
          const float d = dist3(dx, dy, dz);
          if (d < mindis) {
            mindis = d;
            best = s;
          }
        }
    int ok = !((double)mindis > 1.419999 * a.DX) && best >= 0;
    float pw = 0.f;
    if (ok) {
      const float pp = (float)(((double)a.mom[best] - 1.) / 3. * 10000.);
      pw = pp - pgauge;
    }
    if (pw < 1.f) ok = 0;
    if (press) press[m] = pw;
    if (valid) valid[m] = ok;
  }
  // wall shear stress from the velocity one DX into the lumen (:320-369)
  float UU = 0.f, VV = 0.f, WW = 0.f;
  wss_stencil(a, xm, ym, zm, n0, n1, n2, [&](int64_t s, float w) {
    UU += w * a.mom[a.ns + s];
    VV += w * a.mom[2 * a.ns + s];
    WW += w * a.mom[3 * a.ns + s];
  });
  float W0, W1, W2;
  wss_of(a, UU, VV, WW, n0, n1, n2, W0, W1, W2);
  wss[m] = W0;
  wss[a.nw + m] = W1;
  wss[2 * a.nw + m] = W2;
}

// ---- adjoint pieces of a WSS objective -------------------------------------------
//
// J = c sum_{m in patch} |WSS_m| for one state (c = 1 / (window length x patch
// size)).  The patch's stencils (slot, Peskin weight, in the order of
// wss_stencil) depend on the geometry only, so they are listed once per call:
// entry e of node i (off[i] <= e < off[i+1]) has weight w[e] and reads the
// velocity of compact point idx[e]; the compact points are the distinct slots
// of all stencils, whose velocities each step computes from the populations
// (k_moments_at).  Per step the objective is then a short sparse sum per node,
// and its adjoint the transposed sum:
//   WSS = k (v - (v.n) n), k = -0.0012 / (DX 1e-6)  =>  dJ/dv = c k P_n WSS/|WSS|.
__global__ void k_wss_stencil_count(IbArgs a, const float* __restrict__ nrm, const int32_t* __restrict__ patch,
                                    int np, int32_t* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int m = patch[i];
  int n = 0;
  wss_stencil(a, a.wxyz[m], a.wxyz[a.nw + m], a.wxyz[2 * a.nw + m], nrm[m], nrm[a.nw + m], nrm[2 * a.nw + m],
              [&](int64_t, float) { ++n; });
  cnt[i] = n;
}

__global__ void k_wss_stencil_fill(IbArgs a, const float* __restrict__ nrm, const int32_t* __restrict__ patch,
                                   int np, const int32_t* __restrict__ off, int32_t* __restrict__ slot,
                                   float* __restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int m = patch[i];
  int e = off[i];
  wss_stencil(a, a.wxyz[m], a.wxyz[a.nw + m], a.wxyz[2 * a.nw + m], nrm[m], nrm[a.nw + m], nrm[2 * a.nw + m],
              [&](int64_t s, float wt) {
                slot[e] = (int32_t)s;
                w[e] = wt;
                ++e;
              });
}

// the probe velocity of patch node i from the compact velocities U[3][nu]
__device__ __forceinline__ void patch_probe(const PatchStencil& ps, const float* __restrict__ U, int i,
                                            float& UU, float& VV, float& WW) {
  UU = VV = WW = 0.f;
  for (int e = ps.off[i]; e < ps.off[i + 1]; ++e) {
    const int u = ps.idx[e];
    const float w = ps.w[e];
    UU += w * U[u];
    VV += w * U[ps.nu + u];
    WW += w * U[2 * ps.nu + u];
  }
}

__global__ void k_wss_patch(IbArgs a, PatchStencil ps, const float* __restrict__ nrm,
                            const float* __restrict__ U, double c, double* acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < ps.np) {
    const int m = ps.patch[i];
    const float n0 = nrm[m], n1 = nrm[a.nw + m], n2 = nrm[2 * a.nw + m];
    float UU, VV, WW;
    patch_probe(ps, U, i, UU, VV, WW);
    float W0, W1, W2;
    wss_of(a, UU, VV, WW, n0, n1, n2, W0, W1, W2);
    v = c * sqrt((double)W0 * W0 + (double)W1 * W1 + (double)W2 * W2);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(acc, v);
}

// gU[3][nu] += dJ/dU at the compact points
__global__ void k_wss_patch_adj(IbArgs a, PatchStencil ps, const float* __restrict__ nrm,
                                const float* __restrict__ U, double c, float* __restrict__ gU) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ps.np) return;
  const int m = ps.patch[i];
  const float n0 = nrm[m], n1 = nrm[a.nw + m], n2 = nrm[2 * a.nw + m];
  float UU, VV, WW;
  patch_probe(ps, U, i, UU, VV, WW);
  float W0, W1, W2;
  wss_of(a, UU, VV, WW, n0, n1, n2, W0, W1, W2);
  const double mag = sqrt((double)W0 * W0 + (double)W1 * W1 + (double)W2 * W2);
  if (!(mag > 0.0)) return;
  const double k = -0.0012 / a.DX / 1.e-06;
  const double h0 = W0 / mag, h1 = W1 / mag, h2 = W2 / mag;
  const double hn = h0 * n0 + h1 * n1 + h2 * n2;
  const float g0 = (float)(c * k * (h0 - hn * n0)), g1 = (float)(c * k * (h1 - hn * n1)),
              g2 = (float)(c * k * (h2 - hn * n2));
  for (int e = ps.off[i]; e < ps.off[i + 1]; ++e) {
    const int u = ps.idx[e];
    const float w = ps.w[e];
    atomicAdd(&gU[u], w * g0);
    atomicAdd(&gU[ps.nu + u], w * g1);
    atomicAdd(&gU[2 * ps.nu + u], w * g2);
  }
}

// ---- flux-split objective ---------------------------------------------------------
//
// For two sets of listed points (outlet cross-sections) with unit normals n_0,
// n_1: Q_s = sum over set s of U.n_s, U the moments (no force shift) of the
// populations, and J = c Q_0 / (Q_0 + Q_1) for one state; the compact points
// of `ps` are the points of both sets, set[u] telling which.  This objective
// has no counterpart in the reference.
struct Nrm6 {
  float v[6];
};

__global__ void k_flux_q(PatchStencil ps, const uint8_t* __restrict__ set, Nrm6 n, const float* __restrict__ U,
                         double* q) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  double q0 = 0.0, q1 = 0.0;
  if (u < ps.nu) {
    const int st = set[u];
    const float* nn = n.v + 3 * st;
    const double f = (double)U[u] * nn[0] + (double)U[ps.nu + u] * nn[1] + (double)U[2 * ps.nu + u] * nn[2];
    if (st) q1 = f;
    else q0 = f;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    q0 += __shfl_down_sync(0xffffffffu, q0, o);
    q1 += __shfl_down_sync(0xffffffffu, q1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (q0 != 0.0) atomicAdd(&q[0], q0);
    if (q1 != 0.0) atomicAdd(&q[1], q1);
  }
}

__global__ void k_flux_j(const double* __restrict__ q, double c, double* acc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const double den = q[0] + q[1];
    if (den != 0.0) *acc += c * q[0] / den;
  }
}

// gU[3][nu] += c dJ/dU:  dJ/dQ_0 = Q_1/(Q_0+Q_1)^2, dJ/dQ_1 = -Q_0/(Q_0+Q_1)^2
__global__ void k_flux_gu(PatchStencil ps, const uint8_t* __restrict__ set, Nrm6 n, const double* __restrict__ q,
                          double c, float* __restrict__ gU) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ps.nu) return;
  const double den = q[0] + q[1];
  if (den == 0.0) return;
  const int st = set[u];
  const double g = c * (st ? -q[0] : q[1]) / (den * den);
  const float* nn = n.v + 3 * st;
  gU[u] += (float)(g * nn[0]);
  gU[ps.nu + u] += (float)(g * nn[1]);
  gU[2 * ps.nu + u] += (float)(g * nn[2]);
}

// transpose of the spreading (k_ib_spread without the repulsion term): for
// every node, g_v = force_scale sum_s w(s) G_v(s) over the spreading stencil
__global__ void k_spread_adj(IbArgs a, CellArgs c, int spread_walls, const float* __restrict__ G,
                             float* __restrict__ g_mem, float* __restrict__ g_nuc) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  const int64_t nmem = (int64_t)nc * c.nn;
  const bool nuc = gid >= nmem;
  if (gid >= nmem + (int64_t)nc * c.nnn) return;
  const int n = nuc ? c.nnn : c.nn;
  const int64_t lid = nuc ? gid - nmem : gid;
  const int cell = (int)(lid / n), node = (int)(lid % n);
  float* out = nuc ? g_nuc : g_mem;
  double acc[3] = {0.0, 0.0, 0.0};
  if (c.status[cell] > 0) {
    float xp, yp, zp;
    node_pos(nuc ? c.xn : c.x, nc, n, cell, node, a.LZ, a.Z0, xp, yp, zp);
    const float h2 = 2.f * a.DX;
    StencilAxis SX, SY, SZ;
    node_stencil(a, xp, yp, zp, SX, SY, SZ);
    stencil_walk(SX, SY, SZ, h2, [&](int i, int j, int k, double w) {
      const int64_t s = slot_of(a, i, j, wrapk(a, k));
      if (s < 0 || s >= a.ns) return;
      const uint8_t cd = a.code[s];
      if (!(zf_code_fluid(cd) || (spread_walls && (cd == ZF_CODE_WALL || zf_code_pressure(cd))))) return;
      for (int v = 0; v < 3; ++v) acc[v] += w * G[v * a.ns + s];
    });
  }
  for (int v = 0; v < 3; ++v) out[((size_t)v * nc + cell) * n + node] = (float)(acc[v] * a.force_scale);
}

// Es enters the membrane forces through the calibrated springs only, and at
// the calibration's fixed point kT/Plength and kp are both proportional to Es
// (ZebraflowWT.c:1989-1990, :6906-6907); scaling them by s = 2 or 1/2 (exact in
// binary) gives the forces at s Es.
__global__ void k_scale_springs(CellArgs c, float s) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  float* ep = const_cast<float*>(c.epar);
  float* epn = const_cast<float*>(c.epar_n);
  if (e < c.ne) {
    ep[c.ne + e] /= s;     // Plength
    ep[2 * c.ne + e] *= s; // kp
  }
  if (e < c.nen) {
    epn[c.nen + e] /= s;
    epn[2 * c.nen + e] *= s;
  }
}

int wss_launch(zf_ctx* ctx, const float* d_normals, double pgauge, float* d_wss, float* d_press,
               int32_t* d_valid) {
  const IbArgs& a = ctx->ib;
  if (a.nw == 0) return ZF_OK;
  int rc = lbm_moments_launch(ctx);
  if (rc) return rc;
  k_wss<<<(a.nw + 127) / 128, 128, 0, ctx->stream>>>(a, d_normals ? d_normals : a.wnnrm, (float)pgauge,
                                                     d_wss, d_press, d_valid);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

// Lists the patch's stencils (see k_wss_stencil_count); device buffers and
// their sizes are appended to `bufs` (the caller frees them).
int wss_patch_stencil(zf_ctx* ctx, const float* d_nrm, const int32_t* d_patch, int np, PatchStencil& ps,
                      std::vector<std::pair<void*, size_t>>& bufs) {
  ps = PatchStencil{};
  ps.np = np;
  ps.patch = d_patch;
  if (np <= 0) return ZF_OK;
  auto grab = [&](void** p, size_t b) -> int {
    b = b < 4 ? 4 : b;
    int r = dev_alloc(ctx, p, b);
    if (!r) bufs.emplace_back(*p, b);
    return r;
  };
  int32_t* d_cnt = nullptr;
  int rc = grab((void**)&d_cnt, (size_t)np * sizeof(int32_t));
  if (rc) return rc;
  k_wss_stencil_count<<<(np + 127) / 128, 128, 0, ctx->stream>>>(ctx->ib, d_nrm, d_patch, np, d_cnt);
  ZF_CUDA(cudaGetLastError());
  std::vector<int32_t> off(np + 1, 0);
  ZF_CUDA(cudaMemcpyAsync(off.data() + 1, d_cnt, (size_t)np * sizeof(int32_t), cudaMemcpyDeviceToHost,
                          ctx->stream));
  ZF_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < np; ++i) off[i + 1] += off[i];
  const int ne = off[np];
  int32_t *d_off = nullptr, *d_slot = nullptr, *d_idx = nullptr, *d_us = nullptr;
  float* d_w = nullptr;
  if ((rc = grab((void**)&d_off, (size_t)(np + 1) * sizeof(int32_t))) ||
      (rc = grab((void**)&d_slot, (size_t)ne * sizeof(int32_t))) ||
      (rc = grab((void**)&d_w, (size_t)ne * sizeof(float))))
    return rc;
  ZF_CUDA(cudaMemcpyAsync(d_off, off.data(), (size_t)(np + 1) * sizeof(int32_t), cudaMemcpyHostToDevice,
                          ctx->stream));
  k_wss_stencil_fill<<<(np + 127) / 128, 128, 0, ctx->stream>>>(ctx->ib, d_nrm, d_patch, np, d_off, d_slot, d_w);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 2;
  // distinct slots, and each entry's index among them
  std::vector<int32_t> slot(ne), us, idx(ne);
  ZF_CUDA(cudaMemcpyAsync(slot.data(), d_slot, (size_t)ne * sizeof(int32_t), cudaMemcpyDeviceToHost,
                          ctx->stream));
  ZF_CUDA(cudaStreamSynchronize(ctx->stream));
  us = slot;
  std::sort(us.begin(), us.end());
  us.erase(std::unique(us.begin(), us.end()), us.end());
  for (int e = 0; e < ne; ++e) idx[e] = (int32_t)(std::lower_bound(us.begin(), us.end(), slot[e]) - us.begin());
  const int nu = (int)us.size();
  if ((rc = grab((void**)&d_idx, (size_t)ne * sizeof(int32_t))) ||
      (rc = grab((void**)&d_us, (size_t)nu * sizeof(int32_t))))
    return rc;
  ZF_CUDA(cudaMemcpyAsync(d_idx, idx.data(), (size_t)ne * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
  ZF_CUDA(cudaMemcpyAsync(d_us, us.data(), (size_t)nu * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
  ZF_CUDA(cudaStreamSynchronize(ctx->stream));
  ps.off = d_off;
  ps.idx = d_idx;
  ps.w = d_w;
  ps.uslot = d_us;
  ps.nu = nu;
  return ZF_OK;
}

int wss_patch_launch(zf_ctx* ctx, const PatchStencil& ps, const float* d_nrm, const float* d_U, double c,
                     double* d_acc) {
  if (ps.np <= 0) return ZF_OK;
  k_wss_patch<<<(ps.np + 127) / 128, 128, 0, ctx->stream>>>(ctx->ib, ps, d_nrm, d_U, c, d_acc);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

int wss_patch_adj_launch(zf_ctx* ctx, const PatchStencil& ps, const float* d_nrm, const float* d_U, double c,
                         float* d_gU) {
  if (ps.np <= 0) return ZF_OK;
  k_wss_patch_adj<<<(ps.np + 127) / 128, 128, 0, ctx->stream>>>(ctx->ib, ps, d_nrm, d_U, c, d_gU);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

int flux_objective_launch(zf_ctx* ctx, const PatchStencil& ps, const uint8_t* d_set, const float* nrm6,
                          const float* d_U, double c, double* d_q, double* d_acc) {
  if (ps.nu <= 0) return ZF_OK;
  Nrm6 n;
  for (int i = 0; i < 6; ++i) n.v[i] = nrm6[i];
  ZF_CUDA(cudaMemsetAsync(d_q, 0, 2 * sizeof(double), ctx->stream));
  k_flux_q<<<(ps.nu + 255) / 256, 256, 0, ctx->stream>>>(ps, d_set, n, d_U, d_q);
  k_flux_j<<<1, 32, 0, ctx->stream>>>(d_q, c, d_acc);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 2;
  return ZF_OK;
}

int flux_adj_launch(zf_ctx* ctx, const PatchStencil& ps, const uint8_t* d_set, const float* nrm6, const float* d_U,
                    double c, double* d_q, float* d_gU) {
  if (ps.nu <= 0) return ZF_OK;
  Nrm6 n;
  for (int i = 0; i < 6; ++i) n.v[i] = nrm6[i];
  ZF_CUDA(cudaMemsetAsync(d_q, 0, 2 * sizeof(double), ctx->stream));
  k_flux_q<<<(ps.nu + 255) / 256, 256, 0, ctx->stream>>>(ps, d_set, n, d_U, d_q);
  k_flux_gu<<<(ps.nu + 255) / 256, 256, 0, ctx->stream>>>(ps, d_set, n, d_q, c, d_gU);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 2;
  return ZF_OK;
}

int spread_adj_launch(zf_ctx* ctx, const float* d_G, float* d_gmem, float* d_gnuc) {
  const CellArgs& c = ctx->cells;
  const int64_t n = (int64_t)c.n_cells * (c.nn + c.nnn);
  if (n == 0) return ZF_OK;
  k_spread_adj<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(
      ctx->ib, c, ctx->p.wall_mode == ZF_WALL_REF_EQ, d_G, d_gmem, d_gnuc);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

int scale_springs_launch(zf_ctx* ctx, float s) {
  const CellArgs& c = ctx->cells;
  const int n = c.ne > c.nen ? c.ne : c.nen;
  if (n == 0) return ZF_OK;
  k_scale_springs<<<(n + 255) / 256, 256, 0, ctx->stream>>>(c, s);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

namespace {

// the tile kernels need the 3x3x3 tile neighbourhood of a tile to hold every
// window point: along a periodic z axis the tiles must wrap with the lattice
// (nz a multiple of the tile edge) and be at least three
bool tiles_ok(const IbArgs& a) { return !a.per_z || (a.nz % ZF_TS == 0 && a.ntz >= 3); }

template <typename K>
int persistent_blocks(K kernel, int threads) {
  int dev = 0, sms = 0, per_sm = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  ZF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  ZF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
  return sms * (per_sm > 0 ? per_sm : 1);
}

// exclusive scan of in[0..n) into out[0..n]; bsum holds (n+1023)/1024 + 1 ints
void scan_launch(const int32_t* in, int64_t n, int32_t* out, int32_t* bsum, cudaStream_t st) {
  const int nb = (int)((n + 1023) / 1024);
  k_scan_blocks<<<nb, 1024, 0, st>>>(in, n, out, bsum);
  k_scan_sums<<<1, 1024, 0, st>>>(bsum, nb, bsum + nb);
  k_scan_add<<<nb, 1024, 0, st>>>(out, n, bsum);
}

}  // namespace

// Builds the per-point lists of k_wall_rel into ctx->ib (wrel_cnt, wrel_off,
// wrel); device buffers are appended to `own`.
int wall_rel_build(zf_ctx* ctx, std::vector<void*>& own) {
  IbArgs& a = ctx->ib;
  a.wrel_cnt = a.wrel_off = a.wrel = nullptr;
  const int64_t ng = (int64_t)a.ntx * a.nty * a.ntz;
  if (ng == 0 || a.nw == 0 || a.ns_all == 0) return ZF_OK;
  const int64_t n = a.ns_all;
  const int64_t nb = (n + 1 + 1023) / 1024;
  auto grab = [&](void** p, size_t b) -> int {
    int r = dev_alloc(ctx, p, b);
    if (!r) own.push_back(*p);
    return r;
  };
  int32_t *cnt = nullptr, *off = nullptr, *tmp = nullptr, *list = nullptr;
  int rc;
  if ((rc = grab((void**)&cnt, (size_t)n * sizeof(int32_t))) ||
      (rc = grab((void**)&off, (size_t)(n + 1) * sizeof(int32_t))))
    return rc;
  // scratch: clipped counts (n + 1, the last 0) and the scan's block sums
  if ((rc = dev_alloc(ctx, (void**)&tmp, (size_t)(n + 1 + nb + 1) * sizeof(int32_t)))) return rc;
  ZF_CUDA(cudaMemsetAsync(tmp, 0, (size_t)(n + 1) * sizeof(int32_t), ctx->stream));
  k_wall_rel<false><<<(unsigned)ng, ZF_TC, 0, ctx->stream>>>(a, cnt, tmp, nullptr, nullptr);
  ZF_CUDA(cudaGetLastError());
  scan_launch(tmp, n + 1, off, tmp + n + 1, ctx->stream);
  int32_t total = 0;
  ZF_CUDA(cudaMemcpyAsync(&total, off + n, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  ZF_CUDA(cudaStreamSynchronize(ctx->stream));
  cudaFree(tmp);
  ctx->device_bytes -= (int64_t)((n + 1 + nb + 1) * sizeof(int32_t));
  if ((rc = grab((void**)&list, (size_t)std::max<int32_t>(total, 1) * sizeof(int32_t)))) return rc;
  k_wall_rel<true><<<(unsigned)ng, ZF_TC, 0, ctx->stream>>>(a, cnt, nullptr, off, list);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 5;
  a.wrel_cnt = cnt;
  a.wrel_off = off;
  a.wrel = list;
  return ZF_OK;
}

int ib_node_tiles_launch(zf_ctx* ctx) {
  const CellArgs& c = ctx->cells;
  IbArgs& a = ctx->ib;
  const int64_t n = (int64_t)c.n_cells * (c.nn + c.nnn);
  if (n == 0) return ZF_OK;
  const int64_t ng1 = a.ngrid + 1;
  ZF_CUDA(cudaMemsetAsync(a.node_cnt, 0, ng1 * sizeof(int32_t), ctx->stream));
  ZF_CUDA(cudaMemsetAsync(a.tile_ctr, 0, 4 * sizeof(int32_t), ctx->stream));
  k_node_tiles<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(a, c);
  scan_launch(a.node_cnt, ng1, a.node_off, a.node_bsum, ctx->stream);
  ZF_CUDA(cudaMemsetAsync(a.node_cnt, 0, ng1 * sizeof(int32_t), ctx->stream));
  k_node_fill<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(a, c);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 5;
  ctx->node_tiles_valid = true;
  return ZF_OK;
}

int ib_interp_launch(zf_ctx* ctx) {
  const CellArgs& c = ctx->cells;
  IbArgs& a = ctx->ib;
  const int64_t n = (int64_t)c.n_cells * (c.nn + c.nnn);
  if (n == 0) return ZF_OK;
  k_ib_interp<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(a, c);
  ctx->launches += 1;
  if (a.nw > 0) {
    if (tiles_ok(a)) {
      // [0] queued nodes, [1] their work counter
      ZF_CUDA(cudaMemsetAsync(a.wall_walk_ctr, 0, 4 * sizeof(int32_t), ctx->stream));
      k_wall_nodes<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(a, c, a.wall_walk, a.wall_walk_ctr);
      k_wall_lists<<<persistent_blocks(k_wall_lists, kTileThreads), kTileThreads, 0, ctx->stream>>>(
          a, c, a.wall_walk, a.wall_walk_ctr, a.wall_walk_ctr + 3);
      k_wall_walk<<<persistent_blocks(k_wall_walk, kTileThreads), kTileThreads, 0, ctx->stream>>>(
          a, c, a.wall_walk, a.wall_walk_ctr, a.wall_walk_ctr + 1);
      ctx->launches += 2;
    } else {
      k_ib_wall<<<(unsigned)((n + kRepWarps * 32 - 1) / (kRepWarps * 32)), kRepWarps * 32, 0, ctx->stream>>>(
          a, c);
    }
    ctx->launches += 1;
  }
  ZF_CUDA(cudaGetLastError());
  return ZF_OK;
}

int ib_bins_launch(zf_ctx* ctx) {
  const CellArgs& c = ctx->cells;
  IbArgs& a = ctx->ib;
  const int64_t ntri = (int64_t)c.n_cells * c.nt;
  if (ntri == 0) return ZF_OK;
  int32_t* counts = const_cast<int32_t*>(a.bin_off) + (a.ns + 1);  // scratch after off
  int32_t* tri_bin = counts + (a.ns + 1);
  int32_t* bsum = tri_bin + ntri;
  int32_t* off = const_cast<int32_t*>(a.bin_off);
  ZF_CUDA(cudaMemsetAsync(counts, 0, (a.ns + 1) * sizeof(int32_t), ctx->stream));
  k_bin_assign<<<(unsigned)((ntri + 255) / 256), 256, 0, ctx->stream>>>(a, c, tri_bin, counts);
  scan_launch(counts, a.ns + 1, off, bsum, ctx->stream);
  ZF_CUDA(cudaMemsetAsync(counts, 0, (a.ns + 1) * sizeof(int32_t), ctx->stream));
  k_bin_fill<<<(unsigned)((ntri + 255) / 256), 256, 0, ctx->stream>>>(c, tri_bin, off, counts,
                                                                       const_cast<int32_t*>(a.bin_tri), a.bin_kk);
  k_bin_sort<<<(unsigned)((a.ns + 255) / 256), 256, 0, ctx->stream>>>(off, a.ns,
                                                                       const_cast<int32_t*>(a.bin_tri));
  k_bin_records<<<(unsigned)((ntri + 255) / 256), 256, 0, ctx->stream>>>(a, c, off + a.ns);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 7;
  return ZF_OK;
}

int ib_nuc_memb_launch(zf_ctx* ctx, int rebuild) {
  const CellArgs& c = ctx->cells;
  const int64_t n = (int64_t)c.n_cells * c.nnn;
  if (n == 0) return ZF_OK;
  k_nuc_memb<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(ctx->ib, c, rebuild,
                                                                     c.counters + 2);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

int ib_rbc_rbc_launch(zf_ctx* ctx) {
  const CellArgs& c = ctx->cells;
  IbArgs& a = ctx->ib;
  const int64_t n = (int64_t)c.n_cells * c.nn;
  if (n == 0) return ZF_OK;
  if (tiles_ok(a)) {
    if (!ctx->node_tiles_valid) {
      const int rc = ib_node_tiles_launch(ctx);
      if (rc) return rc;
    }
    ZF_CUDA(cudaMemsetAsync(a.tile_ctr + 1, 0, sizeof(int32_t), ctx->stream));
    static bool smem_set[256] = {};
    const size_t smem = sizeof(RgShared);
    if (!smem_set[ctx->device & 255]) {
      ZF_CUDA(cudaFuncSetAttribute(k_rbc_group, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      smem_set[ctx->device & 255] = true;
    }
    int dev = 0, sms = 0, per_sm = 0;
    ZF_CUDA(cudaGetDevice(&dev));
    ZF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ZF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rbc_group, kRgThreads, smem));
    k_rbc_group<<<sms * (per_sm > 0 ? per_sm : 1), kRgThreads, smem, ctx->stream>>>(a, c);
  } else {
    k_rbc_rbc<<<(unsigned)((n + kRepWarps * 32 - 1) / (kRepWarps * 32)), kRepWarps * 32, 0, ctx->stream>>>(
        a, c);
  }
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

int ib_spread_launch(zf_ctx* ctx) {
  const CellArgs& c = ctx->cells;
  IbArgs& a = ctx->ib;
  const int64_t n = (int64_t)c.n_cells * (c.nn + c.nnn);
  if (n == 0) return ZF_OK;
  if (tiles_ok(a) && !ctx->ib_allocs.empty()) {
    if (!ctx->node_tiles_valid) {
      const int rc = ib_node_tiles_launch(ctx);
      if (rc) return rc;
    }
    ZF_CUDA(cudaMemsetAsync(a.tile_ctr + 3, 0, sizeof(int32_t), ctx->stream));
    k_spread_tiles<<<persistent_blocks(k_spread_tiles, 256), 256, 0, ctx->stream>>>(
        a, c, ctx->p.wall_mode == ZF_WALL_REF_EQ);
  } else {
    k_ib_spread<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(a, c, ctx->p.wall_mode == ZF_WALL_REF_EQ);
  }
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

// node velocities and repulsion velocities <-> one fp64 buffer
// [vel: 3 nc nn][vel_n: 3 nc nnn][wrep: 3 nc nn] (dir 0: into the buffer, 1: back)
__global__ void k_kin_buffer(CellArgs c, double* buf, int dir) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nm = 3 * (int64_t)c.n_cells * c.nn, nn_ = 3 * (int64_t)c.n_cells * c.nnn;
  if (i >= 2 * nm + nn_) return;
  if (i < nm) {
    if (dir == 0) buf[i] = c.vel[i];
    else c.vel[i] = buf[i];
  } else if (i < nm + nn_) {
    if (dir == 0) buf[i] = c.vel_n[i - nm];
    else c.vel_n[i - nm] = buf[i];
  } else {
    if (dir == 0) buf[i] = (double)c.wrep[i - nm - nn_];
    else c.wrep[i - nm - nn_] = (float)buf[i];
  }
}

int ib_kin_buffer_launch(zf_ctx* ctx, double* buf, int dir) {
  const CellArgs& c = ctx->cells;
  const int64_t n = 3 * (int64_t)c.n_cells * (2 * c.nn + c.nnn);
  if (n == 0) return ZF_OK;
  k_kin_buffer<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(c, buf, dir);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

int ib_update_launch(zf_ctx* ctx) {
  const CellArgs& c = ctx->cells;
  if (c.n_cells == 0) return ZF_OK;
  const int rc = cells_write_fence(ctx);  // positions and statuses change
  if (rc) return rc;
  k_update<<<c.n_cells, 256, 0, ctx->stream>>>(ctx->ib, c);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  ctx->node_tiles_valid = false;  // positions moved
  return ZF_OK;
}

}  // namespace zf

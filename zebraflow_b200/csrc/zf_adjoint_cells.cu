// Adjoint pieces of the cells' side of the coupled step.
//
// k_membrane_vjp: the vector-Jacobian product of the membrane and nucleus
// forces of k_membrane (ZebraflowWT.c:5749-7535) with respect to the node
// positions, Es and kb: given lam (the adjoint of the force of every node),
//   gx  += lam^T dF/dx,   gEs += lam^T dF/dEs,   gkb += lam^T dF/dkb.
// One CTA per cell.  Each edge thread recomputes its term of the forward in
// forward-mode dual numbers: 18 tangents, the 12 coordinates of its four nodes,
// the cell centroid (3), the global-area force FAG (1), Es and kb.  The
// per-cell couplings (centroid, cell area -> FAG, volume -> FVS) are chained in
// a second pass over the triangles, whose own terms (area, volume and the
// sliver push) use 9-tangent duals.  Branches (clamps, screening of large
// terms, the |cos| > 0.99 cut of bending) follow the forward's values, so the
// product is the derivative of the branch the forward took.  Cells the
// forward removed (status <= -5000) contribute nothing.
//
// k_ib_vjp: the transposes of one membrane iteration's IB interpolation
// (ZebraflowWT.c:8963-8996), spreading (:10745-10870) and position update
// (:11965-11997) at the positions x the iteration started from, one thread
// per node:
//   update      x' = x + dt (u_interp + wrep)       lam_u = dt lam_x'
//   spreading   BF(s) += fs w(s; x) Fsp,  Fsp = gamma_p wrep + ftot
//               lam_F  = fs sum_s w G(s)             (G = dJ/dBF)
//               lam_x += fs sum_s grad_x w (Fsp . G(s))
//   interp      u = sum_s w(s; x) vs U(s)
//               GU(s) += vs w lam_u   (fluid points; the seed of dJ/dU)
//               lam_x += vs sum_s grad_x w (U(s) . lam_u)
// with w = prod_a (1 + cos(pi |d_a| / (2 DX))) / 64, d_a = x_lat,a - x_a, so
// dw/dx_a = (pi / (2 DX)) sin(pi |d_a| / (2 DX)) sign(d_a) prod_{b != a}(...) / 64.
// It also forms lam_w = lam_u + gamma_p lam_F, the adjoint of the repulsion
// velocities wrep, which k_rbc_vjp, k_wall_vjp and k_nuc_vjp (below) carry
// through the RBC-RBC (:9919-10053), wall (:9055-9077) and nucleus-membrane
// (:9516-9730) repulsions to the positions.
#include "zf_internal.h"

namespace zf {

namespace {

// ---- forward-mode dual numbers ---------------------------------------------------

template <int N>
struct Dl {
  float v;
  float d[N];
};

template <int N>
__device__ __forceinline__ Dl<N> cst(float v) {
  Dl<N> r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = 0.f;
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> var(float v, int k) {
  Dl<N> r = cst<N>(v);
  r.d[k] = 1.f;
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> operator+(const Dl<N>& a, const Dl<N>& b) {
  Dl<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> operator-(const Dl<N>& a, const Dl<N>& b) {
  Dl<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> operator-(const Dl<N>& a) {
  Dl<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> operator*(const Dl<N>& a, const Dl<N>& b) {
  Dl<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> operator*(float s, const Dl<N>& a) {
  Dl<N> r;
  r.v = s * a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> operator+(const Dl<N>& a, float s) {
  Dl<N> r = a;
  r.v += s;
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> operator/(const Dl<N>& a, const Dl<N>& b) {
  Dl<N> r;
  const float ib = 1.f / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> inv(const Dl<N>& b) {
  Dl<N> r;
  const float ib = 1.f / b.v;
  r.v = ib;
  const float k = -ib * ib;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = k * b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dl<N> dsqrt(const Dl<N>& a) {
  Dl<N> r;
  r.v = sqrtf(a.v);
  const float k = r.v > 0.f ? 0.5f / r.v : 0.f;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = k * a.d[i];
  return r;
}

template <int N>
struct V3d {
  Dl<N> x, y, z;
};
template <int N>
__device__ __forceinline__ V3d<N> vsub(const V3d<N>& a, const V3d<N>& b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int N>
__device__ __forceinline__ V3d<N> vadd(const V3d<N>& a, const V3d<N>& b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <int N>
__device__ __forceinline__ V3d<N> vmul(float s, const V3d<N>& a) {
  return {s * a.x, s * a.y, s * a.z};
}
template <int N>
__device__ __forceinline__ V3d<N> vmul(const Dl<N>& s, const V3d<N>& a) {
  return {s * a.x, s * a.y, s * a.z};
}
template <int N>
__device__ __forceinline__ Dl<N> vdot(const V3d<N>& a, const V3d<N>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <int N>
__device__ __forceinline__ V3d<N> vcross(const V3d<N>& a, const V3d<N>& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <int N>
__device__ __forceinline__ V3d<N> vzero() {
  return {cst<N>(0.f), cst<N>(0.f), cst<N>(0.f)};
}
// the forward's screening of a force term (k_membrane bad_components)
template <int N>
__device__ __forceinline__ bool bad(const V3d<N>& f) {
  auto b = [](float v) { return isnan(v) || isinf(v) || fabsf(v) > 1.e-10f; };
  return b(f.x.v) || b(f.y.v) || b(f.z.v);
}
// lam . d(f)/d(tangent k), accumulated into acc[k] for all k
template <int N>
__device__ __forceinline__ void vjp_acc(float (&acc)[N], const V3d<N>& f, float lx, float ly, float lz) {
#pragma unroll
  for (int k = 0; k < N; ++k) acc[k] += lx * f.x.d[k] + ly * f.y.d[k] + lz * f.z.d[k];
}

__device__ double bsum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < nw; ++i) t += red[i];
  return t;
}

__device__ __forceinline__ void satom3(float* p, int n, int i, float x, float y, float z) {
  atomicAdd(&p[i], x);
  atomicAdd(&p[n + i], y);
  atomicAdd(&p[2 * n + i], z);
}

}  // namespace

// ---- membrane and nucleus forces -------------------------------------------------

namespace {

constexpr int kEd = 18;  // edge tangents: 4 nodes x 3, centroid 3, FAG, Es, kb
constexpr int kTd = 9;   // triangle tangents: 3 nodes x 3
constexpr int kNd = 7;   // nucleus-edge tangents: 2 nodes x 3, Es
using DE = Dl<kEd>;
using VE = V3d<kEd>;
using DT = Dl<kTd>;
using VT = V3d<kTd>;

struct VjpArgs {
  const float* lam;    // [3][nc][nn] adjoint of the membrane node forces (ftot)
  const float* lam_n;  // [3][nc][nnn] adjoint of the nucleus node forces (ftot_n)
  float* gx;           // [3][nc][nn]  += lam^T dF/dx
  float* gxn;          // [3][nc][nnn] += lam^T dF/dxn
  double* gpar;        // [2] += lam^T dF/dEs, lam^T dF/dkb
  float Es;            // shear modulus the springs are calibrated for
};

// one triangle's area vector A = 0.5e-12 (p2 - p1) x (p1 - p3), its area and
// centroid, as k_membrane's CGSM_AREA pass forms them
template <int N>
__device__ __forceinline__ void tri_geom(const V3d<N>& p1, const V3d<N>& p2, const V3d<N>& p3, Dl<N>& ar,
                                         V3d<N>& nrm, V3d<N>& c) {
  const float third = 1.f / 3.f;
  c = {third * (p1.x + p2.x + p3.x), third * (p1.y + p2.y + p3.y), third * (p1.z + p2.z + p3.z)};
  const V3d<N> A = vmul(0.5e-12f, vcross(vsub(p2, p1), vsub(p1, p3)));
  ar = dsqrt(vdot(A, A));
  nrm = vmul(-inv(ar), A);
}

__device__ __forceinline__ float3 ldx(const float* xs, int nn, int i) {
  return make_float3(xs[i], xs[nn + i], xs[2 * nn + i]);
}

}  // namespace

__global__ void __launch_bounds__(256) k_membrane_vjp(CellArgs a, VjpArgs v) {
  const int cell = blockIdx.x;
  if (a.status[cell] <= -5000) return;
  const int nn = a.nn, nt = a.nt, ne = a.ne, nnn = a.nnn, nen = a.nen, nc = a.n_cells;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* red = reinterpret_cast<double*>(smem_raw);
  float* xs = reinterpret_cast<float*>(red + 32);
  float* gs = xs + 3 * nn;
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int i = tid; i < nn; i += nth)
    for (int c = 0; c < 3; ++c) {
      xs[c * nn + i] = (float)a.x[((size_t)c * nc + cell) * nn + i];
      gs[c * nn + i] = 0.f;
    }
  __syncthreads();

  // the forward's per-cell values: area, centroid, volume, FAG, FVS
  double asum = 0.0, vsum = 0.0;
  for (int t = tid; t < nt; t += nth) {
    const float3 p1 = ldx(xs, nn, a.tri[3 * t]), p2 = ldx(xs, nn, a.tri[3 * t + 1]),
                 p3 = ldx(xs, nn, a.tri[3 * t + 2]);
    const float cx = (p1.x + p2.x + p3.x) / 3.f, cy = (p1.y + p2.y + p3.y) / 3.f, cz = (p1.z + p2.z + p3.z) / 3.f;
    const float e1x = p2.x - p1.x, e1y = p2.y - p1.y, e1z = p2.z - p1.z;
    const float e3x = p1.x - p3.x, e3y = p1.y - p3.y, e3z = p1.z - p3.z;
    const float Ax = 0.5e-12f * (e1y * e3z - e1z * e3y), Ay = 0.5e-12f * (e1z * e3x - e1x * e3z),
                Az = 0.5e-12f * (e1x * e3y - e1y * e3x);
    const float ar = sqrtf(Ax * Ax + Ay * Ay + Az * Az);
    const float nx = -Ax / ar, ny = -Ay / ar, nz = -Az / ar;
    asum += (double)ar;
    vsum += (double)(ar * (cx * nx + cy * ny + cz * nz) * 1.e-006f);
  }
  const double cell_area = bsum(asum, red);
  const float vol = (float)(bsum(vsum, red) / 3.0);
  double cx = 0.0, cy = 0.0, cz = 0.0;
  for (int i = tid; i < nn; i += nth) {
    cx += (double)(xs[i] / (float)nn);
    cy += (double)(xs[nn + i] / (float)nn);
    cz += (double)(xs[2 * nn + i] / (float)nn);
  }
  const float Cx = (float)bsum(cx, red), Cy = (float)bsum(cy, red), Cz = (float)bsum(cz, red);
  const float FAG = -a.ka * ((float)cell_area - a.area0) / a.area0;
  const float FVS = -a.kv * (vol - a.volume0) / a.volume0;

  const float* LMAX = a.epar;
  const float* PLEN = a.epar + ne;
  const float* KP = a.epar + 2 * ne;
  const float* SIN0 = a.epar + 3 * ne;
  const float* COS0 = a.epar + 4 * ne;
  const float* L = v.lam;
  double gC[3] = {0.0, 0.0, 0.0}, gFAG = 0.0, gFVS = 0.0, gEs = 0.0, gkb = 0.0;
  const VE Cd = {var<kEd>(Cx, 12), var<kEd>(Cy, 13), var<kEd>(Cz, 14)};
  const DE FAGd = var<kEd>(FAG, 15);
  for (int e = tid; e < ne; e += nth) {
    const int* E = a.edge + 6 * e;
    const int nd[4] = {E[0], E[1], E[2], E[3]};
    const int t1 = E[4], t2 = E[5];
    VE c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float3 p = ldx(xs, nn, nd[k]);
      c[k] = {var<kEd>(p.x, 3 * k), var<kEd>(p.y, 3 * k + 1), var<kEd>(p.z, 3 * k + 2)};
    }
    // a triangle vertex as a dual: one of the edge's four nodes, else held
    auto pos = [&](int id) -> VE {
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (id == nd[k]) return c[k];
      const float3 p = ldx(xs, nn, id);
      return {cst<kEd>(p.x), cst<kEd>(p.y), cst<kEd>(p.z)};
    };
    float lam[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int q = 0; q < 3; ++q) lam[k][q] = L[((size_t)q * nc + cell) * nn + nd[k]];
    float acc[kEd];
#pragma unroll
    for (int k = 0; k < kEd; ++k) acc[k] = 0.f;

    // WLC + POW springs
    {
      const VE d12 = vsub(c[0], c[1]);
      DE len = dsqrt(vdot(d12, d12));
      const DE il = inv(len);
      const VE e1v = vmul(il, d12);
      const VE e2v = vmul(-il, d12);
      DE er = (1.e-06f / LMAX[e]) * len;
      if (er.v > 0.95f) er = cst<kEd>(0.95f);
      if (er.v < 0.02435f) len = cst<kEd>(0.02435f * LMAX[e] / 1.e-06f);
      const float kt = -a.kT / PLEN[e];
      DE kts = cst<kEd>(kt);
      kts.d[16] = kt / v.Es;
      DE kps = cst<kEd>(KP[e]);
      kps.d[16] = KP[e] / v.Es;
      const DE om = cst<kEd>(1.f) - er;
      const DE wlc = kts * ((er + (-0.25f)) + inv(4.f * (om * om)));
      const DE comp = kps * inv(1.e-012f * (len * len));
      const DE s = wlc + comp;
      vjp_acc(acc, vmul(s, e1v), lam[0][0], lam[0][1], lam[0][2]);
      vjp_acc(acc, vmul(s, e2v), lam[1][0], lam[1][1], lam[1][2]);
    }
    // the rhombus: triangles t1 = (n1, n2, n3) and t2 = (n2, n1, n4)
    DE A1, A2;
    VE N1, N2, C1, C2;
    tri_geom(pos(a.tri[3 * t1]), pos(a.tri[3 * t1 + 1]), pos(a.tri[3 * t1 + 2]), A1, N1, C1);
    tri_geom(pos(a.tri[3 * t2]), pos(a.tri[3 * t2 + 1]), pos(a.tri[3 * t2 + 2]), A2, N2, C2);
    const float A1eq = a.tri_area_eq[t1], A2eq = a.tri_area_eq[t2];
    if (A1.v < 0.1f * A1eq) A1 = cst<kEd>(0.1f * A1eq);
    else if (A1.v > 10.f * A1eq) A1 = cst<kEd>(10.f * A1eq);
    if (A2.v < 0.1f * A2eq) A2 = cst<kEd>(0.1f * A2eq);
    else if (A2.v > 10.f * A2eq) A2 = cst<kEd>(10.f * A2eq);
    const VE dp21 = vmul(1.e-6f, vsub(c[1], c[0])), dp24 = vmul(1.e-6f, vsub(c[1], c[3])),
             dp32 = vmul(1.e-6f, vsub(c[2], c[1])), dp41 = vmul(1.e-6f, vsub(c[3], c[0])),
             dp13 = vmul(1.e-6f, vsub(c[0], c[2]));
    const VE cp1 = vmul(A1, vcross(N1, dp21)), cp2 = vmul(A2, vcross(N2, dp21));
    const VE cp5 = vmul(A1, vcross(N1, dp32)), cp9 = vmul(A1, vcross(N1, dp13));
    const VE cp4 = vmul(A2, vcross(N2, dp24)), cp8 = vmul(A2, vcross(N2, dp41));

    // bending
    {
      DE cs = vdot(N1, N2);
      if (cs.v > 1.f) cs = cst<kEd>(1.f);
      else if (cs.v < -1.f) cs = cst<kEd>(-1.f);
      if (!(fabsf(cs.v) > 0.99f)) {
        const float ac = vdot(vsub(N1, N2), vmul(1.e-006f, vsub(C1, C2))).v;
        DE sn = dsqrt(cst<kEd>(1.f) - cs * cs);
        if (!(ac >= 0.f)) sn = -sn;
        DE kb = var<kEd>(a.kbend, 17);
        const DE beta = kb * ((COS0[e] * sn - SIN0[e] * cs) / sn);
        const VE cp3 = vmul(A1, vcross(N1, dp24)), cp6 = vmul(A2, vcross(N2, dp32));
        const VE cp7 = vmul(A1, vcross(N1, dp41)), cp10 = vmul(A2, vcross(N2, dp13));
        const DE b11 = -(beta * cs) / (A1 * A1);
        const DE b12 = beta / (A1 * A2);
        const DE b22 = -(beta * cs) / (A2 * A2);
        const VE fb1 = vadd(vadd(vmul(b11, cp5), vmul(b12, vadd(cp3, cp6))), vmul(b22, cp4));
        const VE fb2 = vadd(vadd(vmul(b11, cp9), vmul(b12, vadd(cp7, cp10))), vmul(b22, cp8));
        const VE fb3 = vadd(vmul(b11, cp1), vmul(b12, cp2));
        const VE fb4 = vadd(vmul(-b12, cp1), vmul(-b22, cp2));
        if (!bad(fb1)) vjp_acc(acc, fb1, lam[0][0], lam[0][1], lam[0][2]);
        if (!bad(fb2)) vjp_acc(acc, fb2, lam[1][0], lam[1][1], lam[1][2]);
        if (!bad(fb3)) vjp_acc(acc, fb3, lam[2][0], lam[2][1], lam[2][2]);
        if (!bad(fb4)) vjp_acc(acc, fb4, lam[3][0], lam[3][1], lam[3][2]);
      }
    }
    // local area, global area and volume terms by each triangle's first edge
    for (int side = 0; side < 2; ++side) {
      if (!((a.area_first[e] >> side) & 1)) continue;
      const DE& Ar = side ? A2 : A1;
      const float Aeq = side ? A2eq : A1eq;
      const VE& Nr = side ? N2 : N1;
      const VE lc = vmul(1.e-006f, vsub(side ? C2 : C1, Cd));
      const DE al = (-a.kd / (4.f * Aeq)) * ((Ar + (-Aeq)) / Ar);
      const DE ag = 0.25f * (FAGd / Ar);
      const VE m2 = vmul(-1.f, cp2);
      const VE cpk[3] = {side ? cp4 : cp5, side ? cp8 : cp9, side ? m2 : cp1};
      const VE base = vmul(1.f / 3.f, vmul(Ar, Nr));
      const VE fv[3] = {vmul(1.f / 6.f, vadd(base, vcross(lc, side ? dp24 : dp32))),
                        vmul(1.f / 6.f, vadd(base, vcross(lc, side ? dp41 : dp13))),
                        vmul(1.f / 6.f, vadd(base, side ? vmul(-1.f, vcross(lc, dp21)) : vcross(lc, dp21)))};
      const int tk[3] = {0, 1, side ? 3 : 2};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float* lk = lam[tk[k]];
        const VE fa = vmul(al, cpk[k]);
        if (!bad(fa)) vjp_acc(acc, fa, lk[0], lk[1], lk[2]);
        const VE fg = vmul(ag, cpk[k]);
        if (!bad(fg)) vjp_acc(acc, fg, lk[0], lk[1], lk[2]);
        if (!bad(fv[k])) {
          vjp_acc(acc, fv[k], FVS * lk[0], FVS * lk[1], FVS * lk[2]);
          gFVS += (double)(lk[0] * fv[k].x.v + lk[1] * fv[k].y.v + lk[2] * fv[k].z.v);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) satom3(gs, nn, nd[k], acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]);
    gC[0] += acc[12];
    gC[1] += acc[13];
    gC[2] += acc[14];
    gFAG += acc[15];
    gEs += acc[16];
    gkb += acc[17];
  }
  const double sC0 = bsum(gC[0], red), sC1 = bsum(gC[1], red), sC2 = bsum(gC[2], red);
  const double sFAG = bsum(gFAG, red), sFVS = bsum(gFVS, red);
  const double sEs = bsum(gEs, red), skb = bsum(gkb, red);
  // chain of FAG = -ka (A_cell - A0)/A0 and FVS = -kv (V - V0)/V0 to the
  // triangles' areas and volume terms, and the sliver push (k_membrane's
  // CGSM_AREA pass, ZebraflowWT.c:6042-6084)
  const float g_area = (float)(sFAG * (double)(-a.ka / a.area0));
  const float g_vol = (float)(sFVS * (double)(-a.kv / a.volume0));
  for (int t = tid; t < nt; t += nth) {
    const int nd[3] = {a.tri[3 * t], a.tri[3 * t + 1], a.tri[3 * t + 2]};
    VT p[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float3 q = ldx(xs, nn, nd[k]);
      p[k] = {var<kTd>(q.x, 3 * k), var<kTd>(q.y, 3 * k + 1), var<kTd>(q.z, 3 * k + 2)};
    }
    DT ar;
    VT nrm, c;
    tri_geom(p[0], p[1], p[2], ar, nrm, c);
    const DT volt = (1.e-006f / 3.f) * (ar * vdot(c, nrm));
    float acc[kTd];
#pragma unroll
    for (int k = 0; k < kTd; ++k) acc[k] = g_area * ar.d[k] + g_vol * volt.d[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const VT e = vsub(p[k], c);
      const DT l = dsqrt(vdot(e, e));
      if (l.v < 0.05f) {
        const DT il = inv(l);
        const VT u = vmul(il, e);
        const VT f = l.v > 0.001f ? vmul(1.e-14f * il, u) : vmul(1.e-11f, u);
        vjp_acc(acc, f, L[((size_t)0 * nc + cell) * nn + nd[k]], L[((size_t)1 * nc + cell) * nn + nd[k]],
                L[((size_t)2 * nc + cell) * nn + nd[k]]);
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) satom3(gs, nn, nd[k], acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]);
  }
  __syncthreads();
  // the centroid is the mean of the nodes
  const float gcx = (float)(sC0 / nn), gcy = (float)(sC1 / nn), gcz = (float)(sC2 / nn);
  for (int i = tid; i < nn; i += nth) {
    v.gx[((size_t)0 * nc + cell) * nn + i] += gs[i] + gcx;
    v.gx[((size_t)1 * nc + cell) * nn + i] += gs[nn + i] + gcy;
    v.gx[((size_t)2 * nc + cell) * nn + i] += gs[2 * nn + i] + gcz;
  }

  // nucleus springs, ZebraflowWT.c:7388-7471
  double gEs_n = 0.0;
  for (int e = tid; e < nen; e += nth) {
    const int n1 = a.edge_n[2 * e], n2 = a.edge_n[2 * e + 1];
    V3d<kNd> c1, c2;
    {
      const double* X = a.xn;
      c1 = {var<kNd>((float)X[((size_t)0 * nc + cell) * nnn + n1], 0),
            var<kNd>((float)X[((size_t)1 * nc + cell) * nnn + n1], 1),
            var<kNd>((float)X[((size_t)2 * nc + cell) * nnn + n1], 2)};
      c2 = {var<kNd>((float)X[((size_t)0 * nc + cell) * nnn + n2], 3),
            var<kNd>((float)X[((size_t)1 * nc + cell) * nnn + n2], 4),
            var<kNd>((float)X[((size_t)2 * nc + cell) * nnn + n2], 5)};
    }
    const V3d<kNd> d12 = vsub(c1, c2);
    Dl<kNd> len = dsqrt(vdot(d12, d12));
    const Dl<kNd> il = inv(len);
    const float LM = a.epar_n[e], PL = a.epar_n[nen + e], KPn = a.epar_n[2 * nen + e];
    Dl<kNd> er = (1.e-06f / LM) * len;
    if (er.v > 0.95f) er = cst<kNd>(0.95f);
    if (er.v < 0.02435f) len = cst<kNd>(0.02435f * LM / 1.e-06f);
    const float kt = -a.kT / PL;
    Dl<kNd> kts = cst<kNd>(kt), kps = cst<kNd>(KPn);
    kts.d[6] = kt / v.Es;
    kps.d[6] = KPn / v.Es;
    const Dl<kNd> om = cst<kNd>(1.f) - er;
    const Dl<kNd> s = kts * ((er + (-0.25f)) + inv(4.f * (om * om))) + kps * inv(1.e-012f * (len * len));
    const V3d<kNd> f1 = vmul(s * il, d12);
    float acc[kNd];
#pragma unroll
    for (int k = 0; k < kNd; ++k) acc[k] = 0.f;
    const float* Ln = v.lam_n;
    const float l1[3] = {Ln[((size_t)0 * nc + cell) * nnn + n1], Ln[((size_t)1 * nc + cell) * nnn + n1],
                         Ln[((size_t)2 * nc + cell) * nnn + n1]};
    const float l2[3] = {Ln[((size_t)0 * nc + cell) * nnn + n2], Ln[((size_t)1 * nc + cell) * nnn + n2],
                         Ln[((size_t)2 * nc + cell) * nnn + n2]};
    // f2 = -f1
    vjp_acc(acc, f1, l1[0] - l2[0], l1[1] - l2[1], l1[2] - l2[2]);
    float* G = v.gxn;
    for (int q = 0; q < 3; ++q) {
      atomicAdd(&G[((size_t)q * nc + cell) * nnn + n1], acc[q]);
      atomicAdd(&G[((size_t)q * nc + cell) * nnn + n2], acc[3 + q]);
    }
    gEs_n += acc[6];
  }
  const double sEs_n = bsum(gEs_n, red);
  if (tid == 0) {
    atomicAdd(&v.gpar[0], sEs + sEs_n);
    atomicAdd(&v.gpar[1], skb);
  }
}

size_t membrane_vjp_smem_bytes(const CellArgs& a) { return 32 * sizeof(double) + sizeof(float) * 6 * a.nn; }

int membrane_vjp_launch(zf_ctx* c, const float* lam, const float* lam_n, float* gx, float* gxn, double* gpar) {
  const CellArgs& a = c->cells;
  if (a.n_cells == 0) return ZF_OK;
  VjpArgs v{lam, lam_n, gx, gxn, gpar, (float)c->p.Es};
  const size_t smem = membrane_vjp_smem_bytes(a);
  ZF_CUDA(cudaFuncSetAttribute(k_membrane_vjp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_membrane_vjp<<<a.n_cells, 256, smem, c->stream>>>(a, v);
  ZF_CUDA(cudaGetLastError());
  c->launches += 1;
  return ZF_OK;
}

// ---- interpolation, spreading and position update --------------------------------

namespace {

constexpr double kPi = 3.14159265358979;  // PI, ZebraflowWT.c:34

__device__ __forceinline__ int lat_idx(float x, double x0, double dx) {
  return (int)floor(((double)x - x0) / dx + 1.01) - 1;
}
__device__ __forceinline__ int64_t slot_at(const IbArgs& a, int i, int j, int k) {
  if (a.per_z) k = ((k % a.nz) + a.nz) % a.nz;
  const int t = a.tile_map[((k >> 2) * a.nty + (j >> 2)) * a.ntx + (i >> 2)];
  if (t < 0) return -1;
  return (int64_t)t * ZF_TC + (i & 3) + 4 * (j & 3) + 16 * (k & 3);
}

// one axis of the Peskin stencil (k_ib_interp's stencil_axis) with the
// derivative of each factor 1 + cos(pi |d| / (2 DX)) with respect to the node
// coordinate
struct GradAxis {
  int b;
  unsigned ok;
  float s[4];   // d^2
  float f[4];   // 1 + cos
  float g[4];   // d(1 + cos)/dx_node
};

__device__ __forceinline__ void grad_axis(GradAxis& ax, float xp, double x0, double dx, int lo, int hi) {
  const int i0 = lat_idx(xp, x0, dx);
  ax.b = (int)floor(((double)xp - x0) / dx) - 1;
  ax.ok = 0u;
  const double h2 = 2.0 * dx;
  const float k = (float)(kPi / h2);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int i = ax.b + m;
    if (i >= lo && i <= hi && i >= i0 - 4 && i <= i0 + 4) ax.ok |= 1u << m;
    const float d = (float)(x0 + i * dx) - xp;
    ax.s[m] = __fmul_rn(d, d);
    const float arg = (float)(kPi * (double)fabsf(d) / h2);
    ax.f[m] = 1.f + cosf(arg);
    ax.g[m] = d > 0.f ? k * sinf(arg) : (d < 0.f ? -k * sinf(arg) : 0.f);
  }
}

struct IbVjpArgs {
  const float* G;        // [3][ns] dJ/dBODYFORCE of the field this iteration spread, or null
  const float* lam_x;    // [3][nc][nn] adjoint of the updated positions, or null (no update)
  const float* lam_xn;   // [3][nc][nnn]
  float* gx;             // [3][nc][nn]  += position terms (may be lam_x itself)
  float* gxn;            // [3][nc][nnn]
  float* gF;             // [3][nc][nn]  := adjoint of the spread node forces
  float* gFn;            // [3][nc][nnn]
  float* GU;             // [3][ns] += dJ/dU (fluid points), with lam_x
  float* lam_w;          // [3][nc][nn] := adjoint of the membrane nodes' repulsion velocities, or null
  const float* ftot;     // the spread forces: gamma_p wrep + ftot, as the forward formed them
  const float* ftot_n;
  const float* wrep;
  const float* wrep_n;
  int spread_walls;
};

}  // namespace

// one thread per node: membrane nodes of all cells, then nucleus nodes
__global__ void k_ib_vjp(IbArgs a, CellArgs c, IbVjpArgs v) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  const int64_t nmem = (int64_t)nc * c.nn;
  const bool nuc = gid >= nmem;
  if (gid >= nmem + (int64_t)nc * c.nnn) return;
  const int n = nuc ? c.nnn : c.nn;
  const int64_t lid = nuc ? gid - nmem : gid;
  const int cell = (int)(lid / n), node = (int)(lid % n);
  auto at = [&](int q) { return ((size_t)q * nc + cell) * n + node; };
  float* gF = nuc ? v.gFn : v.gF;
  if (c.status[cell] <= 0) {
    for (int q = 0; q < 3; ++q) {
      gF[at(q)] = 0.f;
      if (v.lam_w && !nuc) v.lam_w[at(q)] = 0.f;
    }
    return;
  }
  const double* X = nuc ? c.xn : c.x;
  const float xp = (float)X[at(0)], yp = (float)X[at(1)];
  double zd = X[at(2)];
  if (a.LZ > 0.f) zd -= (double)a.LZ * floor((zd - a.Z0) / (double)a.LZ);
  const float zp = (float)zd;
  float Fs[3] = {0.f, 0.f, 0.f}, lu[3] = {0.f, 0.f, 0.f};
  if (v.G) {
    const float* FT = nuc ? v.ftot_n : v.ftot;
    const float* R = nuc ? v.wrep_n : v.wrep;
    for (int q = 0; q < 3; ++q) Fs[q] = (float)((double)a.gamma_p * (double)R[at(q)] + (double)FT[at(q)]);
  }
  const float* LX = nuc ? v.lam_xn : v.lam_x;
  if (LX)
    for (int q = 0; q < 3; ++q) lu[q] = (float)(a.dt_stagger * (double)LX[at(q)]);
  GradAxis AX, AY, AZ;
  grad_axis(AX, xp, a.X0, a.DX, 0, a.nx - 1);
  grad_axis(AY, yp, a.Y0, a.DX, 0, a.ny - 1);
  grad_axis(AZ, zp, a.Z0, a.DX, a.kmin, a.kmax);
  const float h2 = 2.f * a.DX;
  double gf[3] = {0.0, 0.0, 0.0}, gp[3] = {0.0, 0.0, 0.0};
  const double fs = a.force_scale, vs = (double)a.vel_scale;
  for (int mi = 0; mi < 4; ++mi) {
    if (!((AX.ok >> mi) & 1u)) continue;
    for (int mj = 0; mj < 4; ++mj) {
      if (!((AY.ok >> mj) & 1u)) continue;
      const float sxy = __fadd_rn(AX.s[mi], AY.s[mj]);
      for (int mk = 0; mk < 4; ++mk) {
        if (!((AZ.ok >> mk) & 1u)) continue;
        if (!(sqrtf(__fadd_rn(sxy, AZ.s[mk])) <= h2)) continue;
        const double fx = AX.f[mi], fy = AY.f[mj], fz = AZ.f[mk];
        const double w = fx * fy * fz / 64.0;
        if (!(w > 0.0)) continue;
        const double dw[3] = {AX.g[mi] * fy * fz / 64.0, fx * AY.g[mj] * fz / 64.0, fx * fy * AZ.g[mk] / 64.0};
        const int64_t s = slot_at(a, AX.b + mi, AY.b + mj, AZ.b + mk);
        if (s < 0) continue;
        const uint8_t cd = a.code[s];
        if (v.G && s < a.ns &&
            (zf_code_fluid(cd) || (v.spread_walls && (cd == ZF_CODE_WALL || zf_code_pressure(cd))))) {
          double fg = 0.0;
          for (int q = 0; q < 3; ++q) {
            const double g = v.G[q * a.ns + s];
            gf[q] += w * g;
            fg += (double)Fs[q] * g;
          }
          for (int q = 0; q < 3; ++q) gp[q] += fs * dw[q] * fg;
        }
        if (LX) {
          const bool fluid = (zf_code_fluid(cd) || zf_code_pressure(cd)) && s < a.ns;
          if (!fluid && a.windex[s] <= 0) continue;
          float U[3];
          if (fluid) {
            for (int q = 0; q < 3; ++q) U[q] = a.mom[(1 + q) * a.ns + s];
          } else {
            for (int q = 0; q < 3; ++q) U[q] = a.uvoid[q * a.ns_all + s];
          }
          const double ul = (double)U[0] * lu[0] + (double)U[1] * lu[1] + (double)U[2] * lu[2];
          for (int q = 0; q < 3; ++q) gp[q] += vs * dw[q] * ul;
          if (fluid && v.GU)
            for (int q = 0; q < 3; ++q) atomicAdd(&v.GU[q * a.ns + s], (float)(vs * w * (double)lu[q]));
        }
      }
    }
  }
  float* GX = nuc ? v.gxn : v.gx;
  for (int q = 0; q < 3; ++q) {
    const float g = (float)(gf[q] * fs);
    gF[at(q)] = g;
    GX[at(q)] += (float)gp[q];
    // the repulsion velocity wrep moves the node (update) and is spread as
    // gamma_p wrep (:10749-10754)
    if (v.lam_w && !nuc) v.lam_w[at(q)] = lu[q] + a.gamma_p * g;
  }
}

int ib_vjp_launch(zf_ctx* ctx, const float* G, const float* lam_x, const float* lam_xn, float* gx, float* gxn,
                  float* gF, float* gFn, float* GU, float* lam_w, const float* ftot, const float* ftot_n,
                  const float* wrep, const float* wrep_n) {
  const CellArgs& c = ctx->cells;
  const int64_t n = (int64_t)c.n_cells * (c.nn + c.nnn);
  if (n == 0) return ZF_OK;
  IbVjpArgs v{G, lam_x, lam_xn, gx, gxn, gF, gFn, GU, lam_w, ftot, ftot_n, wrep, wrep_n,
              ctx->p.wall_mode == ZF_WALL_REF_EQ};
  k_ib_vjp<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(ctx->ib, c, v);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

// ---- repulsions --------------------------------------------------------------------

namespace {

__device__ __forceinline__ float wrapd_(float d, float L) {
  if (L > 0.f) {
    if (d > 0.5f * L) d -= L;
    else if (d < -0.5f * L) d += L;
  }
  return d;
}
__device__ __forceinline__ float d3_(float dx, float dy, float dz) {
  return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}
__device__ __forceinline__ float rec_rb_(float w) { return (float)(__float_as_uint(w) >> 8) * (1.f / 1048576.f); }
__device__ __forceinline__ void npos(const IbArgs& a, const double* X, int nc, int n, int cell, int node, float& xp,
                                     float& yp, float& zp) {
  xp = (float)X[((size_t)0 * nc + cell) * n + node];
  yp = (float)X[((size_t)1 * nc + cell) * n + node];
  double z = X[((size_t)2 * nc + cell) * n + node];
  if (a.LZ > 0.f) z -= (double)a.LZ * floor((z - a.Z0) / (double)a.LZ);
  zp = (float)z;
}

// barycentric weights of the 15 points of the subdivided triangle (1-based,
// ZebraflowWT.c:9981-10027, as k_rbc_rbc's rbc_entry forms them)
__device__ __forceinline__ void sub_points(float (&b)[16][3]) {
  for (int k = 0; k < 16; ++k) b[k][0] = b[k][1] = b[k][2] = 0.f;
  b[1][0] = b[2][1] = b[3][2] = 1.f;
  const int pa[12] = {1, 2, 1, 1, 2, 2, 5, 3, 6, 4, 4, 5}, pb[12] = {2, 3, 3, 4, 4, 5, 3, 6, 1, 6, 5, 6};
  for (int k = 0; k < 12; ++k)
    for (int q = 0; q < 3; ++q) b[4 + k][q] = 0.5f * (b[pa[k]][q] + b[pb[k]][q]);
}

}  // namespace

// RBC-RBC repulsion (ZebraflowWT.c:9919-10053; k_rbc_rbc's search, one thread
// per membrane node): wrep += f(r) = -K (1 - d)/d r, r = c_sub - x, d = |r| < 1,
// over the facing triangles near the node.  With J = df/dr = -K ((1-d)/d I -
// r r^T / d^3) (symmetric): gx(node) -= J lam, gx(vertex i) += alpha_i J lam,
// alpha the sub-centroid's barycentric weights.
__global__ void k_rbc_vjp(IbArgs a, CellArgs c, const float* __restrict__ lam_w, float* gx) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  if (gid >= (int64_t)nc * c.nn) return;
  const int cell = (int)(gid / c.nn), node = (int)(gid % c.nn);
  if (c.status[cell] <= 0) return;
  auto at = [&](int q, int m, int i) { return ((size_t)q * nc + m) * c.nn + i; };
  const float lx = lam_w[at(0, cell, node)], ly = lam_w[at(1, cell, node)], lz = lam_w[at(2, cell, node)];
  if (lx == 0.f && ly == 0.f && lz == 0.f) return;
  float xc, yc, zc;
  npos(a, c.x, nc, c.nn, cell, node, xc, yc, zc);
  const float e1x = c.node_normal[at(0, cell, node)], e1y = c.node_normal[at(1, cell, node)],
              e1z = c.node_normal[at(2, cell, node)];
  const int i0 = (int)floor(((double)xc - a.X0) / a.DX + 1.01) - 1;
  const int j0 = (int)floor(((double)yc - a.Y0) / a.DX + 1.01) - 1;
  const int k0 = (int)floor(((double)zc - a.Z0) / a.DX + 1.01) - 1;
  const int i1 = max(i0 - 4, 0), i2 = min(i0 + 4, a.nx - 1), j1 = max(j0 - 4, 0), j2 = min(j0 + 4, a.ny - 1);
  const int k1 = a.per_z ? k0 - 4 : max(k0 - 4, 2), k2 = a.per_z ? k0 + 4 : min(k0 + 4, a.nz - 4);
  if (i1 > i2 || j1 > j2 || k1 > k2) return;
  float bw[16][3];
  sub_points(bw);
  constexpr int kA[16] = {1, 7, 7, 4, 4, 8, 8, 12, 13, 13, 14, 14, 6, 15, 15, 11};
  constexpr int kB[16] = {7, 13, 4, 14, 8, 9, 2, 13, 15, 14, 5, 9, 15, 10, 5, 10};
  constexpr int kC[16] = {12, 12, 13, 13, 14, 14, 9, 6, 6, 15, 15, 5, 11, 11, 10, 3};
  const int64_t stride = (int64_t)nc * c.nt, n_pop_tiles = a.ns / ZF_TC;
  const float K = 8.333e-07f;
  float gn[3] = {0.f, 0.f, 0.f};
  for (int ci = i1; ci <= i2; ++ci)
    for (int cj = j1; cj <= j2; ++cj)
      for (int ck = k1; ck <= k2; ++ck) {
        const int kw = a.per_z ? ((ck % a.nz) + a.nz) % a.nz : ck;
        const int t = a.tile_map[((kw >> 2) * a.nty + (cj >> 2)) * a.ntx + (ci >> 2)];
        if (t < 0 || t >= n_pop_tiles) continue;
        const int64_t key = (int64_t)t * ZF_TC + 16 * (ci & 3) + 4 * (cj & 3) + (kw & 3);
        for (int e = a.bin_off[key]; e < a.bin_off[key + 1]; ++e) {
          const float4 cr = a.bin_rec[2 * e];
          const float dzc = wrapd_(cr.z - zc, a.LZ);
          const float dcen = d3_(xc - cr.x, yc - cr.y, -dzc);
          if (!(dcen < 2.f) || dcen - rec_rb_(cr.w) > 1.f) continue;
          const float4 nr = a.bin_rec[2 * e + 1];
          if (!(e1x * nr.x + e1y * nr.y + e1z * nr.z < 0.f)) continue;
          const int g = __float_as_int(nr.w);
          const int m = g / c.nt, tri = g - m * c.nt;
          if (m == cell && (c.tri[3 * tri] == node || c.tri[3 * tri + 1] == node || c.tri[3 * tri + 2] == node))
            continue;
          const float4 v1 = a.bin_v[e], v2 = a.bin_v[stride + e], v3 = a.bin_v[2 * stride + e];
          const float shift = (cr.z - zc) - dzc;
          const float P[3][3] = {{v1.x, v1.y, v1.z - shift}, {v2.x, v2.y, v2.z - shift}, {v3.x, v3.y, v3.z - shift}};
          const int vid[3] = {__float_as_int(v1.w), __float_as_int(v2.w), __float_as_int(v3.w)};
          float gv[3][3] = {};
          for (int v = 0; v < 16; ++v) {
            float al[3], r[3];
            for (int q = 0; q < 3; ++q) al[q] = (bw[kA[v]][q] + bw[kB[v]][q] + bw[kC[v]][q]) * (1.f / 3.f);
            for (int q = 0; q < 3; ++q) r[q] = al[0] * P[0][q] + al[1] * P[1][q] + al[2] * P[2][q];
            r[0] -= xc;
            r[1] -= yc;
            r[2] -= zc;
            const float d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (!(d2 < 1.f)) continue;
            const float d = sqrtf(d2);
            if (!(d < 1.f) || !(d > 0.f)) continue;
            const float aI = -K * (1.f - d) / d, bR = K / (d2 * d);
            const float rl = r[0] * lx + r[1] * ly + r[2] * lz;
            const float Jl[3] = {aI * lx + bR * r[0] * rl, aI * ly + bR * r[1] * rl, aI * lz + bR * r[2] * rl};
            for (int q = 0; q < 3; ++q) {
              gn[q] -= Jl[q];
              for (int i = 0; i < 3; ++i) gv[i][q] += al[i] * Jl[q];
            }
          }
          for (int i = 0; i < 3; ++i)
            for (int q = 0; q < 3; ++q)
              if (gv[i][q] != 0.f) atomicAdd(&gx[at(q, m, vid[i])], gv[i][q]);
        }
      }
  for (int q = 0; q < 3; ++q)
    if (gn[q] != 0.f) atomicAdd(&gx[at(q, cell, node)], gn[q]);
}

// wall repulsion (ZebraflowWT.c:9055-9077): wrep += (0.25 - dist) 1e-4 n for
// -0.75 <= dist < 0.25, dist = (x - w1) . n the signed distance to the plane of
// the node's wall triangle (constant 1e-4 n below -0.75): gx -= 1e-4 (n . lam) n.
// Nucleus nodes add to the membrane node of their own index (as the forward).
__global__ void k_wall_vjp(IbArgs a, CellArgs c, const float* __restrict__ lam_w, float* gx, float* gxn) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  const int64_t nmem = (int64_t)nc * c.nn;
  const bool nuc = gid >= nmem;
  if (gid >= nmem + (int64_t)nc * c.nnn) return;
  const int n = nuc ? c.nnn : c.nn;
  const int64_t lid = nuc ? gid - nmem : gid;
  const int cell = (int)(lid / n), node = (int)(lid % n);
  if (c.status[cell] <= 0 || node >= c.nn) return;
  const int tw = a.wall_tri[gid];
  if (tw < 0) return;
  float xp, yp, zp;
  npos(a, nuc ? c.xn : c.x, nc, n, cell, node, xp, yp, zp);
  const int w1 = a.wtri[3 * tw];
  const float n0 = a.wnrm[tw], n1 = a.wnrm[a.mt + tw], n2 = a.wnrm[2 * a.mt + tw];
  const float ddx = xp - a.wxyz[w1], ddy = yp - a.wxyz[a.nw + w1], ddz = wrapd_(zp - a.wxyz[2 * a.nw + w1], a.LZ);
  const float dist = __fadd_rn(__fadd_rn(__fmul_rn(ddx, n0), __fmul_rn(ddy, n1)), __fmul_rn(ddz, n2));
  if (!(dist < 0.25f && fabsf(dist) < 1.0f) || dist < -0.75f) return;
  const size_t m = (size_t)cell * c.nn + node;
  const float nl = n0 * lam_w[m] + n1 * lam_w[nmem + m] + n2 * lam_w[2 * nmem + m];
  float* G = nuc ? gxn : gx;
  const int64_t stride = nuc ? (int64_t)nc * c.nnn : nmem;
  G[lid] -= 1.e-4f * nl * n0;
  G[stride + lid] -= 1.e-4f * nl * n1;
  G[2 * stride + lid] -= 1.e-4f * nl * n2;
}

// nucleus-membrane repulsion (ZebraflowWT.c:9516-9730; k_nuc_memb, one thread
// per nucleus node, over its current list): for each listed triangle within
// 1 um and each of its 19 sample points tp within d <= 0.2 of the nucleus node
// xc, the triangle's three nodes get wrep += repulf n / 3, repulf = (0.2 - d)/0.2
// 4.1666667e-7, n the triangle's unit normal.  Differentiated in 12-tangent
// duals (the three vertices, xc).
__global__ void k_nuc_vjp(IbArgs a, CellArgs c, const float* __restrict__ lam_w, float* gx, float* gxn) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = c.n_cells;
  if (gid >= (int64_t)nc * c.nnn) return;
  const int cell = (int)(gid / c.nnn), node = (int)(gid % c.nnn);
  if (c.status[cell] <= 0) return;
  using D = Dl<12>;
  using V = V3d<12>;
  auto atm = [&](int q, int i) { return ((size_t)q * nc + cell) * c.nn + i; };
  auto atn = [&](int q) { return ((size_t)q * nc + cell) * c.nnn + node; };
  const float xcf = (float)c.xn[atn(0)], ycf = (float)c.xn[atn(1)], zcf = (float)c.xn[atn(2)];
  const V xc = {var<12>(xcf, 9), var<12>(ycf, 10), var<12>(zcf, 11)};
  const uint16_t* list = a.nuc_list + (size_t)gid * a.nuc_cap;
  const int cnt = a.nuc_cnt[gid];
  float gnode[3] = {0.f, 0.f, 0.f};
  for (int l = 0; l < cnt; ++l) {
    const int tri = list[l];
    const int nd[3] = {c.tri[3 * tri], c.tri[3 * tri + 1], c.tri[3 * tri + 2]};
    float L[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < 3; ++k)
      for (int q = 0; q < 3; ++q) L[q] += lam_w[atm(q, nd[k])];
    if (L[0] == 0.f && L[1] == 0.f && L[2] == 0.f) continue;
    V p[3];
    for (int k = 0; k < 3; ++k)
      p[k] = {var<12>((float)c.x[atm(0, nd[k])], 3 * k), var<12>((float)c.x[atm(1, nd[k])], 3 * k + 1),
              var<12>((float)c.x[atm(2, nd[k])], 3 * k + 2)};
    D ar;
    V nrm, cen;
    tri_geom(p[0], p[1], p[2], ar, nrm, cen);
    if (!(d3_(xcf - cen.x.v, ycf - cen.y.v, zcf - cen.z.v) < 1.f)) continue;
    // 19 sample points as k_nuc_memb forms them: vertices' midpoints ep, then tp
    V ep[10], tp[20];
    ep[1] = vmul(0.5f, vadd(p[0], p[1]));
    ep[2] = vmul(0.5f, vadd(p[1], p[2]));
    ep[3] = vmul(0.5f, vadd(p[2], p[0]));
    ep[4] = vmul(0.5f, vadd(p[0], ep[1]));
    ep[5] = vmul(0.5f, vadd(ep[1], p[1]));
    ep[6] = vmul(0.5f, vadd(p[1], ep[2]));
    ep[7] = vmul(0.5f, vadd(ep[2], p[2]));
    ep[8] = vmul(0.5f, vadd(p[2], ep[3]));
    ep[9] = vmul(0.5f, vadd(ep[3], p[0]));
    const float third = 1.f / 3.f;
    tp[1] = vmul(third, vadd(vadd(p[0], p[1]), p[2]));
    tp[2] = vmul(third, vadd(vadd(ep[3], p[0]), ep[1]));
    tp[3] = vmul(third, vadd(vadd(ep[1], p[1]), ep[2]));
    tp[4] = vmul(third, vadd(vadd(ep[2], p[2]), ep[3]));
    tp[5] = vmul(0.5f, vadd(ep[1], ep[3]));
    tp[6] = vmul(0.5f, vadd(ep[1], ep[2]));
    tp[7] = vmul(0.5f, vadd(ep[2], ep[3]));
    tp[8] = vmul(0.5f, vadd(p[0], tp[2]));
    tp[9] = vmul(0.5f, vadd(ep[1], tp[2]));
    tp[10] = vmul(0.5f, vadd(ep[3], tp[2]));
    tp[11] = vmul(0.5f, vadd(ep[1], tp[3]));
    tp[12] = vmul(0.5f, vadd(p[1], tp[3]));
    tp[13] = vmul(0.5f, vadd(ep[2], tp[3]));
    tp[14] = vmul(0.5f, vadd(ep[3], tp[4]));
    tp[15] = vmul(0.5f, vadd(ep[2], tp[4]));
    tp[16] = vmul(0.5f, vadd(p[2], tp[4]));
    tp[17] = vmul(0.5f, vadd(ep[1], tp[1]));
    tp[18] = vmul(0.5f, vadd(ep[2], tp[1]));
    tp[19] = vmul(0.5f, vadd(ep[3], tp[1]));
    float acc[12];
    for (int k = 0; k < 12; ++k) acc[k] = 0.f;
    for (int v = 1; v <= 19; ++v) {
      const V r = vsub(tp[v], xc);
      const D d = dsqrt(vdot(r, r));
      if (!(d.v <= 0.2f)) continue;
      const D rf = (4.1666667e-07f / 0.2f) * (cst<12>(0.2f) - d);
      vjp_acc(acc, vmul(third, vmul(rf, nrm)), L[0], L[1], L[2]);
    }
    for (int k = 0; k < 3; ++k)
      for (int q = 0; q < 3; ++q)
        if (acc[3 * k + q] != 0.f) atomicAdd(&gx[atm(q, nd[k])], acc[3 * k + q]);
    for (int q = 0; q < 3; ++q) gnode[q] += acc[9 + q];
  }
  for (int q = 0; q < 3; ++q)
    if (gnode[q] != 0.f) atomicAdd(&gxn[atn(q)], gnode[q]);
}

int repulsion_vjp_launch(zf_ctx* ctx, const float* lam_w, float* gx, float* gxn) {
  const CellArgs& c = ctx->cells;
  const int64_t nm = (int64_t)c.n_cells * c.nn, nn_ = (int64_t)c.n_cells * c.nnn;
  if (nm == 0) return ZF_OK;
  k_rbc_vjp<<<(unsigned)((nm + 127) / 128), 128, 0, ctx->stream>>>(ctx->ib, c, lam_w, gx);
  if (ctx->ib.nw > 0 && ctx->ib.wall_tri)
    k_wall_vjp<<<(unsigned)((nm + nn_ + 127) / 128), 128, 0, ctx->stream>>>(ctx->ib, c, lam_w, gx, gxn);
  if (nn_ > 0) k_nuc_vjp<<<(unsigned)((nn_ + 127) / 128), 128, 0, ctx->stream>>>(ctx->ib, c, lam_w, gx, gxn);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 3;
  return ZF_OK;
}

__global__ void k_add(float* __restrict__ y, const float* __restrict__ x, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

int add_launch(zf_ctx* ctx, float* y, const float* x, int64_t n) {
  if (n <= 0) return ZF_OK;
  k_add<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(y, x, n);
  ZF_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return ZF_OK;
}

}  // namespace zf

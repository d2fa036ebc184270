// Membrane and nucleus mechanics of every cell, one CTA per cell.
//
// k_membrane fuses the reference's per-cell OpenMP passes of one membrane
// step into one kernel whose working set stays in shared memory:
//   CGSM_NODAL_FORCE_ZERO                         ZebraflowWT.c:5704-5745
//   CGSM_AREA: triangle centroid/area/normal, node area and normal,
//              sliver repulsion                   ZebraflowWT.c:5749-6096 (no cell-list insert)
//   cell centroid, area, global-area force        ZebraflowWT.c:6717-6796
//   CGSM_LOCAL_FORCES: WLC+POW springs, bending, local and global area,
//              volume gradient, force screening  ZebraflowWT.c:6800-7386
//   nucleus springs                               ZebraflowWT.c:7388-7471
//   bad-cell removal                              ZebraflowWT.c:7473-7501
//   CGSM_VOLUME_CALC                              ZebraflowWT.c:7510-7535
// Arithmetic is fp32 on fp32 copies of the fp64 positions, as the reference's
// float locals; per-cell sums (area, centroid, volume) are reduced in fp64.
// Scatters into node accumulators use shared-memory atomics; the reference
// accumulates serially, so sums agree to rounding.
#include "zf_internal.h"

namespace zf {

namespace {

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 mul(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// reference screening of a force term: NaN, inf or a component above 1e-10 N
__device__ __forceinline__ int bad_components(V3 f) {
  auto b = [](float v) { return (isnan(v) || isinf(v) || fabsf(v) > 1.e-10f) ? 1 : 0; };
  return b(f.x) + b(f.y) + b(f.z);
}

struct Smem {
  float *xs, *fT, *fV, *nA, *nN, *tA, *tN, *tC, *fTn;
  double* red;
  int* cnt;
};

__device__ __forceinline__ V3 ld3(const float* p, int n, int i) { return {p[i], p[n + i], p[2 * n + i]}; }
__device__ __forceinline__ void atom3(float* p, int n, int i, V3 v) {
  atomicAdd(&p[i], v.x);
  atomicAdd(&p[n + i], v.y);
  atomicAdd(&p[2 * n + i], v.z);
}

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < nw; ++i) t += red[i];  // fixed order: deterministic
  return t;
}

}  // namespace

// three blocks per SM (80 registers; the shared memory of a 642-node cell,
// about 71 KB, also allows three)
__global__ void __launch_bounds__(256, 3) k_membrane(CellArgs a) {
  const int cell = blockIdx.x;
  if (a.status[cell] <= -5000) return;
  const int nn = a.nn, nt = a.nt, ne = a.ne, nnn = a.nnn, nen = a.nen, nc = a.n_cells;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem s;
  {
    double* d = reinterpret_cast<double*>(smem_raw);
    s.red = d;
    float* f = reinterpret_cast<float*>(d + 32);
    s.xs = f; f += 3 * nn;
    s.fT = f; f += 3 * nn;
    s.fV = f; f += 3 * nn;
    s.nA = f; f += nn;
    s.nN = f; f += 3 * nn;
    s.tA = f; f += nt;
    s.tN = f; f += 3 * nt;
    s.tC = f; f += 3 * nt;
    s.fTn = f; f += 3 * nnn;
    s.cnt = reinterpret_cast<int*>(f);
  }
  const int tid = threadIdx.x, nth = blockDim.x;

  // zero accumulators (ZebraflowWT.c:5713-5738) and load positions as float
  for (int i = tid; i < nn; i += nth) {
    for (int c = 0; c < 3; ++c) {
      const size_t g = ((size_t)c * nc + cell) * nn + i;
      s.xs[c * nn + i] = (float)a.x[g];
      s.fT[c * nn + i] = 0.f;
      s.fV[c * nn + i] = 0.f;
      s.nN[c * nn + i] = 0.f;
      a.wrep[g] = 0.f;
      a.vel[g] = 0.0;
    }
    s.nA[i] = 0.f;
  }
  for (int i = tid; i < nnn; i += nth) {
    for (int c = 0; c < 3; ++c) {
      const size_t g = ((size_t)c * nc + cell) * nnn + i;
      s.fTn[c * nnn + i] = 0.f;
      a.wrep_n[g] = 0.f;
      a.vel_n[g] = 0.0;
    }
  }
  if (tid < 2) s.cnt[tid] = 0;
  __syncthreads();

  // CGSM_AREA: per triangle centroid, area, normal, node area/normal, sliver push
  double asum = 0.0;
  for (int t = tid; t < nt; t += nth) {
    const int n1 = a.tri[3 * t], n2 = a.tri[3 * t + 1], n3 = a.tri[3 * t + 2];
    const V3 p1 = ld3(s.xs, nn, n1), p2 = ld3(s.xs, nn, n2), p3 = ld3(s.xs, nn, n3);
    const V3 c = {(p1.x + p2.x + p3.x) / 3.f, (p1.y + p2.y + p3.y) / 3.f, (p1.z + p2.z + p3.z) / 3.f};
    const V3 e1 = sub(p2, p1), e3 = sub(p1, p3);
    const V3 A = mul(0.5e-12f, cross(e1, e3));
    const float ar = sqrtf(dot(A, A));
    const V3 nrm = mul(-1.f / ar, A);
    s.tA[t] = ar;
    s.tN[t] = nrm.x; s.tN[nt + t] = nrm.y; s.tN[2 * nt + t] = nrm.z;
    s.tC[t] = c.x; s.tC[nt + t] = c.y; s.tC[2 * nt + t] = c.z;
    asum += (double)ar;
    const float a3 = ar / 3.f;
    const int nd[3] = {n1, n2, n3};
    for (int v = 0; v < 3; ++v) {
      atomicAdd(&s.nA[nd[v]], a3);
      atom3(s.nN, nn, nd[v], mul(a3, nrm));
    }
    // sliver repulsion, ZebraflowWT.c:6042-6084
    const V3 pv[3] = {p1, p2, p3};
    for (int v = 0; v < 3; ++v) {
      const V3 e = sub(pv[v], c);
      const float l = sqrtf(dot(e, e));
      if (l < 0.05f) {
        const V3 u = mul(1.f / l, e);
        atom3(s.fT, nn, nd[v], mul(l > 0.001f ? 1.e-14f / l : 1.e-11f, u));
      }
    }
  }
  const double cell_area = block_sum(asum, s.red);
  __syncthreads();

  // node normals (ZebraflowWT.c:6088-6092) and the cell centroid (:6747-6750)
  double cx = 0.0, cy = 0.0, cz = 0.0;
  for (int i = tid; i < nn; i += nth) {
    const float inv = 1.f / s.nA[i];
    for (int c = 0; c < 3; ++c)
      a.node_normal[((size_t)c * nc + cell) * nn + i] = s.nN[c * nn + i] * inv;
    cx += (double)(s.xs[i] / (float)nn);
    cy += (double)(s.xs[nn + i] / (float)nn);
    cz += (double)(s.xs[2 * nn + i] / (float)nn);
  }
  const V3 C = {(float)block_sum(cx, s.red), (float)block_sum(cy, s.red), (float)block_sum(cz, s.red)};
  // global-area force, ZebraflowWT.c:6791
  const float FAG = -a.ka * ((float)cell_area - a.area0) / a.area0;

  // CGSM_LOCAL_FORCES, one thread per edge
  const float* LMAX = a.epar;
  const float* PLEN = a.epar + ne;
  const float* KP = a.epar + 2 * ne;
  const float* SIN0 = a.epar + 3 * ne;
  const float* COS0 = a.epar + 4 * ne;
  for (int e = tid; e < ne; e += nth) {
    const int* E = a.edge + 6 * e;
    const int n1 = E[0], n2 = E[1], n3 = E[2], n4 = E[3], t1 = E[4], t2 = E[5];
    const V3 c1 = ld3(s.xs, nn, n1), c2 = ld3(s.xs, nn, n2), c3 = ld3(s.xs, nn, n3),
             c4 = ld3(s.xs, nn, n4);
    // WLC + POW, ZebraflowWT.c:6880-6924
    const V3 d12 = sub(c1, c2);
    float len = sqrtf(dot(d12, d12));
    const V3 e1v = mul(1.f / len, d12);
    const V3 e2v = mul(-1.f / len, d12);
    float er = len * 1.e-06f / LMAX[e];
    if (er > 0.95f) er = 0.95f;
    if (er < 0.02435f) len = 0.02435f * LMAX[e] / 1.e-06f;
    const float wlc = -a.kT / PLEN[e] * (er - 0.25f + 1.f / (4.f * (1.f - er) * (1.f - er)));
    const float comp = KP[e] * (1.f / (len * len * 1.e-012f));
    V3 f1 = add(mul(wlc, e1v), mul(comp, e1v));
    V3 f2 = add(mul(wlc, e2v), mul(comp, e2v));
    V3 f3 = {0.f, 0.f, 0.f}, f4 = {0.f, 0.f, 0.f};

    // geometry of the rhombus, ZebraflowWT.c:6930-6978
    float A1 = s.tA[t1], A2 = s.tA[t2];
    const float A1eq = a.tri_area_eq[t1], A2eq = a.tri_area_eq[t2];
    if (A1 < 0.1f * A1eq) A1 = 0.1f * A1eq;
    else if (A1 > 10.f * A1eq) A1 = 10.f * A1eq;
    if (A2 < 0.1f * A2eq) A2 = 0.1f * A2eq;
    else if (A2 > 10.f * A2eq) A2 = 10.f * A2eq;
    const V3 N1 = ld3(s.tN, nt, t1), N2 = ld3(s.tN, nt, t2);
    const V3 C1 = ld3(s.tC, nt, t1), C2 = ld3(s.tC, nt, t2);
    const V3 adiff = sub(N1, N2), cdiff = mul(1.e-006f, sub(C1, C2));
    float cs = dot(N1, N2);
    if (cs > 1.f) cs = 1.f;
    else if (cs < -1.f) cs = -1.f;
    const float ac = dot(adiff, cdiff);
    const float sn = ac >= 0.f ? sqrtf(1.f - cs * cs) : -sqrtf(1.f - cs * cs);

    // bending, ZebraflowWT.c:6988-7081
    const float beta = fabsf(cs) > 0.99f ? 0.f : a.kbend * (sn * COS0[e] - cs * SIN0[e]) / sn;
    const V3 dp21 = mul(1.e-6f, sub(c2, c1)), dp24 = mul(1.e-6f, sub(c2, c4)),
             dp32 = mul(1.e-6f, sub(c3, c2)), dp41 = mul(1.e-6f, sub(c4, c1)),
             dp13 = mul(1.e-6f, sub(c1, c3));
    const V3 cp1 = mul(A1, cross(N1, dp21)), cp2 = mul(A2, cross(N2, dp21));
    const V3 cp3 = mul(A1, cross(N1, dp24)), cp4 = mul(A2, cross(N2, dp24));
    const V3 cp5 = mul(A1, cross(N1, dp32)), cp6 = mul(A2, cross(N2, dp32));
    const V3 cp7 = mul(A1, cross(N1, dp41)), cp8 = mul(A2, cross(N2, dp41));
    const V3 cp9 = mul(A1, cross(N1, dp13)), cp10 = mul(A2, cross(N2, dp13));
    const V3 lc1 = mul(1.e-006f, sub(C1, C)), lc2 = mul(1.e-006f, sub(C2, C));
    const float b11 = -beta * cs / (A1 * A1);
    const float b12 = beta / (A1 * A2);
    const float b22 = -beta * cs / (A2 * A2);
    const V3 fb1 = add(add(mul(b11, cp5), mul(b12, add(cp3, cp6))), mul(b22, cp4));
    const V3 fb2 = add(add(mul(b11, cp9), mul(b12, add(cp7, cp10))), mul(b22, cp8));
    const V3 fb3 = add(mul(b11, cp1), mul(b12, cp2));
    const V3 fb4 = add(mul(-b12, cp1), mul(-b22, cp2));
    int removes = 0, screened = 0;
    {
      const int k1 = bad_components(fb1), k2 = bad_components(fb2), k3 = bad_components(fb3),
                k4 = bad_components(fb4);
      removes += k1 + k2 + k3 + k4;
      if (!k1) f1 = add(f1, fb1);
      if (!k2) f2 = add(f2, fb2);
      if (!k3) f3 = add(f3, fb3);
      if (!k4) f4 = add(f4, fb4);
    }
    // local area, global area and volume terms by each triangle's first
    // visiting edge (AREA_UPDATE), ZebraflowWT.c:7126-7359
    if (a.area_first[e] & 1) {
      const float al = -a.kd * (A1 - A1eq) / (4.f * A1eq * A1);
      const float ag = 0.25f * FAG / A1;
      const V3 fa[3] = {mul(al, cp5), mul(al, cp9), mul(al, cp1)};
      const V3 fg[3] = {mul(ag, cp5), mul(ag, cp9), mul(ag, cp1)};
      const V3 base = mul(1.f / 3.f, mul(A1, N1));
      const V3 fv[3] = {mul(1.f / 6.f, add(base, cross(lc1, dp32))),
                        mul(1.f / 6.f, add(base, cross(lc1, dp13))),
                        mul(1.f / 6.f, add(base, cross(lc1, dp21)))};
      V3* tgt[3] = {&f1, &f2, &f3};
      const int nd[3] = {n1, n2, n3};
      for (int k = 0; k < 3; ++k) {
        const int ba = bad_components(fa[k]);
        removes += ba;
        if (!ba) *tgt[k] = add(*tgt[k], fa[k]);
      }
      for (int k = 0; k < 3; ++k) {
        const int bg = bad_components(fg[k]);
        removes += bg;
        if (!bg) *tgt[k] = add(*tgt[k], fg[k]);
      }
      for (int k = 0; k < 3; ++k) {
        const int bv = bad_components(fv[k]);
        removes += bv;
        if (!bv) atom3(s.fV, nn, nd[k], fv[k]);
      }
    }
    if (a.area_first[e] & 2) {  // tri2 = (n2, n1, n4); screened terms do not count for removal
      const float al = -a.kd * (A2 - A2eq) / (4.f * A2eq * A2);
      const float ag = 0.25f * FAG / A2;
      const V3 m2 = mul(-1.f, cp2);
      const V3 fa[3] = {mul(al, cp4), mul(al, cp8), mul(al, m2)};
      const V3 fg[3] = {mul(ag, cp4), mul(ag, cp8), mul(ag, m2)};
      const V3 base = mul(1.f / 3.f, mul(A2, N2));
      const V3 c12v = mul(-1.f, cross(lc2, dp21));
      const V3 fv[3] = {mul(1.f / 6.f, add(base, cross(lc2, dp24))),
                        mul(1.f / 6.f, add(base, cross(lc2, dp41))),
                        mul(1.f / 6.f, add(base, c12v))};
      V3* tgt[3] = {&f1, &f2, &f4};
      const int nd[3] = {n1, n2, n4};
      for (int k = 0; k < 3; ++k) {
        const int ba = bad_components(fa[k]);
        screened += ba;
        if (!ba) *tgt[k] = add(*tgt[k], fa[k]);
      }
      for (int k = 0; k < 3; ++k) {
        const int bg = bad_components(fg[k]);
        screened += bg;
        if (!bg) *tgt[k] = add(*tgt[k], fg[k]);
      }
      for (int k = 0; k < 3; ++k) {
        const int bv = bad_components(fv[k]);
        screened += bv;
        if (!bv) atom3(s.fV, nn, nd[k], fv[k]);
      }
    }
    atom3(s.fT, nn, n1, f1);
    atom3(s.fT, nn, n2, f2);
    atom3(s.fT, nn, n3, f3);
    atom3(s.fT, nn, n4, f4);
    if (removes) atomicAdd(&s.cnt[0], removes);
    if (removes + screened) atomicAdd(&s.cnt[1], removes + screened);
  }

  // nucleus springs, ZebraflowWT.c:7388-7471
  for (int e = tid; e < nen; e += nth) {
    const int n1 = a.edge_n[2 * e], n2 = a.edge_n[2 * e + 1];
    V3 c1, c2;
    c1.x = (float)a.xn[((size_t)0 * nc + cell) * nnn + n1];
    c1.y = (float)a.xn[((size_t)1 * nc + cell) * nnn + n1];
    c1.z = (float)a.xn[((size_t)2 * nc + cell) * nnn + n1];
    c2.x = (float)a.xn[((size_t)0 * nc + cell) * nnn + n2];
    c2.y = (float)a.xn[((size_t)1 * nc + cell) * nnn + n2];
    c2.z = (float)a.xn[((size_t)2 * nc + cell) * nnn + n2];
    const V3 d12 = sub(c1, c2);
    float len = sqrtf(dot(d12, d12));
    const V3 e1v = mul(1.f / len, d12), e2v = mul(-1.f / len, d12);
    const float LM = a.epar_n[e], PL = a.epar_n[nen + e], KPn = a.epar_n[2 * nen + e];
    float er = len * 1.e-06f / LM;
    if (er > 0.95f) er = 0.95f;
    if (er < 0.02435f) len = 0.02435f * LM / 1.e-06f;
    const float wlc = -a.kT / PL * (er - 0.25f + 1.f / (4.f * (1.f - er) * (1.f - er)));
    const float comp = KPn * (1.f / (len * len * 1.e-012f));
    atom3(s.fTn, nnn, n1, add(mul(wlc, e1v), mul(comp, e1v)));
    atom3(s.fTn, nnn, n2, add(mul(wlc, e2v), mul(comp, e2v)));
  }
  __syncthreads();

  // bad-cell removal, ZebraflowWT.c:7473-7501
  const bool remove = s.cnt[0] > a.remove_count;

  // CGSM_VOLUME_CALC, ZebraflowWT.c:7513-7535
  double vsum = 0.0;
  for (int t = tid; t < nt; t += nth)
    vsum += (double)(s.tA[t] * (s.tC[t] * s.tN[t] + s.tC[nt + t] * s.tN[nt + t] +
                                s.tC[2 * nt + t] * s.tN[2 * nt + t]) * 1.e-006f);
  const float vol = (float)(block_sum(vsum, s.red) / 3.0);
  const float FVS = -a.kv * (vol - a.volume0) / a.volume0;

  for (int i = tid; i < nn; i += nth)
    for (int c = 0; c < 3; ++c) {
      const size_t g = ((size_t)c * nc + cell) * nn + i;
      a.ftot[g] = remove ? 0.f : s.fT[c * nn + i] + FVS * s.fV[c * nn + i];
      if (remove) a.x[g] = -5000.0;
    }
  for (int i = tid; i < nnn; i += nth)
    for (int c = 0; c < 3; ++c) {
      const size_t g = ((size_t)c * nc + cell) * nnn + i;
      a.ftot_n[g] = remove ? 0.f : s.fTn[c * nnn + i];
      if (remove) a.xn[g] = -5000.0;
    }
  for (int t = tid; t < nt; t += nth) {
    a.tri_a[(size_t)cell * nt + t] = s.tA[t];
    for (int c = 0; c < 3; ++c) {
      a.tri_nrm[((size_t)c * nc + cell) * nt + t] = s.tN[c * nt + t];
      a.tri_c[((size_t)c * nc + cell) * nt + t] = s.tC[c * nt + t];
    }
  }
  if (tid == 0) {
    float* cf = a.cell_f + 8 * cell;
    cf[0] = (float)cell_area;
    cf[1] = vol;
    cf[2] = C.x;
    cf[3] = C.y;
    cf[4] = C.z;
    cf[5] = FAG;
    cf[6] = FVS;
    a.caps_remove[cell] = s.cnt[0];
    if (s.cnt[1]) atomicAdd(&a.counters[0], (unsigned long long)s.cnt[1]);
    if (remove) {
      a.status[cell] = -5000;
      atomicAdd(&a.counters[1], 1ull);
    }
  }
}

size_t membrane_smem_bytes(const CellArgs& a) {
  return 32 * sizeof(double) +
         sizeof(float) * (3 * a.nn * 4 + a.nn + a.nt * 7 + 3 * a.nnn) + 2 * sizeof(int);
}

int cells_membrane_launch(zf_ctx* c) {
  const CellArgs& a = c->cells;
  if (a.n_cells == 0) return ZF_OK;
  int rc0 = cells_write_fence(c);  // k_membrane may remove cells (status)
  if (rc0) return rc0;
  const size_t smem = membrane_smem_bytes(a);
  ZF_CUDA(cudaFuncSetAttribute(k_membrane, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_membrane<<<a.n_cells, 256, smem, c->stream>>>(a);
  ZF_CUDA(cudaGetLastError());
  c->launches += 1;
  return ZF_OK;
}

}  // namespace zf

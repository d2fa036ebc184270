// D3Q19 LBM kernels for sm_100a over the sparse 4x4x4-tile lattice.
//
// k_lbm fuses what the reference does in three OpenMP passes per step:
//   pull stream + moments + BGK/Guo collision   ZebraflowWT.c:6100-6145
//   wall equilibrium (reference wall mode)       ZebraflowWT.c:6290-6315, :6429-6432
//   moments + F_OLD copy + BODYFORCE reset       ZebraflowWT.c:6599-6626
// The copy pass disappears (ping-pong buffers), the write-only FEQ array is
// never formed, moments are written only when the caller asks for them, and
// halfway bounce-back replaces the wall pass in the bounce-back mode.
//
// Layout in HBM: populations are SoA planes [19][ns] with ns = tiles*64; a
// tile holds 4x4x4 lattice points, x fastest.  One thread updates one fluid
// point; a 256-thread block covers 4 tiles.  Per point a 32-bit link word
// (bit q: the pull along q bounces back; bit 31: fluid point) replaces any
// neighbour-code lookup; the 27-neighbour tile table of a block's tiles is
// staged in shared memory.
//
// Arithmetic is done on deviations d_q = f_q/w_q - rho_ref in fp32 whatever
// the storage form, so that the small body-force increments are not lost in
// the rounding of O(0.05) populations.  Storage forms: plain fp32 f (as the
// reference), fp32 deviations, and fp16 / bf16 deviations scaled by 2^16,
// written with Blackwell's stochastic-rounding conversion (cvt.rs) from
// hashed random bits, or with round-to-nearest.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <mutex>
#include <type_traits>

#include "zf_internal.h"

namespace zf {

// D3Q19 in the reference order (ZebraflowWT.c:2471-2497), as compile-time
// constants so that zero components and signs fold away after unrolling.
__host__ __device__ constexpr int EX(int q) {
  return (q == 0 || q == 6 || q == 9 || q == 10 || q == 13) ? 1
         : (q == 1 || q == 7 || q == 8 || q == 11 || q == 12) ? -1 : 0;
}
__host__ __device__ constexpr int EY(int q) {
  return (q == 2 || q == 6 || q == 8 || q == 14 || q == 17) ? 1
         : (q == 3 || q == 7 || q == 9 || q == 15 || q == 16) ? -1 : 0;
}
__host__ __device__ constexpr int EZ(int q) {
  return (q == 4 || q == 10 || q == 12 || q == 14 || q == 16) ? 1
         : (q == 5 || q == 11 || q == 13 || q == 15 || q == 17) ? -1 : 0;
}
// weights 1/18, 1/36, 1/3 (ZebraflowWT.c:72-74, :2329-2333)
__host__ __device__ constexpr float WQ(int q) {
  return q < 6 ? 1.f / 18.f : (q < 18 ? 1.f / 36.f : 1.f / 3.f);
}
__host__ __device__ constexpr float IWQ(int q) { return q < 6 ? 18.f : (q < 18 ? 36.f : 3.f); }
__host__ __device__ constexpr int OPP(int q) { return q == 18 ? 18 : (q ^ 1); }

// c_q . (x, y, z) from the nonzero components of c_q only (q is a constant
// after unrolling, so this folds to at most one add; 0*x would not fold)
__device__ __forceinline__ float cdot(int q, float x, float y, float z) {
  const float tx = EX(q) > 0 ? x : -x, ty = EY(q) > 0 ? y : -y, tz = EZ(q) > 0 ? z : -z;
  if (EX(q)) {
    if (EY(q)) return tx + ty;
    if (EZ(q)) return tx + tz;
    return tx;
  }
  if (EY(q)) return EZ(q) ? ty + tz : ty;
  return EZ(q) ? tz : 0.f;
}

// ---- storage codecs: decode to / encode from the deviation d = f/w - rho_ref
// Plain populations, as the reference keeps F.  f = w (rho_ref + d) is
// formed with one rounding, fma(w, d, w rho_ref), and read back as
// (f - w rho_ref) / w: the subtraction is exact (f lies within a factor 2 of
// w rho_ref), so the only error left is the storage rounding itself.  (The
// form f/w - rho_ref would add (w_fp32/w - 1)(rho_ref + d), a fixed offset
// of about 3e-8 per population per step, since 1/18, 1/36, 1/3 have no exact
// fp32 value.)
struct RawF32 {
  using T = float;
  __device__ static float wr(int q, const LbmArgs& a) { return __fmul_rn(WQ(q), a.rho_ref); }
  __device__ static float dec(T v, int q, const LbmArgs& a) { return __fmul_rn(__fsub_rn(v, wr(q, a)), IWQ(q)); }
  __device__ static T enc(float d, int q, const LbmArgs& a) { return __fmaf_rn(WQ(q), d, wr(q, a)); }
};
struct DevF32 {
  using T = float;
  __device__ static float dec(T v, int, const LbmArgs&) { return v; }
  __device__ static T enc(float d, int, const LbmArgs&) { return d; }
};
struct DevF16 {
  using T = __half;
  __device__ static float dec(T v, int, const LbmArgs& a) { return __half2float(v) * a.inv_scale; }
  __device__ static T enc(float d, int, const LbmArgs& a) { return __float2half_rn(d * a.scale); }
  __device__ static T from_bits(unsigned short u) { return __ushort_as_half(u); }
  // values already in storage units (x 2^16): round to nearest, or a pair
  // with stochastic rounding (lo -> low half, hi -> high half)
  __device__ static T cvt_rn(float v) { return __float2half_rn(v); }
  __device__ static void cvt2_sr(uint32_t& r, float lo, float hi, uint32_t rbits) {
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
  }
};
struct DevBF16 {
  using T = __nv_bfloat16;
  __device__ static float dec(T v, int, const LbmArgs& a) { return __bfloat162float(v) * a.inv_scale; }
  __device__ static T enc(float d, int, const LbmArgs& a) { return __float2bfloat16_rn(d * a.scale); }
  __device__ static T from_bits(unsigned short u) { return __ushort_as_bfloat16(u); }
  __device__ static T cvt_rn(float v) { return __float2bfloat16_rn(v); }
  __device__ static void cvt2_sr(uint32_t& r, float lo, float hi, uint32_t rbits) {
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
  }
};
template <class C>
struct IsHalf {
  static constexpr bool v = sizeof(typename C::T) == 2;
};

__device__ __forceinline__ uint32_t mix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x7feb352du;
  h ^= h >> 15;
  h *= 0x846ca68bu;
  h ^= h >> 16;
  return h;
}

constexpr int kTilesPerBlock = 4;

// Pull sources of one point.  A pull along q reads x - e_q; it leaves the
// point's tile only across the faces the point lies on, so a point needs at
// most 7 tiles (its own, three across faces, three across edges: D3Q19 has no
// corner directions).  The offsets below are those tiles' population bases,
// each already shifted by the wrap of the cell coordinate (x - e_x wraps by
// 4 across an x face, y by 16 cells, z by 64), so that the source of q is
// base(crossing pattern) + q*64 - (e_x + 4 e_y + 16 e_z): a selection and a
// constant per direction.  A missing neighbour tile (id -1) maps to tile 0;
// it is only reached by links that bounce back.
template <typename I>
struct PullBases {
  I b0, bx, by, bz, bxy, bxz, byz;
  bool xlo, xhi, ylo, yhi, zlo, zhi;
  __device__ __forceinline__ PullBases(const int32_t* __restrict__ nbr, int tile, int cell) {
    const int x = cell & 3, y = (cell >> 2) & 3, z = cell >> 4;
    xlo = x == 0; xhi = x == 3; ylo = y == 0; yhi = y == 3; zlo = z == 0; zhi = z == 3;
    const int sx = xlo ? -1 : (int)xhi, sy = ylo ? -1 : (int)yhi, sz = zlo ? -1 : (int)zhi;
    const int32_t* __restrict__ row = nbr + (int64_t)tile * 27 + 13;
    auto nb = [&](int o) -> I { return (I)max(__ldg(row + o), 0) * (I)ZF_PT; };
    b0 = (I)tile * (I)ZF_PT + (I)cell;
    bx = nb(sx) + (I)(cell - 4 * sx);
    by = nb(3 * sy) + (I)(cell - 16 * sy);
    bz = nb(9 * sz) + (I)(cell - 64 * sz);
    bxy = nb(sx + 3 * sy) + (I)(cell - 4 * sx - 16 * sy);
    bxz = nb(sx + 9 * sz) + (I)(cell - 4 * sx - 64 * sz);
    byz = nb(3 * sy + 9 * sz) + (I)(cell - 16 * sy - 64 * sz);
  }
  // source of the pull along q (q < 18; a constant after unrolling)
  __device__ __forceinline__ I src(int q) const {
    const bool cx = EX(q) > 0 ? xlo : (EX(q) < 0 ? xhi : false);
    const bool cy = EY(q) > 0 ? ylo : (EY(q) < 0 ? yhi : false);
    const bool cz = EZ(q) > 0 ? zlo : (EZ(q) < 0 ? zhi : false);
    I b;
    if (EX(q) && EY(q)) b = cx ? (cy ? bxy : bx) : (cy ? by : b0);
    else if (EX(q) && EZ(q)) b = cx ? (cz ? bxz : bx) : (cz ? bz : b0);
    else if (EY(q) && EZ(q)) b = cy ? (cz ? byz : by) : (cz ? bz : b0);
    else if (EX(q)) b = cx ? bx : b0;
    else if (EY(q)) b = cy ? by : b0;
    else b = cz ? bz : b0;
    return b + (I)(q * ZF_TC - EX(q) - 4 * EY(q) - 16 * EZ(q));
  }
  // where the pull along q comes from, given the point's link word
  __device__ __forceinline__ I pull(int q, uint32_t link) const {
    if (q == 18) return b0 + (I)(18 * ZF_TC);
    return (link & (1u << q)) ? b0 + (I)(OPP(q) * ZF_TC) : src(q);
  }
};

// 32 random bits for the pair of directions (q-1, q) from the point's seed:
// an odd multiply and an xor-shift of a Weyl step (the seed itself is a full
// avalanche hash of point and step)
__device__ __forceinline__ uint32_t pair_bits(uint32_t seed, int q) {
  uint32_t h = (seed + (uint32_t)q * 0x9E3779B9u) * 0x85EBCA6Bu;
  return h ^ (h >> 16);
}

// kMom: write the post-collision moments (the step before a membrane/IB
// block); kSR: stochastic rounding of the 16-bit forms.  Both are launch
// constants made template parameters so that the unrolled direction loop
// carries no branch on them.
template <class C, typename I, bool kMom, bool kSR>
__global__ void __launch_bounds__(kTilesPerBlock * ZF_TC, 6) k_lbm(LbmArgs a) {
  using T = typename C::T;
  constexpr bool kHalf = IsHalf<C>::v;
  const int lt = threadIdx.x >> 6, cell = threadIdx.x & 63;
  const int ti = blockIdx.x * kTilesPerBlock + lt;
  bool live = ti < a.n_active;
  const int tile = live ? __ldg(a.active + ti) : 0;
  const I self = (I)tile * ZF_TC + (I)cell;  // point slot
  const uint32_t link = live ? __ldg(a.link + self) : 0u;
  live = live && (link >> 31);
  float rho = 0.f;

  if (live) {
    const I ns = (I)a.ns;
    const T* __restrict__ fin = static_cast<const T*>(a.fin);
    T* __restrict__ fout = static_cast<T*>(a.fout);
    const PullBases<I> pb(a.nbr, tile, cell);

    // pull from the upstream point x - e_q; halfway bounce-back where flagged.
    // 16-bit forms stay in storage units (deviation x 2^16) until the moments.
    float d[ZF_Q];
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) {
      const T v = fin[pb.pull(q, link)];
      if constexpr (kHalf) d[q] = (float)v;
      else d[q] = C::dec(v, q, a);
    }

    float tau = a.tau;
    if (a.tau_from_phase) tau = 0.5f + 0.72f * (float)a.code[self];  // ZebraflowWT.c:6110
    float Fx = a.gx, Fy = a.gy, Fz = a.gz;
    {
      const float bx = a.force[self], by = a.force[ns + self], bz = a.force[2 * ns + self];
      Fx += a.force_dt * bx;
      Fy += a.force_dt * by;
      Fz += a.force_dt * bz;
      if (a.zero_force) {
        a.force[self] = 0.f;
        a.force[ns + self] = 0.f;
        a.force[2 * ns + self] = 0.f;
      }
    }

    // moments with the half-force shift, ZebraflowWT.c:6125-6135:
    // rho = rho_ref + sum w d,  m = sum w c d  (sum w c = 0)
    float drho = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
    if constexpr (kHalf) {
      // from the sums and differences of the opposite pairs (q, q + 1), q even
      // (fewer instructions; the fp32 forms keep the per-direction order)
      float S[9], Dd[9];
#pragma unroll
      for (int p = 0; p < 9; ++p) {
        S[p] = d[2 * p] + d[2 * p + 1];
        Dd[p] = d[2 * p] - d[2 * p + 1];
      }
      drho = fmaf(WQ(18), d[18], fmaf(WQ(0), S[0] + S[1] + S[2], WQ(6) * ((S[3] + S[4]) + (S[5] + S[6]) + (S[7] + S[8]))));
      mx = fmaf(WQ(0), Dd[0], WQ(6) * ((Dd[3] - Dd[4]) + (Dd[5] - Dd[6])));  // c_x of q = 6, 8, 10, 12: +, -, +, -
      my = fmaf(WQ(0), Dd[1], WQ(6) * ((Dd[3] + Dd[4]) + (Dd[7] - Dd[8])));  // c_y of q = 6, 8, 14, 16: +, +, +, -
      mz = fmaf(WQ(0), Dd[2], WQ(6) * ((Dd[5] + Dd[6]) + (Dd[7] + Dd[8])));  // c_z of q = 10, 12, 14, 16: all +
    } else {
#pragma unroll
      for (int q = 0; q < ZF_Q; ++q) {
        const float wd = WQ(q) * d[q];
        drho += wd;
        if (EX(q)) mx += EX(q) * wd;
        if (EY(q)) my += EY(q) * wd;
        if (EZ(q)) mz += EZ(q) * wd;
      }
    }
    if constexpr (kHalf) {
      drho *= a.inv_scale;
      mx *= a.inv_scale;
      my *= a.inv_scale;
      mz *= a.inv_scale;
    }
    rho = a.rho_ref + drho;
    const float irho = 1.f / rho;
    const float ux = (mx + 0.5f * Fx) * irho, uy = (my + 0.5f * Fy) * irho,
                uz = (mz + 0.5f * Fz) * irho;
    const float omega = 1.f / tau;
    const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);
    const float uF = ux * Fx + uy * Fy + uz * Fz;
    const float sfac = 1.f - 0.5f * omega;

    // BGK + Guo source in deviation form, ZebraflowWT.c:6138-6142:
    // d' = d + omega (deq - d) + src/w,  deq = drho + rho (3cu + 4.5cu^2 - 1.5u^2),
    // src/w = sfac (3 (cF - uF) + 9 cu cF); per point constants A, K1..K5 turn
    // deq into two FMAs and the source into two.  fp32 deviations keep the
    // form d + omega (deq - d) + src, which rounds only the non-equilibrium
    // part (exact mass to fp32 round-off); 16-bit forms, whose storage rounds
    // at 2^-11, use d' = (1 - omega) d + E with E = omega deq + src folded
    // into per-point constants in storage units.
    const float A = drho - rho * usq15;
    const float K1 = 3.f * rho, K2 = 4.5f * rho, K3 = 9.f * sfac, K4 = 3.f * sfac, K5 = 3.f * sfac * uF;
    const float sc = kHalf ? a.scale : 1.f;
    const float omc = 1.f - omega;
    const float Aw = sc * (omega * A - K5), K1w = sc * omega * K1, K2w = sc * omega * K2,
                K3s = sc * K3, K4s = sc * K4;
    float r2 = 0.f, m2x = 0.f, m2y = 0.f, m2z = 0.f;
    uint32_t rseed = 0;
    if (kHalf) rseed = mix32((uint32_t)self * 0x9E3779B1u + a.step * 0x85EBCA77u);
    float dn_prev = 0.f, dn_odd = 0.f;
    T* __restrict__ fo = fout + pb.b0;
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) {
      float dn;
      if constexpr (std::is_same<C, RawF32>::value) {
        // plain populations: the reference's expression as written
        const float cu = cdot(q, ux, uy, uz), cF = cdot(q, Fx, Fy, Fz);
        const float deq = drho + rho * (3.f * cu + 4.5f * cu * cu - usq15);
        const float src = sfac * (3.f * (cF - uF) + 9.f * cu * cF);
        dn = d[q] + omega * (deq - d[q]) + src;
      } else if constexpr (kHalf) {
        // E(q) = Aw + K1w cu + K2w cu^2 + K4s cF + K3s cu cF; the opposite
        // direction q + 1 has -cu, -cF: E = S +- T with S, T shared
        if (q == 18) {
          dn = fmaf(omc, d[q], Aw);
        } else if ((q & 1) == 0) {
          const float cu = cdot(q, ux, uy, uz), cF = cdot(q, Fx, Fy, Fz);
          const float Sq = fmaf(cu, fmaf(K2w, cu, K3s * cF), Aw), Tq = fmaf(K1w, cu, K4s * cF);
          dn = fmaf(omc, d[q], Sq + Tq);
          dn_odd = fmaf(omc, d[q + 1], Sq - Tq);
        } else {
          dn = dn_odd;
        }
      } else if (q == 18) {
        dn = fmaf(omega, A - d[q], d[q]) - K5;
      } else {
        const float cu = cdot(q, ux, uy, uz), cF = cdot(q, Fx, Fy, Fz);
        const float deq = fmaf(cu, fmaf(K2, cu, K1), A);
        const float src = fmaf(K3 * cu, cF, fmaf(K4, cF, -K5));
        dn = fmaf(omega, deq - d[q], d[q]) + src;
      }
      if constexpr (kHalf) {
        if (kSR && q < 18) {
          if (q & 1) {  // pairs (q-1, q): one stochastic-rounding conversion
            uint32_t r;
            C::cvt2_sr(r, dn_prev, dn, pair_bits(rseed, q));
            const T lo = C::from_bits((unsigned short)(r & 0xffffu));
            const T hi = C::from_bits((unsigned short)(r >> 16));
            fo[(q - 1) * ZF_TC] = lo;
            fo[q * ZF_TC] = hi;
            if (kMom) {
              const float d0 = (float)lo, d1 = (float)hi;
              r2 += WQ(q - 1) * d0 + WQ(q) * d1;
              if (EX(q - 1)) m2x += EX(q - 1) * WQ(q - 1) * d0;
              if (EY(q - 1)) m2y += EY(q - 1) * WQ(q - 1) * d0;
              if (EZ(q - 1)) m2z += EZ(q - 1) * WQ(q - 1) * d0;
              if (EX(q)) m2x += EX(q) * WQ(q) * d1;
              if (EY(q)) m2y += EY(q) * WQ(q) * d1;
              if (EZ(q)) m2z += EZ(q) * WQ(q) * d1;
            }
          } else {
            dn_prev = dn;
          }
          continue;
        }
        const T v = C::cvt_rn(dn);
        fo[q * ZF_TC] = v;
        if (kMom) {
          const float ds = (float)v;
          r2 += WQ(q) * ds;
          if (EX(q)) m2x += EX(q) * WQ(q) * ds;
          if (EY(q)) m2y += EY(q) * WQ(q) * ds;
          if (EZ(q)) m2z += EZ(q) * WQ(q) * ds;
        }
      } else {
        const T v = C::enc(dn, q, a);
        fo[q * ZF_TC] = v;
        if (kMom) {
          const float ds = C::dec(v, q, a);
          r2 += WQ(q) * ds;
          if (EX(q)) m2x += EX(q) * WQ(q) * ds;
          if (EY(q)) m2y += EY(q) * WQ(q) * ds;
          if (EZ(q)) m2z += EZ(q) * WQ(q) * ds;
        }
      }
    }
    if (kMom) {  // post-collision moments without force shift, ZebraflowWT.c:6611-6614
      if constexpr (kHalf) {
        r2 *= a.inv_scale;
        m2x *= a.inv_scale;
        m2y *= a.inv_scale;
        m2z *= a.inv_scale;
      }
      const float D = a.rho_ref + r2;
      a.mom[self] = D;
      a.mom[ns + self] = m2x / D;
      a.mom[2 * ns + self] = m2y / D;
      a.mom[3 * ns + self] = m2z / D;
    }
    if (a.write_rho_pre) a.rho_pre[self] = rho;
    if (a.write_u_pre) {  // U, V, W of the collision pass, ZebraflowWT.c:6133-6135
      a.u_pre[self] = ux;
      a.u_pre[ns + self] = uy;
      a.u_pre[2 * ns + self] = uz;
    }
  }

  if (a.mass_partial) {  // FP64 block sum of the fluid density (uniform branch)
    double m = (double)rho;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m += __shfl_down_sync(0xffffffffu, m, o);
    __shared__ double s_part[kTilesPerBlock * ZF_TC / 32];
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kTilesPerBlock * ZF_TC / 32; ++w) t += s_part[w];
      a.mass_partial[blockIdx.x] = t;
    }
  }
}

// Inlet/outlet pressure (Pa) of reference code 1001..1009 at iteration iter:
// the reference's cardiac waveforms (ZebraflowWT.c:6318-6418) with its float
// locals (simtime, cycletime, taucycle, pressure; :2283) and double constants.
__device__ float inlet_pressure(int code, int64_t iter, double dt_us) {
  const float simtime = (float)((double)iter * (dt_us * 1.e-06));  // iter*T_SCALE
  const double T = 0.36;
  const double lag = code == 1001 ? 0.0 : (code == 1002 ? 0.06 * 0.36 : 0.2 * 0.36);
  float cycletime = (float)fmod((double)simtime - lag, T);
  if (code != 1001 && cycletime < 0) cycletime = (float)(cycletime + T);
  const float taucycle = (float)(cycletime / T);
  if (code == 1003 || code == 1004 || code == 1005) {
    const double base = code == 1003 ? 11. : (code == 1004 ? 18. : 23.);
    const double amp = code == 1003 ? 23. : 27.;
    if (taucycle <= 0.3) return (float)(120. + base + amp * sinf((float)(3.14159265359 * taucycle / 0.6)));
    return (float)(120. + base +
                   amp * (1. + sinf((float)(2 * 3.14159265359 * (taucycle + 0.4) / 1.4 - 3.14159265359 / 2.))) / 2.);
  }
  double base = 28.5, amp = 60.;  // 1007, 1009
  if (code == 1001) base = 54., amp = 82.;
  else if (code == 1002) base = 48., amp = 68.;
  else if (code == 1006 || code == 1008) base = 29., amp = 66.;
  if (taucycle <= 0.23) {
    const float s1 = sinf((float)(3.14159265359 * taucycle / 0.46));
    return (float)(120. + base + amp * s1 * s1);
  }
  return (float)(120. + base +
                 amp * (1. + sinf((float)(2 * 3.14159265359 * (taucycle + 0.54) / 1.54 - 3.14159265359 / 2.))) / 2.);
}

// Reference boundary points (ZebraflowWT.c:6292-6433): a wall point takes
// F[c][n] = feq(D[m], u=0) and a pressure inlet/outlet feq(P(t)/
// LBM_PRESSURE_SCALE + 1, u[m]) (LBM_PRESSURE_SCALE = 1e4/3 Pa), m its
// designated neighbour; then the moments pass for those points (:6603-6616).
template <class C>
__global__ void k_lbm_wall(LbmArgs a, const int32_t* __restrict__ wall_slot,
                           const int32_t* __restrict__ wall_nbr, int n_wall) {
  using T = typename C::T;
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_wall) return;
  const int64_t slot = wall_slot[w];
  const int nb = wall_nbr[w];
  const uint8_t self_code = a.code[slot];
  const T* __restrict__ fin = static_cast<const T*>(a.fin);
  // density and momentum of a boundary neighbour as the reference's copy pass
  // left them in D, U, V, W: the moments of its previous populations
  auto bc_moments = [&](float& r, float& mx, float& my, float& mz) {
    r = mx = my = mz = 0.f;
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) {
      const float d = C::dec(fin[pop_at(q, (int64_t)nb)], q, a);
      r += WQ(q) * d;
      if (EX(q)) mx += EX(q) * WQ(q) * d;
      if (EY(q)) my += EY(q) * WQ(q) * d;
      if (EZ(q)) mz += EZ(q) * WQ(q) * d;
    }
    r += a.rho_ref;  // sum w = 1, sum w c = 0
  };
  float rho_m = a.rho_ref, ux = 0.f, uy = 0.f, uz = 0.f;
  if (zf_code_pressure(self_code)) {
    const float P = inlet_pressure(1000 + (self_code - ZF_CODE_PRESSURE0), a.iter_now, a.dt_us);
    rho_m = (float)(P / (1. / 3. * 10. * 1000.) + 1.);  // D_bc, ZebraflowWT.c:6421
    if (nb >= 0) {
      if (zf_code_fluid(a.code[nb])) {  // U, V, W of this step's collision pass
        ux = a.u_pre[nb];
        uy = a.u_pre[a.ns + nb];
        uz = a.u_pre[2 * a.ns + nb];
      } else {
        float r, mx, my, mz;
        bc_moments(r, mx, my, mz);
        ux = mx / r;
        uy = my / r;
        uz = mz / r;
      }
    }
  } else if (nb >= 0) {
    // D_bc = D[m] (ZebraflowWT.c:6306-6311): a fluid neighbour's density is this
    // step's (k_lbm wrote it); a boundary neighbour's is what the reference's
    // copy pass left in D, the density of its populations of the previous step
    if (zf_code_fluid(a.code[nb])) {
      rho_m = a.rho_pre[nb];
    } else {
      float r, mx, my, mz;
      bc_moments(r, mx, my, mz);
      rho_m = r;
    }
  }
  T* __restrict__ fout = static_cast<T*>(a.fout);
  const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);
  float r2 = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) {
    const float cu = cdot(q, ux, uy, uz);
    // feq(rho, u)/w - rho_ref (ZebraflowWT.c:6430)
    const T v = C::enc(rho_m * (1.f + 3.f * cu + 4.5f * cu * cu - usq15) - a.rho_ref, q, a);
    fout[pop_at(q, slot)] = v;
    const float ds = C::dec(v, q, a);
    r2 += WQ(q) * ds;
    mx += EX(q) * WQ(q) * ds;
    my += EY(q) * WQ(q) * ds;
    mz += EZ(q) * WQ(q) * ds;
  }
  if (a.store_moments) {
    const float D = a.rho_ref + r2;
    a.mom[slot] = D;
    a.mom[a.ns + slot] = mx / D;
    a.mom[2 * a.ns + slot] = my / D;
    a.mom[3 * a.ns + slot] = mz / D;
  }
  if (a.zero_force) {
    a.force[slot] = 0.f;
    a.force[a.ns + slot] = 0.f;
    a.force[2 * a.ns + slot] = 0.f;
  }
}

// populations f at the boundary <-> stored values (plain fp32 stores f itself)
template <class C>
__device__ __forceinline__ typename C::T from_f(float f, int q, const LbmArgs& a) {
  if constexpr (std::is_same<C, RawF32>::value) return f;
  else return C::enc(__fmul_rn(__fsub_rn(f, RawF32::wr(q, a)), IWQ(q)), q, a);
}
template <class C>
__device__ __forceinline__ float to_f(typename C::T v, int q, const LbmArgs& a) {
  if constexpr (std::is_same<C, RawF32>::value) return v;
  else return __fmaf_rn(WQ(q), C::dec(v, q, a), RawF32::wr(q, a));
}

template <class C>
__global__ void k_fill_equilibrium(typename C::T* f, int64_t ns, LbmArgs a) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) f[pop_at(q, s)] = C::enc(0.f, q, a);
}

template <class C>
__global__ void k_scatter_pop(typename C::T* f, int64_t ns, const float* __restrict__ stage,
                              const int32_t* __restrict__ dom_slot, int64_t n, LbmArgs a) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int64_t s = dom_slot[l];
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q)
    f[pop_at(q, s)] = from_f<C>(stage[q * n + l], q, a);
}

template <class C>
__global__ void k_gather_pop(const typename C::T* f, int64_t ns, float* __restrict__ stage,
                             const int32_t* __restrict__ dom_slot, int64_t n, LbmArgs a) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int64_t s = dom_slot[l];
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) stage[q * n + l] = to_f<C>(f[pop_at(q, s)], q, a);
}

__global__ void k_scatter_planes(float* dst, int64_t ns, const float* __restrict__ stage,
                                 const int32_t* __restrict__ dom_slot, int64_t n, int planes) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int64_t s = dom_slot[l];
  for (int p = 0; p < planes; ++p) dst[p * ns + s] = stage[p * n + l];
}

__global__ void k_gather_planes(const float* src, int64_t ns, float* __restrict__ stage,
                                const int32_t* __restrict__ dom_slot, int64_t n, int planes) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int64_t s = dom_slot[l];
  for (int p = 0; p < planes; ++p) stage[p * n + l] = src[p * ns + s];
}

// Global mass: per-block FP64 partial sums into scratch, then one block sums
// the partials in a fixed order (deterministic).
template <class C>
__global__ void k_mass_partial(const typename C::T* __restrict__ f, int64_t ns,
                               const uint8_t* __restrict__ code, int include_walls,
                               double* __restrict__ partial, LbmArgs a) {
  double acc = 0.0;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ns;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t cd = code[s];
    const bool take = zf_code_fluid(cd) || (include_walls && (cd == ZF_CODE_WALL || zf_code_pressure(cd)));
    if (!take) continue;
    double r = a.rho_ref;
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) r += (double)WQ(q) * (double)C::dec(f[pop_at(q, s)], q, a);
    acc += r;
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_sum_partials(const double* __restrict__ partial, int n, double* out) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

static LbmArgs make_args(zf_ctx* c) {
  LbmArgs a{};
  const zf_params& P = c->p;
  a.fin = c->d_f[c->cur];
  a.fout = c->d_f[c->cur ^ 1];
  a.active = c->d_active;
  a.n_active = c->n_active;
  a.nbr = c->d_nbr;
  a.link = c->d_link;
  a.code = c->d_code;
  a.force = c->d_force;
  a.mom = c->d_mom;
  a.rho_pre = c->d_rho_pre;
  a.u_pre = c->d_u_pre;
  a.write_u_pre = c->n_pressure > 0;
  a.iter_now = c->status.iter + 1;
  a.dt_us = P.dt;
  a.ns = c->ns;
  a.tau = P.tau;
  a.force_dt = (float)P.dt;
  a.gx = P.g[0];
  a.gy = P.g[1];
  a.gz = P.g[2];
  a.rho_ref = P.rho_ref;
  // deviations d are O(1e-6..1e-2); 2^16 keeps them in the normal fp16 range
  const bool half = P.storage == ZF_STORE_F16 || P.storage == ZF_STORE_BF16;
  a.scale = half ? 65536.f : 1.f;
  a.inv_scale = 1.f / a.scale;
  a.stochastic = half && P.stochastic_round;
  a.step = (uint32_t)c->status.iter;
  a.tau_from_phase = P.tau_from_phase;
  a.write_rho_pre = P.wall_mode == ZF_WALL_REF_EQ;
  return a;
}

// Dispatch on the storage form.
template <template <class> class K, typename... Args>
static void dispatch_storage(int storage, Args&&... args) {
  switch (storage) {
    case ZF_STORE_F16: K<DevF16>::run(args...); break;
    case ZF_STORE_BF16: K<DevBF16>::run(args...); break;
    case ZF_STORE_F32_DEV: K<DevF32>::run(args...); break;
    default: K<RawF32>::run(args...); break;
  }
}

template <class C>
struct LaunchStep {
  template <typename I>
  static void launch_lbm(zf_ctx* c, const LbmArgs& a, int grid) {
    const int nt = kTilesPerBlock * ZF_TC;
    if constexpr (IsHalf<C>::v) {
      if (a.stochastic) {
        if (a.store_moments) k_lbm<C, I, true, true><<<grid, nt, 0, c->stream>>>(a);
        else k_lbm<C, I, false, true><<<grid, nt, 0, c->stream>>>(a);
        return;
      }
    }
    if (a.store_moments) k_lbm<C, I, true, false><<<grid, nt, 0, c->stream>>>(a);
    else k_lbm<C, I, false, false><<<grid, nt, 0, c->stream>>>(a);
  }
  // a.active / a.n_active: the tiles to step (all active tiles, or a part of
  // them); walls: also run the reference wall pass
  static void run(zf_ctx* c, const LbmArgs& a, bool walls = true) {
    if (a.n_active > 0) {
      const int grid = (a.n_active + kTilesPerBlock - 1) / kTilesPerBlock;
      if ((int64_t)ZF_Q * c->ns < (int64_t)INT32_MAX)
        launch_lbm<int32_t>(c, a, grid);
      else
        launch_lbm<int64_t>(c, a, grid);
    }
    if (walls && c->p.wall_mode == ZF_WALL_REF_EQ && c->n_wall > 0)
      k_lbm_wall<C><<<(c->n_wall + 255) / 256, 256, 0, c->stream>>>(a, c->d_wall_slot,
                                                                    c->d_wall_nbr, c->n_wall);
  }
};

int ensure_red(zf_ctx* c, int n) {
  if (c->red_cap >= n) return ZF_OK;
  if (c->d_red) cudaFree(c->d_red);
  c->d_red = nullptr;
  c->red_cap = 0;
  int rc = dev_alloc(c, (void**)&c->d_red, (size_t)n * sizeof(double));
  if (rc) return rc;
  c->red_cap = n;
  return ZF_OK;
}

int lbm_launch(zf_ctx* c, int store_moments, int zero_force, double* mass_out) {
  LbmArgs a = make_args(c);
  a.store_moments = store_moments;
  a.zero_force = zero_force;
  const int grid = (c->n_active + kTilesPerBlock - 1) / kTilesPerBlock;
  if (mass_out) {
    int rc0 = ensure_red(c, grid + 1);
    if (rc0) return rc0;
    a.mass_partial = c->d_red;
  }
  dispatch_storage<LaunchStep>(c->p.storage, c, a);
  ZF_CUDA(cudaGetLastError());
  c->launches += (c->n_active > 0) + (c->p.wall_mode == ZF_WALL_REF_EQ && c->n_wall > 0) +
                 (mass_out ? 1 : 0);
  c->cur ^= 1;
  if (mass_out) {
    k_sum_partials<<<1, 256, 0, c->stream>>>(c->d_red, grid, c->d_red + grid);
    ZF_CUDA(cudaGetLastError());
    ZF_CUDA(cudaMemcpyAsync(mass_out, c->d_red + grid, sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    ZF_CUDA(cudaStreamSynchronize(c->stream));
  }
  return ZF_OK;
}

// One part of a slab step (zf_set_slab): the inner tile layers (part 0) or
// the two face layers next to the halo (part 1); finish: the step is complete
// (wall pass, swap of the population buffers).
int lbm_launch_part(zf_ctx* c, int part, int finish, int store_moments, int zero_force) {
  LbmArgs a = make_args(c);
  a.active = c->d_active_part[part];
  a.n_active = c->n_active_part[part];
  a.store_moments = store_moments;
  a.zero_force = zero_force;
  dispatch_storage<LaunchStep>(c->p.storage, c, a, finish != 0);
  ZF_CUDA(cudaGetLastError());
  c->launches += (a.n_active > 0) + (finish && c->p.wall_mode == ZF_WALL_REF_EQ && c->n_wall > 0);
  if (finish) c->cur ^= 1;
  return ZF_OK;
}

// Moments D, U, V, W of the current populations at every listed point:
// post-collision values without force shift, as the reference's LBM_FLUID
// pass stores them (ZebraflowWT.c:6603-6616).
template <class C>
__global__ void k_moments(LbmArgs a) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.ns || a.code[s] == ZF_CODE_SOLID) return;
  const typename C::T* __restrict__ f = static_cast<const typename C::T*>(a.fin);
  float r2 = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) {
    const float d = C::dec(f[pop_at(q, s)], q, a);
    r2 += WQ(q) * d;
    if (EX(q)) mx += EX(q) * WQ(q) * d;
    if (EY(q)) my += EY(q) * WQ(q) * d;
    if (EZ(q)) mz += EZ(q) * WQ(q) * d;
  }
  const float D = a.rho_ref + r2;
  a.mom[s] = D;
  a.mom[a.ns + s] = mx / D;
  a.mom[2 * a.ns + s] = my / D;
  a.mom[3 * a.ns + s] = mz / D;
}

template <class C>
struct Moments {
  static void run(zf_ctx* c, const LbmArgs& a) {
    k_moments<C><<<(unsigned)((c->ns + 255) / 256), 256, 0, c->stream>>>(a);
  }
};

int lbm_moments_launch(zf_ctx* c) {
  if (c->ns == 0) return ZF_OK;
  const LbmArgs a = make_args(c);  // a.fin: the current populations
  dispatch_storage<Moments>(c->p.storage, c, a);
  ZF_CUDA(cudaGetLastError());
  c->launches += 1;
  return ZF_OK;
}

// ---- adjoint of the LBM step ----------------------------------------------------
//
// Forward step at a fluid point x (halfway bounce-back walls): pull
// f_q = f_old[q](x - e_q), or f_old[opp q](x) where the link bounces back; then
//   rho = sum f, m = sum c f, u = (m + F/2)/rho, F = g + dt BODYFORCE(x),
//   f'_q = f_q + w (feq_q - f_q) + S_q,   w = 1/tau,
//   feq_q = w_q rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u),
//   S_q   = (1 - w/2) w_q (3 (c - u).F + 9 (c.u)(c.F))      (ZebraflowWT.c:6125-6142).
// Every f_old value of a fluid point is pulled by exactly one fluid point, so
// the transpose of the pull is a permutation: the adjoint of f_q at x is stored
// at the slot the forward pulled it from, with no atomics.  With lam the
// adjoint of f'(x), the transposed collision is
//   lam_in_p = (1 - w) lam_p + A + sum_a B_a (c_pa - u_a)/rho,
//   A   = w sum_q lam_q w_q (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u),
//   B_a = sum_q lam_q [w w_q rho (3 c_qa + 9 (c.u) c_qa - 3 u_a)
//                      + (1 - w/2) w_q (9 c_qa (c.F) - 3 F_a)],
// and the parameter sensitivities of the step are
//   dJ/dF_a = B_a/(2 rho) + sum_q lam_q (1 - w/2) w_q (3 (c_qa - u_a) + 9 (c.u) c_qa),
//   dJ/dw   = sum_q lam_q (feq_q - f_q - S_q / (2 - w)).
// gF accumulates dt dJ/dF (the sensitivity to BODYFORCE), gw per block dJ/dw.
template <class C, typename I>
__global__ void __launch_bounds__(kTilesPerBlock * ZF_TC, 4)
    k_lbm_adj(LbmArgs a, const float* __restrict__ lam, float* __restrict__ lam_prev,
              float* __restrict__ gF, double* __restrict__ gw_partial) {
  __shared__ double s_gw[kTilesPerBlock * ZF_TC / 32];
  const int lt = threadIdx.x >> 6, cell = threadIdx.x & 63;
  const int ti = blockIdx.x * kTilesPerBlock + lt;
  bool live = ti < a.n_active;
  const int tile = live ? __ldg(a.active + ti) : 0;
  const I self = (I)tile * ZF_TC + (I)cell;
  const uint32_t link = live ? a.link[self] : 0u;
  live = live && (link >> 31);
  double gw = 0.0;
  if (live) {
    const I ns = (I)a.ns;
    const typename C::T* __restrict__ fin = static_cast<const typename C::T*>(a.fin);
    const PullBases<I> pb(a.nbr, tile, cell);
    const float* __restrict__ lp = lam + pb.b0;
    // every sum over q below is a polynomial of degree <= 2 in c_q weighted by
    // lam_q w_q, so it is built from the moments of lam: L0 = sum lam w,
    // L1_a = sum lam w c_a, L2_ab = sum lam w c_a c_b, and LD = sum lam w d
    // with d = f/w - rho_ref the populations' deviations
    float drho = 0.f, mx = 0.f, my = 0.f, mz = 0.f, LD = 0.f, L0 = 0.f, L1x = 0.f, L1y = 0.f, L1z = 0.f;
    float Lxx = 0.f, Lyy = 0.f, Lzz = 0.f, Lxy = 0.f, Lxz = 0.f, Lyz = 0.f;
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) {
      const float d = C::dec(fin[pb.pull(q, link)], q, a);
      const float l = lp[q * ZF_TC];
      const float wd = WQ(q) * d;
      drho += wd;
      if (EX(q)) mx += EX(q) * wd;
      if (EY(q)) my += EY(q) * wd;
      if (EZ(q)) mz += EZ(q) * wd;
      const float lw = WQ(q) * l;
      LD = fmaf(lw, d, LD);
      L0 += lw;
      if (EX(q)) {
        L1x += EX(q) * lw;
        Lxx += lw;
      }
      if (EY(q)) {
        L1y += EY(q) * lw;
        Lyy += lw;
      }
      if (EZ(q)) {
        L1z += EZ(q) * lw;
        Lzz += lw;
      }
      if (EX(q) && EY(q)) Lxy += EX(q) * EY(q) * lw;
      if (EX(q) && EZ(q)) Lxz += EX(q) * EZ(q) * lw;
      if (EY(q) && EZ(q)) Lyz += EY(q) * EZ(q) * lw;
    }
    const float Fx = a.gx + a.force_dt * a.force[self], Fy = a.gy + a.force_dt * a.force[ns + self],
                Fz = a.gz + a.force_dt * a.force[2 * ns + self];
    const float rho = a.rho_ref + drho, irho = 1.f / rho;
    const float ux = (mx + 0.5f * Fx) * irho, uy = (my + 0.5f * Fy) * irho, uz = (mz + 0.5f * Fz) * irho;
    const float om = 1.f / a.tau, sfac = 1.f - 0.5f * om;
    const float usq = ux * ux + uy * uy + uz * uz, uF = ux * Fx + uy * Fy + uz * Fz;
    // L2 u and L2 F
    const float U2x = Lxx * ux + Lxy * uy + Lxz * uz, U2y = Lxy * ux + Lyy * uy + Lyz * uz,
                U2z = Lxz * ux + Lyz * uy + Lzz * uz;
    const float F2x = Lxx * Fx + Lxy * Fy + Lxz * Fz, F2y = Lxy * Fx + Lyy * Fy + Lyz * Fz,
                F2z = Lxz * Fx + Lyz * Fy + Lzz * Fz;
    // sum_q lam_q w_q (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u) = L0 + Adev
    const float Adev = -1.5f * usq * L0 + 3.f * (ux * L1x + uy * L1y + uz * L1z) +
                       4.5f * (ux * U2x + uy * U2y + uz * U2z);
    const float Araw = L0 + Adev;
    // B_a = w rho (3 L1_a + 9 (L2 u)_a - 3 u_a L0) + sfac (9 (L2 F)_a - 3 F_a L0)
    const float orho = om * rho;
    const float Bx = orho * (3.f * L1x + 9.f * U2x - 3.f * ux * L0) + sfac * (9.f * F2x - 3.f * Fx * L0);
    const float By = orho * (3.f * L1y + 9.f * U2y - 3.f * uy * L0) + sfac * (9.f * F2y - 3.f * Fy * L0);
    const float Bz = orho * (3.f * L1z + 9.f * U2z - 3.f * uz * L0) + sfac * (9.f * F2z - 3.f * Fz * L0);
    // dJ/dF_a = sfac (3 L1_a - 3 u_a L0 + 9 (L2 u)_a) + B_a / (2 rho)
    const float gFx = sfac * (3.f * (L1x - ux * L0) + 9.f * U2x) + 0.5f * Bx * irho;
    const float gFy = sfac * (3.f * (L1y - uy * L0) + 9.f * U2y) + 0.5f * By * irho;
    const float gFz = sfac * (3.f * (L1z - uz * L0) + 9.f * U2z) + 0.5f * Bz * irho;
    gF[self] += a.force_dt * gFx;
    gF[ns + self] += a.force_dt * gFy;
    gF[2 * ns + self] += a.force_dt * gFz;
    // dJ/dw = sum lam (feq - f) - 1/2 sum lam w (3 (c.F - u.F) + 9 (c.u)(c.F)), with
    // sum lam (feq - f) = sum lam w (rho poly - rho_ref - d) = rho_ref Adev + drho Araw - LD:
    // differences of O(u) terms, not of O(1) sums
    gw = (double)(a.rho_ref * Adev + drho * Araw - LD -
                  0.5f * (3.f * (Fx * L1x + Fy * L1y + Fz * L1z) - 3.f * uF * L0 + 9.f * (ux * F2x + uy * F2y + uz * F2z)));
    // lam_in_q = (1 - w) lam_q + w Araw + B.(c_q - u)/rho; lam is read again
    // (an L1/L2 hit) and the pull sources recomputed rather than held
    const float om1 = 1.f - om;
    const float bx = Bx * irho, by = By * irho, bz = Bz * irho;
    const float A0 = om * Araw - (bx * ux + by * uy + bz * uz);
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) lam_prev[pb.pull(q, link)] = fmaf(om1, lp[q * ZF_TC], A0) + cdot(q, bx, by, bz);
  }
  // per-block sum of dJ/dw (uniform branch)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) gw += __shfl_down_sync(0xffffffffu, gw, o);
  if ((threadIdx.x & 31) == 0) s_gw[threadIdx.x >> 5] = gw;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTilesPerBlock * ZF_TC / 32; ++w) t += s_gw[w];
    gw_partial[blockIdx.x] += t;
  }
}

// Velocities of the populations f at listed slots (the compact points of a
// WSS objective's stencils): the arithmetic of k_moments, U[3][nu].
template <class C>
__global__ void k_moments_at(LbmArgs a, const int32_t* __restrict__ uslot, int nu, float* __restrict__ U) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  const int64_t s = uslot[u];
  const typename C::T* __restrict__ f = static_cast<const typename C::T*>(a.fin);
  float r2 = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) {
    const float d = C::dec(f[pop_at(q, s)], q, a);
    r2 += WQ(q) * d;
    if (EX(q)) mx += EX(q) * WQ(q) * d;
    if (EY(q)) my += EY(q) * WQ(q) * d;
    if (EZ(q)) mz += EZ(q) * WQ(q) * d;
  }
  const float D = a.rho_ref + r2;
  U[u] = mx / D;
  U[nu + u] = my / D;
  U[2 * nu + u] = mz / D;
}

// The objective's seed at the compact points: lam[q](x) += sum_a gU_a(x)
// (c_qa - U_a)/rho, U and rho the moments (no force shift) of the populations
// f; gU is cleared for the next seed.
template <class C>
__global__ void k_seed_at(LbmArgs a, const int32_t* __restrict__ uslot, int nu, float* __restrict__ gU,
                          float* __restrict__ lam) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  const float gx = gU[u], gy = gU[nu + u], gz = gU[2 * nu + u];
  if (gx == 0.f && gy == 0.f && gz == 0.f) return;
  gU[u] = gU[nu + u] = gU[2 * nu + u] = 0.f;
  const int64_t s = uslot[u];
  const typename C::T* __restrict__ f = static_cast<const typename C::T*>(a.fin);
  float fq[ZF_Q], rho = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) {
    fq[q] = to_f<C>(f[pop_at(q, s)], q, a);
    rho += fq[q];
    mx += EX(q) * fq[q];
    my += EY(q) * fq[q];
    mz += EZ(q) * fq[q];
  }
  const float ir = 1.f / rho, Ux = mx * ir, Uy = my * ir, Uz = mz * ir;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q)
    lam[pop_at(q, s)] += (gx * (EX(q) - Ux) + gy * (EY(q) - Uy) + gz * (EZ(q) - Uz)) * ir;
}

template <class C>
struct AdjStep {
  static void run(zf_ctx* c, const LbmArgs& a, const float* lam, float* lam_prev, float* gF, double* gw) {
    if (c->n_active == 0) return;
    const int grid = (c->n_active + kTilesPerBlock - 1) / kTilesPerBlock;
    if ((int64_t)ZF_Q * c->ns < (int64_t)INT32_MAX)
      k_lbm_adj<C, int32_t><<<grid, kTilesPerBlock * ZF_TC, 0, c->stream>>>(a, lam, lam_prev, gF, gw);
    else
      k_lbm_adj<C, int64_t><<<grid, kTilesPerBlock * ZF_TC, 0, c->stream>>>(a, lam, lam_prev, gF, gw);
  }
};
template <class C>
struct MomentsAt {
  static void run(zf_ctx* c, const LbmArgs& a, const PatchStencil& ps, float* U) {
    k_moments_at<C><<<(ps.nu + 255) / 256, 256, 0, c->stream>>>(a, ps.uslot, ps.nu, U);
  }
};
template <class C>
struct SeedAt {
  static void run(zf_ctx* c, const LbmArgs& a, const PatchStencil& ps, float* gU, float* lam) {
    k_seed_at<C><<<(ps.nu + 255) / 256, 256, 0, c->stream>>>(a, ps.uslot, ps.nu, gU, lam);
  }
};
template <class C>
struct StepBuffers {
  static void run(zf_ctx* c, const LbmArgs& a) { LaunchStep<C>::run(c, a); }
};
// number of per-block partial sums k_lbm_adj writes
int lbm_adj_blocks(zf_ctx* c) { return (c->n_active + kTilesPerBlock - 1) / kTilesPerBlock; }

// one adjoint step: f_pre are the populations before the forward step
int lbm_adj_launch(zf_ctx* c, const void* f_pre, const float* lam, float* lam_prev, float* gF,
                   double* gw_partial) {
  LbmArgs a = make_args(c);
  a.fin = f_pre;
  dispatch_storage<AdjStep>(c->p.storage, c, a, lam, lam_prev, gF, gw_partial);
  ZF_CUDA(cudaGetLastError());
  c->launches += c->n_active > 0;
  return ZF_OK;
}

int lbm_moments_of(zf_ctx* c, const void* f) {
  if (c->ns == 0) return ZF_OK;
  LbmArgs a = make_args(c);
  a.fin = f;
  dispatch_storage<Moments>(c->p.storage, c, a);
  ZF_CUDA(cudaGetLastError());
  c->launches += 1;
  return ZF_OK;
}

int lbm_moments_at(zf_ctx* c, const void* f, const PatchStencil& ps, float* d_U) {
  if (ps.nu <= 0) return ZF_OK;
  LbmArgs a = make_args(c);
  a.fin = f;
  dispatch_storage<MomentsAt>(c->p.storage, c, a, ps, d_U);
  ZF_CUDA(cudaGetLastError());
  c->launches += 1;
  return ZF_OK;
}

int lbm_seed_at(zf_ctx* c, const void* f, const PatchStencil& ps, float* d_gU, float* lam) {
  if (ps.nu <= 0) return ZF_OK;
  LbmArgs a = make_args(c);
  a.fin = f;
  dispatch_storage<SeedAt>(c->p.storage, c, a, ps, d_gU, lam);
  ZF_CUDA(cudaGetLastError());
  c->launches += 1;
  return ZF_OK;
}

// forward step from explicit population buffers (the body force and
// parameters of the context; no moments, no force clearing); `step` seeds the
// stochastic rounding of the 16-bit forms, so a step recomputed with the same
// number reproduces its populations bit for bit
int lbm_step_buffers(zf_ctx* c, const void* fin, void* fout, uint32_t step) {
  LbmArgs a = make_args(c);
  a.fin = fin;
  a.fout = fout;
  a.step = step;
  dispatch_storage<StepBuffers>(c->p.storage, c, a);
  ZF_CUDA(cudaGetLastError());
  c->launches += (c->n_active > 0) + (c->p.wall_mode == ZF_WALL_REF_EQ && c->n_wall > 0);
  return ZF_OK;
}

template <class C>
struct Fill {
  static void run(zf_ctx* c, const LbmArgs& a, int b) {
    k_fill_equilibrium<C><<<(int)((c->ns + 255) / 256), 256, 0, c->stream>>>(
        (typename C::T*)c->d_f[b], c->ns, a);
  }
};

int lbm_init_equilibrium(zf_ctx* c) {
  if (c->ns == 0) return ZF_OK;  // a lattice without listed points
  LbmArgs a = make_args(c);
  for (int b = 0; b < 2; ++b) {
    dispatch_storage<Fill>(c->p.storage, c, a, b);
    ZF_CUDA(cudaGetLastError());
  }
  // moments of the rest state: D = rho_ref, U = V = W = 0
  std::vector<float> ones(c->ns, c->p.rho_ref);
  ZF_CUDA(cudaMemcpyAsync(c->d_mom, ones.data(), c->ns * sizeof(float), cudaMemcpyHostToDevice,
                          c->stream));
  ZF_CUDA(cudaMemsetAsync(c->d_mom + c->ns, 0, 3 * c->ns * sizeof(float), c->stream));
  if (c->d_rho_pre) {
    ZF_CUDA(cudaMemcpyAsync(c->d_rho_pre, ones.data(), c->ns * sizeof(float),
                            cudaMemcpyHostToDevice, c->stream));
  }
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

template <class C>
struct Scatter {
  static void run(zf_ctx* c, const LbmArgs& a, int64_t n) {
    k_scatter_pop<C><<<(int)((n + 255) / 256), 256, 0, c->stream>>>(
        (typename C::T*)c->d_f[c->cur], c->ns, c->d_stage, c->d_dom_slot, n, a);
  }
};
template <class C>
struct Gather {
  static void run(zf_ctx* c, const LbmArgs& a, int64_t n) {
    k_gather_pop<C><<<(int)((n + 255) / 256), 256, 0, c->stream>>>(
        (const typename C::T*)c->d_f[c->cur], c->ns, c->d_stage, c->d_dom_slot, n, a);
  }
};

int lbm_upload_populations(zf_ctx* c, const float* h) {
  const int64_t n = c->n_listed;
  if (n == 0) return ZF_OK;
  ZF_CUDA(cudaMemcpyAsync(c->d_stage, h, (size_t)ZF_Q * n * sizeof(float),
                          cudaMemcpyHostToDevice, c->stream));
  dispatch_storage<Scatter>(c->p.storage, c, make_args(c), n);
  ZF_CUDA(cudaGetLastError());
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int lbm_download_populations(zf_ctx* c, float* h) {
  const int64_t n = c->n_listed;
  if (n == 0) return ZF_OK;
  dispatch_storage<Gather>(c->p.storage, c, make_args(c), n);
  ZF_CUDA(cudaGetLastError());
  ZF_CUDA(cudaMemcpyAsync(h, c->d_stage, (size_t)ZF_Q * n * sizeof(float),
                          cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int lbm_scatter_listed(zf_ctx* c, const float* h, int planes, float* d_dst) {
  const int64_t n = c->n_listed;
  if (n == 0) return ZF_OK;
  ZF_CUDA(cudaMemcpyAsync(c->d_stage, h, (size_t)planes * n * sizeof(float),
                          cudaMemcpyHostToDevice, c->stream));
  k_scatter_planes<<<(int)((n + 255) / 256), 256, 0, c->stream>>>(d_dst, c->ns, c->d_stage,
                                                                  c->d_dom_slot, n, planes);
  ZF_CUDA(cudaGetLastError());
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int lbm_gather_listed(zf_ctx* c, const float* d_src, int planes, float* h) {
  const int64_t n = c->n_listed;
  if (n == 0) return ZF_OK;
  k_gather_planes<<<(int)((n + 255) / 256), 256, 0, c->stream>>>(d_src, c->ns, c->d_stage,
                                                                 c->d_dom_slot, n, planes);
  ZF_CUDA(cudaGetLastError());
  ZF_CUDA(cudaMemcpyAsync(h, c->d_stage, (size_t)planes * n * sizeof(float),
                          cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

// z-slab halo exchange: the 5 populations with e_z = dir of the listed points
// of plane k, [n][5] raw storage elements (ET: 4 or 2 bytes), in (x, y) order
__host__ __device__ constexpr int zface_q(int dir, int d) {
  return dir > 0 ? (d == 0 ? 4 : 8 + 2 * d) : (d == 0 ? 5 : 9 + 2 * d);  // {4,10,12,14,16} / {5,11,13,15,17}
}
template <typename ET>
__global__ void k_plane_copy(ET* __restrict__ f, const int32_t* __restrict__ slots, int n, int dir,
                             ET* __restrict__ buf, int pack) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const int64_t s = slots[m];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int q = dir > 0 ? zface_q(1, d) : zface_q(-1, d);
    if (pack) buf[m * 5 + d] = f[pop_at(q, s)];
    else f[pop_at(q, s)] = buf[m * 5 + d];
  }
}

int lbm_plane_slots(zf_ctx* c, int k, zf_ctx::PlaneSlots* out) {
  if (k < 0 || k >= c->p.nz) {
    set_error("plane %d outside the lattice (nz %d)", k, c->p.nz);
    return ZF_ERR_ARG;
  }
  for (const auto& pl : c->planes)
    if (pl.k == k) {
      *out = pl;
      return ZF_OK;
    }
  // listed points of the plane, ordered by (x, y)
  std::vector<std::pair<int64_t, int32_t>> pts;
  const int ntx = c->ntx, nty = c->nty;
  for (int64_t l = 0; l < c->n_listed; ++l) {
    const int i = c->domlist[3 * l], j = c->domlist[3 * l + 1], kk = c->domlist[3 * l + 2];
    if (kk != k) continue;
    const int64_t t = ((int64_t)(kk / ZF_TS) * nty + j / ZF_TS) * ntx + i / ZF_TS;
    const int32_t id = c->h_tile_map[t];
    if (id < 0) continue;
    const int32_t slot = id * ZF_TC + (i % ZF_TS) + ZF_TS * (j % ZF_TS) + ZF_TS * ZF_TS * (kk % ZF_TS);
    pts.emplace_back((int64_t)i * c->p.ny + j, slot);
  }
  std::sort(pts.begin(), pts.end());
  std::vector<int32_t> slots(pts.size());
  for (size_t m = 0; m < pts.size(); ++m) slots[m] = pts[m].second;
  zf_ctx::PlaneSlots pl{k, (int)slots.size(), nullptr};
  int rc = dev_alloc(c, (void**)&pl.d_slots, std::max<size_t>(slots.size(), 1) * sizeof(int32_t));
  if (rc) return rc;
  if (!slots.empty())
    ZF_CUDA(cudaMemcpyAsync(pl.d_slots, slots.data(), slots.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  c->planes.push_back(pl);
  *out = pl;
  return ZF_OK;
}

int lbm_plane_copy(zf_ctx* c, int k, int dir, void* buf, bool pack) {
  zf_ctx::PlaneSlots pl{};
  int rc = lbm_plane_slots(c, k, &pl);
  if (rc) return rc;
  if (pl.n == 0) return ZF_OK;
  if (!buf) return ZF_ERR_ARG;
  const bool half = c->p.storage == ZF_STORE_F16 || c->p.storage == ZF_STORE_BF16;
  const unsigned grid = (unsigned)((pl.n + 255) / 256);
  if (half)
    k_plane_copy<uint16_t><<<grid, 256, 0, c->stream>>>(static_cast<uint16_t*>(c->d_f[c->cur]), pl.d_slots,
                                                         pl.n, dir, static_cast<uint16_t*>(buf), pack);
  else
    k_plane_copy<uint32_t><<<grid, 256, 0, c->stream>>>(static_cast<uint32_t*>(c->d_f[c->cur]), pl.d_slots,
                                                         pl.n, dir, static_cast<uint32_t*>(buf), pack);
  ZF_CUDA(cudaGetLastError());
  c->launches += 1;
  return ZF_OK;
}

template <class C>
struct Mass {
  static void run(zf_ctx* c, const LbmArgs& a, int nblk, int include_walls) {
    k_mass_partial<C><<<nblk, 256, 0, c->stream>>>((const typename C::T*)c->d_f[c->cur], c->ns,
                                                   c->d_code, include_walls, c->d_red, a);
  }
};

int lbm_mass(zf_ctx* c, int include_walls, double* out) {
  const int nblk = 148 * 8;
  int rc0 = ensure_red(c, nblk + 1);
  if (rc0) return rc0;
  dispatch_storage<Mass>(c->p.storage, c, make_args(c), nblk, include_walls);
  ZF_CUDA(cudaGetLastError());
  k_sum_partials<<<1, 256, 0, c->stream>>>(c->d_red, nblk, c->d_red + nblk);
  ZF_CUDA(cudaGetLastError());
  ZF_CUDA(cudaMemcpyAsync(out, c->d_red + nblk, sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

}  // namespace zf

// ---- allocation-free step with the fused FP64 mass sum ----------------------
//
// Some callers cannot call cudaMalloc once their run has started: code whose
// device memory is owned by another allocator that has already reserved the
// GPU (a framework's caching allocator, a fixed memory budget), and time loops
// that must not take cudaMalloc's implicit device synchronisation or risk an
// out-of-memory failure half-way through a run.  For them the per-block
// partial sums of the mass reduction live in this file-scope device array
// instead of scratch memory from cudaMalloc.  Every GPU that loads the
// library holds the array (512 KB) until the process exits.
namespace zf {

constexpr int kNoAllocMaxBlocks = 65536;  // partial sums: one per block of 4 tiles
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks + 1];

// Device address of g_noalloc_scratch on `device`, looked up once per device
// with that device current.  In host code the array's name is only a host-side
// stand-in; kernels must be given this address instead.  The cached address
// belongs to the device's primary context: after cudaDeviceReset on that
// device it is stale, so a process that resets a device must not call the
// allocation-free entry on it again.
static int noalloc_scratch(int device, double** out) {
  static std::mutex mu;
  static double* addr[256] = {};
  if (device < 0 || device >= 256) {
    set_error("zf_lbm_step_mass_noalloc: device %d out of range", device);
    return ZF_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    ZF_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    addr[device] = static_cast<double*>(p);
  }
  *out = addr[device];
  return ZF_OK;
}

int lbm_step_mass_noalloc(zf_ctx* c, int store_moments, int zero_force, double* mass_out) {
  const int grid = (c->n_active + kTilesPerBlock - 1) / kTilesPerBlock;
  if (grid > kNoAllocMaxBlocks) {
    set_error("zf_lbm_step_mass_noalloc: the lattice needs %d partial sums but the "
              "allocation-free scratch holds %d (at most %d tiles of 4x4x4 points with fluid); "
              "use zf_lbm_step_mass",
              grid, kNoAllocMaxBlocks, kNoAllocMaxBlocks * kTilesPerBlock);
    return ZF_ERR_ARG;
  }
  double* scratch = nullptr;
  int rc = noalloc_scratch(c->device, &scratch);
  if (rc) return rc;
  // Every block of the step writes its own partial sum and the final sum
  // overwrites scratch[grid]: nothing accumulates across calls, so nothing
  // needs clearing.  Calls that overlap on the GPU (other streams, other
  // contexts on the same device) share the array and race.
  LbmArgs a = make_args(c);
  a.store_moments = store_moments;
  a.zero_force = zero_force;
  a.mass_partial = scratch;
  dispatch_storage<LaunchStep>(c->p.storage, c, a);
  ZF_CUDA(cudaGetLastError());
  c->cur ^= 1;
  k_sum_partials<<<1, 256, 0, c->stream>>>(scratch, grid, scratch + grid);
  ZF_CUDA(cudaGetLastError());
  // the step kernel, the wall pass where it runs, and the sum
  c->launches += (c->n_active > 0) + (c->p.wall_mode == ZF_WALL_REF_EQ && c->n_wall > 0) + 1;
  ZF_CUDA(cudaMemcpyAsync(mass_out, scratch + grid, sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

}  // namespace zf

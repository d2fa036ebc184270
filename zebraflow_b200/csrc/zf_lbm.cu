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
// point; a 256-thread block covers 4 tiles.  The 27-neighbour tile table and
// the per-tile source masks of a block's tiles are staged in shared memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "zf_internal.h"

namespace zf {

__constant__ int c_ex[ZF_Q] = {1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0, 0};
__constant__ int c_ey[ZF_Q] = {0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 0};
__constant__ int c_ez[ZF_Q] = {0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0};
// Weights: 1/18 for c=1..6, 1/36 for c=7..18, 1/3 for the rest population
// (ZebraflowWT.c:72-74, :2329-2333).
__constant__ float c_w[ZF_Q] = {1.f / 18, 1.f / 18, 1.f / 18, 1.f / 18, 1.f / 18, 1.f / 18,
                                1.f / 36, 1.f / 36, 1.f / 36, 1.f / 36, 1.f / 36, 1.f / 36,
                                1.f / 36, 1.f / 36, 1.f / 36, 1.f / 36, 1.f / 36, 1.f / 36,
                                1.f / 3};
__constant__ float c_iw[ZF_Q] = {18.f, 18.f, 18.f, 18.f, 18.f, 18.f, 36.f, 36.f, 36.f, 36.f,
                                 36.f, 36.f, 36.f, 36.f, 36.f, 36.f, 36.f, 36.f, 3.f};

__host__ __device__ __forceinline__ int opp(int q) {
  // reference: cc = c-1 for even c, c+1 for odd c (ZebraflowWT.c:6114-6115), rest to itself
  return q == 18 ? 18 : (q ^ 1);
}

// Storage codecs: fp32 stores f; fp16/bf16 store S*(f/w - rho_ref).
template <typename T>
struct Codec;
template <>
struct Codec<float> {
  __device__ __forceinline__ static float dec(float v, int, const LbmArgs&) { return v; }
  __device__ __forceinline__ static float enc(float f, int, const LbmArgs&) { return f; }
};
template <>
struct Codec<__half> {
  __device__ __forceinline__ static float dec(__half v, int q, const LbmArgs& a) {
    return c_w[q] * (a.rho_ref + __half2float(v) * a.inv_scale);
  }
  __device__ __forceinline__ static __half enc(float f, int q, const LbmArgs& a) {
    return __float2half_rn((f * c_iw[q] - a.rho_ref) * a.scale);
  }
};
template <>
struct Codec<__nv_bfloat16> {
  __device__ __forceinline__ static float dec(__nv_bfloat16 v, int q, const LbmArgs& a) {
    return c_w[q] * (a.rho_ref + __bfloat162float(v) * a.inv_scale);
  }
  __device__ __forceinline__ static __nv_bfloat16 enc(float f, int q, const LbmArgs& a) {
    return __float2bfloat16_rn((f * c_iw[q] - a.rho_ref) * a.scale);
  }
};

constexpr int kTilesPerBlock = 4;

template <typename T>
__global__ void __launch_bounds__(kTilesPerBlock * ZF_TC) k_lbm(LbmArgs a) {
  __shared__ int s_nbr[kTilesPerBlock][27];
  __shared__ unsigned long long s_mask[kTilesPerBlock][27];
  const int lt = threadIdx.x >> 6, cell = threadIdx.x & 63;
  const int tb = blockIdx.x * kTilesPerBlock;
  for (int t = threadIdx.x; t < kTilesPerBlock * 27; t += blockDim.x) {
    const int l = t / 27, s = t - l * 27;
    int nb = -1;
    unsigned long long m = 0;
    if (tb + l < a.n_active) {
      const int tile = a.active[tb + l];
      nb = a.nbr[(int64_t)tile * 27 + s];
      if (nb >= 0) m = a.src_mask[nb];
    }
    s_nbr[l][s] = nb;
    s_mask[l][s] = m;
  }
  __syncthreads();
  bool live = tb + lt < a.n_active;
  const int tile = live ? s_nbr[lt][13] : 0;
  live = live && ((a.fluid_mask[tile] >> cell) & 1ull);
  float rho = 0.f;

  if (live) {
    const int x = cell & 3, y = (cell >> 2) & 3, z = cell >> 4;
    const int64_t self = (int64_t)tile * ZF_TC + cell;
    const int64_t ns = a.ns;
    const T* __restrict__ fin = static_cast<const T*>(a.fin);
    T* __restrict__ fout = static_cast<T*>(a.fout);

    float f[ZF_Q];
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) {
      const int sx = x - c_ex[q], sy = y - c_ey[q], sz = z - c_ez[q];
      const int slot27 = ((sz >> 2) + 1) * 9 + ((sy >> 2) + 1) * 3 + ((sx >> 2) + 1);
      const int scell = (sx & 3) | ((sy & 3) << 2) | ((sz & 3) << 4);
      const int nb = s_nbr[lt][slot27];
      const bool ok = (s_mask[lt][slot27] >> scell) & 1ull;
      // pull from the upstream point; halfway bounce-back when it is not a source
      const int64_t idx = ok ? (int64_t)q * ns + (int64_t)nb * ZF_TC + scell
                             : (int64_t)opp(q) * ns + self;
      f[q] = Codec<T>::dec(fin[idx], q, a);
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

    // moments with the half-force shift, ZebraflowWT.c:6125-6135
    float mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) {
      rho += f[q];
      mx += f[q] * c_ex[q];
      my += f[q] * c_ey[q];
      mz += f[q] * c_ez[q];
    }
    const float irho = 1.f / rho;
    const float ux = (mx + 0.5f * Fx) * irho, uy = (my + 0.5f * Fy) * irho,
                uz = (mz + 0.5f * Fz) * irho;
    const float omega = 1.f / tau;
    const float usq = ux * ux + uy * uy + uz * uz;
    const float uF = ux * Fx + uy * Fy + uz * Fz;
    const float sfac = 1.f - 0.5f * omega;

    // BGK + Guo source, ZebraflowWT.c:6138-6142
    float r2 = 0.f, m2x = 0.f, m2y = 0.f, m2z = 0.f;
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) {
      const float cu = ux * c_ex[q] + uy * c_ey[q] + uz * c_ez[q];
      const float cF = Fx * c_ex[q] + Fy * c_ey[q] + Fz * c_ez[q];
      const float feq = rho * c_w[q] * (1.f + 3.f * cu + 4.5f * cu * cu - 1.5f * usq);
      const float src = sfac * c_w[q] * (3.f * (cF - uF) + 9.f * cu * cF);
      const float fp = f[q] * (1.f - omega) + feq * omega + src;
      const T v = Codec<T>::enc(fp, q, a);
      fout[(int64_t)q * ns + self] = v;
      if (a.store_moments) {
        const float fs = Codec<T>::dec(v, q, a);
        r2 += fs;
        m2x += fs * c_ex[q];
        m2y += fs * c_ey[q];
        m2z += fs * c_ez[q];
      }
    }
    if (a.store_moments) {  // post-collision moments without force shift, ZebraflowWT.c:6611-6614
      a.mom[self] = r2;
      a.mom[ns + self] = m2x / r2;
      a.mom[2 * ns + self] = m2y / r2;
      a.mom[3 * ns + self] = m2z / r2;
    }
    if (a.write_rho_pre) a.rho_pre[self] = rho;
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

// Reference wall points: F[c][n] = feq(D[m], u=0) with m the designated
// neighbour (ZebraflowWT.c:6303-6315, :6429-6432), then the moments pass for
// those points (ZebraflowWT.c:6603-6616).
template <typename T>
__global__ void k_lbm_wall(LbmArgs a, const int32_t* __restrict__ wall_slot,
                           const int32_t* __restrict__ wall_nbr, int n_wall) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_wall) return;
  const int64_t slot = wall_slot[w];
  const int nb = wall_nbr[w];
  const float rho_m = nb >= 0 ? a.rho_pre[nb] : a.rho_ref;
  T* __restrict__ fout = static_cast<T*>(a.fout);
  float r2 = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) {
    const T v = Codec<T>::enc(rho_m * c_w[q], q, a);
    fout[(int64_t)q * a.ns + slot] = v;
    const float fs = Codec<T>::dec(v, q, a);
    r2 += fs;
    mx += fs * c_ex[q];
    my += fs * c_ey[q];
    mz += fs * c_ez[q];
  }
  if (a.store_moments) {
    a.mom[slot] = r2;
    a.mom[a.ns + slot] = mx / r2;
    a.mom[2 * a.ns + slot] = my / r2;
    a.mom[3 * a.ns + slot] = mz / r2;
  }
  if (a.zero_force) {
    a.force[slot] = 0.f;
    a.force[a.ns + slot] = 0.f;
    a.force[2 * a.ns + slot] = 0.f;
  }
}

template <typename T>
__global__ void k_fill_equilibrium(T* f, int64_t ns, LbmArgs a) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) f[q * ns + s] = Codec<T>::enc(a.rho_ref * c_w[q], q, a);
}

template <typename T>
__global__ void k_scatter_pop(T* f, int64_t ns, const float* __restrict__ stage,
                              const int32_t* __restrict__ dom_slot, int64_t n, LbmArgs a) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int64_t s = dom_slot[l];
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) f[q * ns + s] = Codec<T>::enc(stage[q * n + l], q, a);
}

template <typename T>
__global__ void k_gather_pop(const T* f, int64_t ns, float* __restrict__ stage,
                             const int32_t* __restrict__ dom_slot, int64_t n, LbmArgs a) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const int64_t s = dom_slot[l];
#pragma unroll
  for (int q = 0; q < ZF_Q; ++q) stage[q * n + l] = Codec<T>::dec(f[q * ns + s], q, a);
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
template <typename T>
__global__ void k_mass_partial(const T* __restrict__ f, int64_t ns, const uint8_t* __restrict__ code,
                               int include_walls, double* __restrict__ partial, LbmArgs a) {
  double acc = 0.0;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ns;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t cd = code[s];
    const bool take = (cd >= 1 && cd <= 9) || (include_walls && cd == ZF_CODE_WALL);
    if (!take) continue;
    double r = 0.0;
#pragma unroll
    for (int q = 0; q < ZF_Q; ++q) r += (double)Codec<T>::dec(f[q * ns + s], q, a);
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
  a.src_mask = c->d_src_mask;
  a.fluid_mask = c->d_fluid_mask;
  a.code = c->d_code;
  a.force = c->d_force;
  a.mom = c->d_mom;
  a.rho_pre = c->d_rho_pre;
  a.ns = c->ns;
  a.tau = P.tau;
  a.force_dt = (float)P.dt;
  a.gx = P.g[0];
  a.gy = P.g[1];
  a.gz = P.g[2];
  a.rho_ref = P.rho_ref;
  // deviations (f/w - rho_ref) are O(1e-6..1e-2); 2^16 keeps them normal in fp16
  a.scale = P.storage == ZF_STORE_F32 ? 1.f : 65536.f;
  a.inv_scale = 1.f / a.scale;
  a.tau_from_phase = P.tau_from_phase;
  a.write_rho_pre = P.wall_mode == ZF_WALL_REF_EQ;
  return a;
}

template <typename T>
static int launch_typed(zf_ctx* c, LbmArgs a) {
  if (c->n_active > 0) {
    const int grid = (c->n_active + kTilesPerBlock - 1) / kTilesPerBlock;
    k_lbm<T><<<grid, kTilesPerBlock * ZF_TC, 0, c->stream>>>(a);
    ZF_CUDA(cudaGetLastError());
  }
  if (c->p.wall_mode == ZF_WALL_REF_EQ && c->n_wall > 0) {
    k_lbm_wall<T><<<(c->n_wall + 255) / 256, 256, 0, c->stream>>>(a, c->d_wall_slot,
                                                                   c->d_wall_nbr, c->n_wall);
    ZF_CUDA(cudaGetLastError());
  }
  return ZF_OK;
}

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
  int rc;
  switch (c->p.storage) {
    case ZF_STORE_F16: rc = launch_typed<__half>(c, a); break;
    case ZF_STORE_BF16: rc = launch_typed<__nv_bfloat16>(c, a); break;
    default: rc = launch_typed<float>(c, a); break;
  }
  if (rc != ZF_OK) return rc;
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

int lbm_init_equilibrium(zf_ctx* c) {
  LbmArgs a = make_args(c);
  const int grid = (int)((c->ns + 255) / 256);
  for (int b = 0; b < 2; ++b) {
    switch (c->p.storage) {
      case ZF_STORE_F16:
        k_fill_equilibrium<__half><<<grid, 256, 0, c->stream>>>((__half*)c->d_f[b], c->ns, a);
        break;
      case ZF_STORE_BF16:
        k_fill_equilibrium<__nv_bfloat16>
            <<<grid, 256, 0, c->stream>>>((__nv_bfloat16*)c->d_f[b], c->ns, a);
        break;
      default:
        k_fill_equilibrium<float><<<grid, 256, 0, c->stream>>>((float*)c->d_f[b], c->ns, a);
    }
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

int lbm_upload_populations(zf_ctx* c, const float* h) {
  const int64_t n = c->n_listed;
  if (n == 0) return ZF_OK;
  ZF_CUDA(cudaMemcpyAsync(c->d_stage, h, (size_t)ZF_Q * n * sizeof(float),
                          cudaMemcpyHostToDevice, c->stream));
  LbmArgs a = make_args(c);
  const int grid = (int)((n + 255) / 256);
  switch (c->p.storage) {
    case ZF_STORE_F16:
      k_scatter_pop<__half><<<grid, 256, 0, c->stream>>>((__half*)c->d_f[c->cur], c->ns,
                                                         c->d_stage, c->d_dom_slot, n, a);
      break;
    case ZF_STORE_BF16:
      k_scatter_pop<__nv_bfloat16><<<grid, 256, 0, c->stream>>>(
          (__nv_bfloat16*)c->d_f[c->cur], c->ns, c->d_stage, c->d_dom_slot, n, a);
      break;
    default:
      k_scatter_pop<float><<<grid, 256, 0, c->stream>>>((float*)c->d_f[c->cur], c->ns,
                                                        c->d_stage, c->d_dom_slot, n, a);
  }
  ZF_CUDA(cudaGetLastError());
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int lbm_download_populations(zf_ctx* c, float* h) {
  const int64_t n = c->n_listed;
  if (n == 0) return ZF_OK;
  LbmArgs a = make_args(c);
  const int grid = (int)((n + 255) / 256);
  switch (c->p.storage) {
    case ZF_STORE_F16:
      k_gather_pop<__half><<<grid, 256, 0, c->stream>>>((const __half*)c->d_f[c->cur], c->ns,
                                                        c->d_stage, c->d_dom_slot, n, a);
      break;
    case ZF_STORE_BF16:
      k_gather_pop<__nv_bfloat16><<<grid, 256, 0, c->stream>>>(
          (const __nv_bfloat16*)c->d_f[c->cur], c->ns, c->d_stage, c->d_dom_slot, n, a);
      break;
    default:
      k_gather_pop<float><<<grid, 256, 0, c->stream>>>((const float*)c->d_f[c->cur], c->ns,
                                                       c->d_stage, c->d_dom_slot, n, a);
  }
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

int lbm_mass(zf_ctx* c, int include_walls, double* out) {
  const int nblk = 148 * 8;
  int rc0 = ensure_red(c, nblk + 1);
  if (rc0) return rc0;
  LbmArgs a = make_args(c);
  switch (c->p.storage) {
    case ZF_STORE_F16:
      k_mass_partial<__half><<<nblk, 256, 0, c->stream>>>(
          (const __half*)c->d_f[c->cur], c->ns, c->d_code, include_walls, c->d_red, a);
      break;
    case ZF_STORE_BF16:
      k_mass_partial<__nv_bfloat16><<<nblk, 256, 0, c->stream>>>(
          (const __nv_bfloat16*)c->d_f[c->cur], c->ns, c->d_code, include_walls, c->d_red, a);
      break;
    default:
      k_mass_partial<float><<<nblk, 256, 0, c->stream>>>(
          (const float*)c->d_f[c->cur], c->ns, c->d_code, include_walls, c->d_red, a);
  }
  ZF_CUDA(cudaGetLastError());
  k_sum_partials<<<1, 256, 0, c->stream>>>(c->d_red, nblk, c->d_red + nblk);
  ZF_CUDA(cudaGetLastError());
  ZF_CUDA(cudaMemcpyAsync(out, c->d_red + nblk, sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

}  // namespace zf

// Host side of the C ABI: context lifetime, parameters and the sparse tiled
// lattice built from reference B_index codes.
//
// Reference behaviour restated here:
//  - listed-node order: LBM_DOM_SETUP, ZebraflowWT.c:1481-1502
//  - designated neighbour of each wall point: LBM_BC_SETUP, ZebraflowWT.c:1506-1589
//  - initial state f = feq(rho, 0): ZebraflowWT.c:2562-2572, :5253-5295
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>

#include "zf_internal.h"

namespace {
thread_local std::string g_last_error;

// Reference lattice vectors, ZebraflowWT.c:2471-2497 (slot q = reference c-1).
const int kE[ZF_Q][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},
                         {0, 0, -1}, {1, 1, 0},  {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0},
                         {1, 0, 1},  {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {0, 1, 1},
                         {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 0, 0}};
}  // namespace

namespace zf {
void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int dev_alloc(zf_ctx* c, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    *p = nullptr;
    return e == cudaErrorMemoryAllocation ? ZF_ERR_NOMEM : ZF_ERR_CUDA;
  }
  c->device_bytes += (int64_t)bytes;
  return ZF_OK;
}
}  // namespace zf

using namespace zf;

extern "C" {

const char* zf_last_error(void) { return g_last_error.c_str(); }

size_t zf_params_size(void) { return sizeof(zf_params); }

zf_ctx* zf_create(const zf_params* p, int device) {
  if (!p) {
    set_error("zf_create: params is NULL");
    return nullptr;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error("zf_create: no CUDA device (%s)", cudaGetErrorString(e));
    return nullptr;
  }
  if (device < 0 || device >= ndev) {
    set_error("zf_create: device %d out of range (%d devices)", device, ndev);
    return nullptr;
  }
  if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->tau <= 0.5f || p->dx <= 0 ||
      p->storage < 0 || p->storage > 3 || p->wall_mode < 0 || p->wall_mode > 1 ||
      p->stagger <= 0) {
    set_error("zf_create: invalid parameters (lattice %dx%dx%d, tau %g, storage %d, wall %d)",
              p->nx, p->ny, p->nz, (double)p->tau, p->storage, p->wall_mode);
    return nullptr;
  }
  for (int a = 0; a < 3; ++a) {
    int n = a == 0 ? p->nx : (a == 1 ? p->ny : p->nz);
    if (p->periodic[a] && (n % ZF_TS) != 0) {
      set_error("zf_create: a periodic axis needs a length divisible by %d (axis %d has %d)",
                ZF_TS, a, n);
      return nullptr;
    }
  }
  zf_ctx* c = new zf_ctx();
  c->p = *p;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    set_error("zf_create: CUDA stream/event creation failed");
    delete c;
    return nullptr;
  }
  c->stream = c->own_stream;
  return c;
}

static void free_lattice(zf_ctx* c) {
  void* ptrs[] = {c->d_tile_map, c->d_active, c->d_nbr, c->d_link,
                  c->d_code,     c->d_f[0],   c->d_f[1],  c->d_force,    c->d_mom,
                  c->d_rho_pre,  c->d_dom_slot, c->d_stage, c->d_wall_slot, c->d_wall_nbr,
                  c->d_red,      c->d_u_pre};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (int part = 0; part < 2; ++part) {
    if (c->d_active_part[part]) cudaFree(c->d_active_part[part]);
    c->d_active_part[part] = nullptr;
    c->n_active_part[part] = 0;
  }
  c->slab_set = false;
  for (auto& pl : c->planes) cudaFree(pl.d_slots);
  c->planes.clear();
  c->d_tile_map = c->d_active = c->d_nbr = nullptr;
  c->d_link = nullptr;
  c->d_code = nullptr;
  c->d_f[0] = c->d_f[1] = nullptr;
  c->d_force = c->d_mom = c->d_rho_pre = c->d_stage = c->d_u_pre = nullptr;
  c->n_pressure = 0;
  c->d_dom_slot = c->d_wall_slot = c->d_wall_nbr = nullptr;
  c->d_red = nullptr;
  c->red_cap = 0;
  c->device_bytes = 0;
  c->lattice_set = false;
}

void zf_destroy(zf_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  ib_free(c);
  free_lattice(c);
  cells_free(c);
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->ev_ready) cudaEventDestroy(c->ev_ready);
  if (c->ev_copied) cudaEventDestroy(c->ev_copied);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

int zf_sync(zf_ctx* c) {
  if (!c) return ZF_ERR_ARG;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int zf_get_status(zf_ctx* c, zf_status* out) {
  if (!c || !out) return ZF_ERR_ARG;
  *out = c->status;
  if (c->cells_set) {
    unsigned long long cnt[4];
    ZF_CUDA(cudaMemcpyAsync(cnt, c->cells.counters, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
    ZF_CUDA(cudaStreamSynchronize(c->stream));
    out->screened_terms = (int64_t)cnt[0];
    out->cells_removed = (int64_t)cnt[1];
    out->list_overflows = (int64_t)cnt[2];
  }
  return ZF_OK;
}

int zf_device_bytes(zf_ctx* c, int64_t* bytes) {
  if (!c || !bytes) return ZF_ERR_ARG;
  *bytes = c->device_bytes;
  return ZF_OK;
}

int zf_set_lattice(zf_ctx* c, const int32_t* b) {
  if (!c || !b) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  const zf_params& P = c->p;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int64_t npts = (int64_t)nx * ny * nz;
  int64_t n_pressure = 0;
  for (int64_t n = 0; n < npts; ++n) {
    const bool pressure = b[n] >= 1001 && b[n] <= 1009;
    if (pressure && P.wall_mode != ZF_WALL_REF_EQ) {
      set_error("zf_set_lattice: pressure inlet/outlet code %d at linear index %lld needs the "
                "reference wall mode (ZF_WALL_REF_EQ)", b[n], (long long)n);
      return ZF_ERR_ARG;
    }
    if (b[n] >= 10 && !pressure) {
      set_error("zf_set_lattice: B_index %d at linear index %lld is not supported (codes are <0 "
                "solid, 0 wall, 1..9 fluid phases, 1001..1009 pressure inlets/outlets)",
                b[n], (long long)n);
      return ZF_ERR_ARG;
    }
    n_pressure += pressure;
  }
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  ib_free(c);  // the wall and IB views belong to the previous lattice
  free_lattice(c);
  c->b_index.assign(b, b + npts);

  // Listed nodes in reference DOMLIST order (i outer, k inner), ZebraflowWT.c:1485-1499.
  c->domlist.clear();
  c->n_fluid = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        int32_t v = b[((int64_t)i * ny + j) * nz + k];
        if (v >= 0) {
          c->domlist.push_back(i);
          c->domlist.push_back(j);
          c->domlist.push_back(k);
          if (v > 0 && v < 10) c->n_fluid++;
        }
      }
  c->n_listed = (int64_t)c->domlist.size() / 3;

  // Tiles holding populations: every tile with at least one listed point.
  const int ntx = (nx + ZF_TS - 1) / ZF_TS, nty = (ny + ZF_TS - 1) / ZF_TS,
            ntz = (nz + ZF_TS - 1) / ZF_TS;
  c->ntx = ntx;
  c->nty = nty;
  c->ntz = ntz;
  const int64_t ntiles_box = (int64_t)ntx * nty * ntz;
  std::vector<uint8_t> has_listed(ntiles_box, 0), has_fluid(ntiles_box, 0);
  for (int64_t l = 0; l < c->n_listed; ++l) {
    int i = c->domlist[3 * l], j = c->domlist[3 * l + 1], k = c->domlist[3 * l + 2];
    int64_t t = ((int64_t)(k / ZF_TS) * nty + j / ZF_TS) * ntx + i / ZF_TS;
    has_listed[t] = 1;
    const int32_t v = b[((int64_t)i * ny + j) * nz + k];
    if (v > 0 && v < 10) has_fluid[t] = 1;
  }
  c->h_tile_map.assign(ntiles_box, -1);
  c->h_tile_origin.clear();
  int64_t nt = 0;
  std::vector<int32_t> active;
  // tile ids follow (tz, ty, tx) order so that consecutive blocks touch neighbouring tiles
  for (int64_t t = 0; t < ntiles_box; ++t) {
    if (!has_listed[t]) continue;
    c->h_tile_map[t] = (int32_t)nt;
    int tx = (int)(t % ntx), ty = (int)((t / ntx) % nty), tz = (int)(t / ((int64_t)ntx * nty));
    c->h_tile_origin.push_back(tx * ZF_TS);
    c->h_tile_origin.push_back(ty * ZF_TS);
    c->h_tile_origin.push_back(tz * ZF_TS);
    if (has_fluid[t]) active.push_back((int32_t)nt);
    ++nt;
  }
  if (nt > (int64_t)INT32_MAX / ZF_TC) {
    set_error("zf_set_lattice: %lld tiles exceed the 32-bit slot index", (long long)nt);
    return ZF_ERR_ARG;
  }
  c->n_pop_tiles = nt;
  c->n_all_tiles = nt;
  c->n_active = (int)active.size();
  c->ns = nt * ZF_TC;
  const int64_t ns = c->ns;

  auto slot_of = [&](int i, int j, int k) -> int64_t {
    int64_t t = ((int64_t)(k / ZF_TS) * nty + j / ZF_TS) * ntx + i / ZF_TS;
    int32_t id = c->h_tile_map[t];
    if (id < 0) return -1;
    return (int64_t)id * ZF_TC + (i % ZF_TS) + ZF_TS * (j % ZF_TS) + ZF_TS * ZF_TS * (k % ZF_TS);
  };

  // Codes and slots of listed nodes.
  std::vector<uint8_t> code(ns, ZF_CODE_SOLID);
  std::vector<int32_t> dom_slot(c->n_listed);
  for (int64_t l = 0; l < c->n_listed; ++l) {
    int i = c->domlist[3 * l], j = c->domlist[3 * l + 1], k = c->domlist[3 * l + 2];
    int32_t v = b[((int64_t)i * ny + j) * nz + k];
    int64_t s = slot_of(i, j, k);
    dom_slot[l] = (int32_t)s;
    code[s] = v >= 1000 ? (uint8_t)(ZF_CODE_PRESSURE0 + (v - 1000)) : v > 0 ? (uint8_t)v : (uint8_t)ZF_CODE_WALL;
  }
  // Link word of every fluid point: bit 31 marks the point live, bit q that the
  // pull along q bounces back because its upstream point x - e_q is not a
  // source.  Sources are fluid points (bounce-back mode) or every listed point
  // (reference wall-equilibrium mode: wall points carry feq).
  std::vector<uint32_t> link(ns, 0u);
  const bool ref_eq = P.wall_mode == ZF_WALL_REF_EQ;
  for (int64_t l = 0; l < c->n_listed; ++l) {
    int i = c->domlist[3 * l], j = c->domlist[3 * l + 1], k = c->domlist[3 * l + 2];
    const int32_t v0 = b[((int64_t)i * ny + j) * nz + k];
    if (!(v0 > 0 && v0 < 10)) continue;  // collided points only, ZebraflowWT.c:6109
    uint32_t w = 1u << 31;
    for (int q = 0; q < ZF_Q - 1; ++q) {
      int p3[3] = {i - kE[q][0], j - kE[q][1], k - kE[q][2]}, lim[3] = {nx, ny, nz};
      bool src = true;
      for (int a = 0; a < 3; ++a) {
        if (p3[a] < 0 || p3[a] >= lim[a]) {
          if (!P.periodic[a]) src = false;
          p3[a] = (p3[a] + lim[a]) % lim[a];
        }
      }
      if (src) {
        int32_t v = b[((int64_t)p3[0] * ny + p3[1]) * nz + p3[2]];
        src = ref_eq ? v >= 0 : v > 0;
      }
      if (!src) w |= 1u << q;
    }
    link[dom_slot[l]] = w;
  }

  // 27-neighbour tile table with periodic wrap.
  std::vector<int32_t> nbr(nt * 27, -1);
  for (int64_t t = 0; t < nt; ++t) {
    int tx = c->h_tile_origin[3 * t] / ZF_TS, ty = c->h_tile_origin[3 * t + 1] / ZF_TS,
        tz = c->h_tile_origin[3 * t + 2] / ZF_TS;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int x = tx + dx, y = ty + dy, z = tz + dz;
          if (P.periodic[0]) x = (x + ntx) % ntx;
          if (P.periodic[1]) y = (y + nty) % nty;
          if (P.periodic[2]) z = (z + ntz) % ntz;
          int32_t id = -1;
          if (x >= 0 && x < ntx && y >= 0 && y < nty && z >= 0 && z < ntz)
            id = c->h_tile_map[((int64_t)z * nty + y) * ntx + x];
          nbr[t * 27 + (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] = id;
        }
  }

  // Designated neighbour of each wall and pressure point, reference search
  // order over c=1..18 (a fluid point, else an inlet/outlet point, else a
  // wall), ZebraflowWT.c:1530-1578.
  std::vector<int32_t> wall_slot, wall_nbr;
  c->status.bc_no_neighbour = 0;
  if (P.wall_mode == ZF_WALL_REF_EQ) {
    auto code_at = [&](int i, int j, int k, int* ii, int* jj, int* kk) -> int32_t {
      int n3[3] = {i, j, k}, lim[3] = {nx, ny, nz};
      for (int a = 0; a < 3; ++a) {
        if (n3[a] < 0 || n3[a] >= lim[a]) {
          if (!P.periodic[a]) return INT32_MIN;
          n3[a] = (n3[a] + lim[a]) % lim[a];
        }
      }
      *ii = n3[0];
      *jj = n3[1];
      *kk = n3[2];
      return b[((int64_t)n3[0] * ny + n3[1]) * nz + n3[2]];
    };
    for (int64_t l = 0; l < c->n_listed; ++l) {
      int i = c->domlist[3 * l], j = c->domlist[3 * l + 1], k = c->domlist[3 * l + 2];
      const int32_t self = b[((int64_t)i * ny + j) * nz + k];
      if (self != 0 && self < 1000) continue;
      int64_t found = -1;
      for (int pass = 0; pass < 3 && found < 0; ++pass) {
        for (int q = 0; q < ZF_Q - 1; ++q) {
          int ii, jj, kk;
          int32_t v = code_at(i + kE[q][0], j + kE[q][1], k + kE[q][2], &ii, &jj, &kk);
          if (v == INT32_MIN) continue;
          bool ok = pass == 0 ? (v > 0 && v < 1000) : (pass == 1 ? v > 1000 : v == 0);
          if (ok) {
            found = slot_of(ii, jj, kk);
            break;
          }
        }
      }
      if (found < 0) c->status.bc_no_neighbour++;
      wall_slot.push_back(dom_slot[l]);
      wall_nbr.push_back((int32_t)found);
    }
  }
  c->n_wall = (int)wall_slot.size();

  // Device allocation.
  // bytes per stored population: fp32 forms 4, fp16/bf16 deviations 2
  const size_t esz = (P.storage == ZF_STORE_F16 || P.storage == ZF_STORE_BF16) ? 2 : 4;
  int rc;
#define ALLOC(ptr, bytes)                                         \
  if ((rc = dev_alloc(c, (void**)&(ptr), (bytes))) != ZF_OK) { \
    free_lattice(c);                                              \
    return rc;                                                    \
  }
  ALLOC(c->d_tile_map, ntiles_box * sizeof(int32_t));
  ALLOC(c->d_active, std::max<size_t>(active.size(), 1) * sizeof(int32_t));
  ALLOC(c->d_nbr, nt * 27 * sizeof(int32_t));
  ALLOC(c->d_link, ns * sizeof(uint32_t));
  ALLOC(c->d_code, ns);
  ALLOC(c->d_f[0], (size_t)ZF_Q * ns * esz);
  ALLOC(c->d_f[1], (size_t)ZF_Q * ns * esz);
  ALLOC(c->d_force, 3 * ns * sizeof(float));
  ALLOC(c->d_mom, 4 * ns * sizeof(float));
  c->n_pressure = n_pressure;
  if (n_pressure > 0) ALLOC(c->d_u_pre, 3 * ns * sizeof(float));
  if (P.wall_mode == ZF_WALL_REF_EQ) {
    ALLOC(c->d_rho_pre, ns * sizeof(float));
    ALLOC(c->d_wall_slot, std::max(c->n_wall, 1) * sizeof(int32_t));
    ALLOC(c->d_wall_nbr, std::max(c->n_wall, 1) * sizeof(int32_t));
  }
  ALLOC(c->d_dom_slot, std::max<int64_t>(c->n_listed, 1) * sizeof(int32_t));
  ALLOC(c->d_stage, (size_t)ZF_Q * std::max<int64_t>(c->n_listed, 1) * sizeof(float));
#undef ALLOC

  cudaStream_t s = c->stream;
  ZF_CUDA(cudaMemcpyAsync(c->d_tile_map, c->h_tile_map.data(), ntiles_box * sizeof(int32_t),
                          cudaMemcpyHostToDevice, s));
  if (!active.empty())
    ZF_CUDA(cudaMemcpyAsync(c->d_active, active.data(), active.size() * sizeof(int32_t),
                            cudaMemcpyHostToDevice, s));
  ZF_CUDA(cudaMemcpyAsync(c->d_nbr, nbr.data(), nbr.size() * sizeof(int32_t),
                          cudaMemcpyHostToDevice, s));
  ZF_CUDA(cudaMemcpyAsync(c->d_link, link.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice,
                          s));
  ZF_CUDA(cudaMemcpyAsync(c->d_code, code.data(), ns, cudaMemcpyHostToDevice, s));
  if (c->n_listed)
    ZF_CUDA(cudaMemcpyAsync(c->d_dom_slot, dom_slot.data(), c->n_listed * sizeof(int32_t),
                            cudaMemcpyHostToDevice, s));
  if (c->n_wall) {
    ZF_CUDA(cudaMemcpyAsync(c->d_wall_slot, wall_slot.data(), c->n_wall * sizeof(int32_t),
                            cudaMemcpyHostToDevice, s));
    ZF_CUDA(cudaMemcpyAsync(c->d_wall_nbr, wall_nbr.data(), c->n_wall * sizeof(int32_t),
                            cudaMemcpyHostToDevice, s));
  }
  ZF_CUDA(cudaMemsetAsync(c->d_force, 0, 3 * ns * sizeof(float), s));
  c->cur = 0;
  if ((rc = lbm_init_equilibrium(c)) != ZF_OK) return rc;
  ZF_CUDA(cudaStreamSynchronize(s));  // host vectors above go out of scope
  c->status.iter = 0;
  c->lattice_set = true;
  return ib_prepare(c);
}

int zf_num_listed(zf_ctx* c, int64_t* n_listed, int64_t* n_fluid) {
  if (!c) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_num_listed: lattice not set");
    return ZF_ERR_STATE;
  }
  if (n_listed) *n_listed = c->n_listed;
  if (n_fluid) *n_fluid = c->n_fluid;
  return ZF_OK;
}

int zf_get_domlist(zf_ctx* c, int32_t* ijk) {
  if (!c || !ijk) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_get_domlist: lattice not set");
    return ZF_ERR_STATE;
  }
  std::memcpy(ijk, c->domlist.data(), c->domlist.size() * sizeof(int32_t));
  return ZF_OK;
}

#define NEED_LATTICE(fn)                           \
  if (!c) return ZF_ERR_ARG;                       \
  if (!c->lattice_set) {                           \
    set_error(fn ": lattice not set");             \
    return ZF_ERR_STATE;                           \
  }                                                \
  ZF_CUDA(cudaSetDevice(c->device));

int zf_upload_populations(zf_ctx* c, const float* f) {
  NEED_LATTICE("zf_upload_populations");
  if (!f) return ZF_OK;
  int rc = lbm_upload_populations(c, f);
  if (rc) return rc;
  // the stored moments follow the populations, as the reference's restart
  // loads U, V, W, D with them (ZebraflowWT.c:2649-2700)
  return lbm_moments_launch(c);
}

int zf_download_populations(zf_ctx* c, float* f) {
  NEED_LATTICE("zf_download_populations");
  if (!f) return ZF_ERR_ARG;
  return lbm_download_populations(c, f);
}

int zf_upload_bodyforce(zf_ctx* c, const float* bf) {
  NEED_LATTICE("zf_upload_bodyforce");
  if (!bf) return ZF_ERR_ARG;
  return lbm_scatter_listed(c, bf, 3, c->d_force);
}

int zf_download_bodyforce(zf_ctx* c, float* bf) {
  NEED_LATTICE("zf_download_bodyforce");
  if (!bf) return ZF_ERR_ARG;
  return lbm_gather_listed(c, c->d_force, 3, bf);
}

int zf_download_moments(zf_ctx* c, float* D, float* U, float* V, float* W) {
  NEED_LATTICE("zf_download_moments");
  float* outs[4] = {D, U, V, W};
  for (int a = 0; a < 4; ++a) {
    if (!outs[a]) continue;
    int rc = lbm_gather_listed(c, c->d_mom + (size_t)a * c->ns, 1, outs[a]);
    if (rc) return rc;
  }
  return ZF_OK;
}

int zf_lbm_moments(zf_ctx* c) {
  NEED_LATTICE("zf_lbm_moments");
  ZF_CUDA(cudaSetDevice(c->device));
  return lbm_moments_launch(c);
}

int zf_lbm_step(zf_ctx* c, int store_moments, int zero_bodyforce) {
  NEED_LATTICE("zf_lbm_step");
  int rc = lbm_launch(c, store_moments, zero_bodyforce);
  if (rc == ZF_OK) c->status.iter++;
  return rc;
}

int zf_set_slab(zf_ctx* c, int k_lo, int k_hi) {
  NEED_LATTICE("zf_set_slab");
  if (k_lo < ZF_TS || k_hi > c->p.nz - ZF_TS || k_lo % ZF_TS || k_hi % ZF_TS || k_hi - k_lo < ZF_TS) {
    set_error("zf_set_slab: interior planes [%d, %d) must be whole 4-plane tile layers with at least one "
              "layer of halo on either side (nz %d)", k_lo, k_hi, c->p.nz);
    return ZF_ERR_ARG;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  std::vector<int32_t> active(c->n_active);
  if (c->n_active)
    ZF_CUDA(cudaMemcpy(active.data(), c->d_active, active.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
  const int tz_lo = k_lo / ZF_TS, tz_hi = k_hi / ZF_TS - 1;
  std::vector<int32_t> part[2];
  for (int32_t t : active) {
    const int tz = c->h_tile_origin[3 * (size_t)t + 2] / ZF_TS;
    if (tz > tz_lo && tz < tz_hi) part[0].push_back(t);
    else if (tz == tz_lo || tz == tz_hi) part[1].push_back(t);
  }
  for (int p = 0; p < 2; ++p) {
    if (c->d_active_part[p]) cudaFree(c->d_active_part[p]);
    c->d_active_part[p] = nullptr;
    int rc = dev_alloc(c, (void**)&c->d_active_part[p], std::max<size_t>(part[p].size(), 1) * sizeof(int32_t));
    if (rc) return rc;
    if (!part[p].empty())
      ZF_CUDA(cudaMemcpy(c->d_active_part[p], part[p].data(), part[p].size() * sizeof(int32_t),
                         cudaMemcpyHostToDevice));
    c->n_active_part[p] = (int)part[p].size();
  }
  c->slab_set = true;
  return ZF_OK;
}

int zf_lbm_step_part(zf_ctx* c, int part, int finish) { return zf_lbm_step_part_mf(c, part, finish, 0, 0); }

int zf_lbm_step_part_mf(zf_ctx* c, int part, int finish, int store_moments, int zero_bodyforce) {
  NEED_LATTICE("zf_lbm_step_part");
  if (!c->slab_set || part < 0 || part > 1) {
    set_error("zf_lbm_step_part: %s", c->slab_set ? "part is 0 (inner) or 1 (faces)" : "zf_set_slab first");
    return ZF_ERR_ARG;
  }
  int rc = lbm_launch_part(c, part, finish, store_moments, zero_bodyforce);
  if (rc == ZF_OK && finish) c->status.iter++;
  return rc;
}

int zf_lbm_steps(zf_ctx* c, int n) {
  NEED_LATTICE("zf_lbm_steps");
  for (int s = 0; s < n; ++s) {
    int rc = lbm_launch(c, s == n - 1, 0);
    if (rc) return rc;
    c->status.iter++;
  }
  return ZF_OK;
}

int zf_lbm_steps_timed(zf_ctx* c, int n, float* ms) {
  NEED_LATTICE("zf_lbm_steps_timed");
  if (!ms || n <= 0) return ZF_ERR_ARG;
  ZF_CUDA(cudaEventRecord(c->ev0, c->stream));
  for (int s = 0; s < n; ++s) {
    int rc = lbm_launch(c, 0, 0);
    if (rc) return rc;
    c->status.iter++;
  }
  ZF_CUDA(cudaEventRecord(c->ev1, c->stream));
  ZF_CUDA(cudaEventSynchronize(c->ev1));
  ZF_CUDA(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return ZF_OK;
}

int zf_lbm_step_mass(zf_ctx* c, int store_moments, int zero_bodyforce, double* mass) {
  NEED_LATTICE("zf_lbm_step_mass");
  if (!mass) return ZF_ERR_ARG;
  int rc = lbm_launch(c, store_moments, zero_bodyforce, mass);
  if (rc == ZF_OK) c->status.iter++;
  return rc;
}

int zf_lbm_step_mass_noalloc(zf_ctx* c, int store_moments, int zero_bodyforce, double* mass) {
  NEED_LATTICE("zf_lbm_step_mass_noalloc");
  if (!mass) return ZF_ERR_ARG;
  int rc = lbm_step_mass_noalloc(c, store_moments, zero_bodyforce, mass);
  if (rc == ZF_OK) c->status.iter++;
  return rc;
}

int zf_set_uniform_force(zf_ctx* c, const float* g3) {
  if (!c || !g3) return ZF_ERR_ARG;
  for (int a = 0; a < 3; ++a) c->p.g[a] = g3[a];
  return ZF_OK;
}

int zf_set_stream(zf_ctx* c, void* s) {
  if (!c) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  cudaStream_t ns = s ? (cudaStream_t)s : c->own_stream;
  if (ns != c->stream) {
    // order new work after what is already queued on the previous stream
    ZF_CUDA(cudaEventRecord(c->ev0, c->stream));
    ZF_CUDA(cudaStreamWaitEvent(ns, c->ev0, 0));
  }
  c->stream = ns;
  return ZF_OK;
}

int zf_mass(zf_ctx* c, int include_walls, double* mass) {
  NEED_LATTICE("zf_mass");
  if (!mass) return ZF_ERR_ARG;
  return lbm_mass(c, include_walls, mass);
}

// ---- z-slab halo exchange (no counterpart in the reference, which runs on one
// node): the populations that cross a z face are those of the 5 directions
// with e_z = dir of the listed points of one lattice plane.
int zf_plane_count(zf_ctx* c, int k, int32_t* n) {
  NEED_LATTICE("zf_plane_count");
  if (!n) return ZF_ERR_ARG;
  zf_ctx::PlaneSlots pl{};
  const int rc = lbm_plane_slots(c, k, &pl);
  if (rc) return rc;
  *n = pl.n;
  return ZF_OK;
}

int zf_plane_pack(zf_ctx* c, int k, int dir, void* dev_buf) {
  NEED_LATTICE("zf_plane_pack");
  if (dir != 1 && dir != -1) return ZF_ERR_ARG;
  return lbm_plane_copy(c, k, dir, dev_buf, true);
}

int zf_plane_unpack(zf_ctx* c, int k, int dir, const void* dev_buf) {
  NEED_LATTICE("zf_plane_unpack");
  if (dir != 1 && dir != -1) return ZF_ERR_ARG;
  return lbm_plane_copy(c, k, dir, const_cast<void*>(dev_buf), false);
}

}  // extern "C"

// Host side of the IB coupling: wall mesh upload, the lattice view the IB
// kernels read (population tiles plus auxiliary tiles that hold wall data
// only), buffers of the cell list and nucleus lists, and the coupled step.
#include <algorithm>
#include <cstring>
#include <vector>

#include "zf_internal.h"

using namespace zf;

namespace {

void free_list(std::vector<void*>& v) {
  for (void* p : v) cudaFree(p);
  v.clear();
}

template <typename T>
int dalloc(zf_ctx* c, std::vector<void*>& own, T** out, size_t n, const T* src = nullptr) {
  void* p = nullptr;
  int rc = dev_alloc(c, &p, (n ? n : 1) * sizeof(T));
  if (rc) return rc;
  own.push_back(p);
  if (src && n) ZF_CUDA(cudaMemcpyAsync(p, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  else ZF_CUDA(cudaMemsetAsync(p, 0, (n ? n : 1) * sizeof(T), c->stream));
  *out = (T*)p;
  return ZF_OK;
}

// Fills the lattice part of the IB view; W (may be null) adds wall data and
// auxiliary tiles for lattice points that carry a wall index or a void velocity.
int build_view(zf_ctx* c, const WallHost* W) {
  free_list(c->wall_allocs);
  IbArgs& a = c->ib;
  const zf_params& P = c->p;
  a.nx = P.nx;
  a.ny = P.ny;
  a.nz = P.nz;
  a.ntx = c->ntx;
  a.nty = c->nty;
  a.ntz = c->ntz;
  a.per_z = P.periodic[2];
  a.kmin = a.per_z ? -(1 << 29) : 2;
  a.kmax = a.per_z ? (1 << 29) : P.nz - 4;
  a.X0 = P.origin[0];
  a.Y0 = P.origin[1];
  a.Z0 = P.origin[2];
  a.DX = P.dx;
  a.LZ = P.periodic[2] ? (float)(P.nz * P.dx) : 0.f;
  a.own_k0 = -(1 << 30);
  a.own_k1 = 1 << 30;
  if (c->ib_slab) {  // one slab of a split lattice: see zf_set_ib_slab
    a.own_k0 = c->ib_k0;
    a.own_k1 = c->ib_k1;
    a.kmin = 0;
    a.kmax = P.nz - 1;
    a.LZ = (float)c->ib_lz;
  }
  a.mom = c->d_mom;
  a.force = c->d_force;
  a.ns = c->ns;
  a.vel_scale = (float)P.vel_scale;
  a.gamma_p = (float)P.gamma_p;
  a.force_scale = 1.0 / (P.unit_mass * P.bforce_scale);
  a.dt_stagger = P.dt * (double)P.stagger;
  a.vmax_remove = (float)P.vmax_remove;

  std::vector<int32_t> tmap = c->h_tile_map;
  int64_t n_all = c->n_pop_tiles;
  const int ntx = c->ntx, nty = c->nty;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  auto tile_of = [&](int i, int j, int k) {
    return ((int64_t)(k / ZF_TS) * nty + j / ZF_TS) * ntx + i / ZF_TS;
  };
  if (W) {
    for (int64_t p = 0; p < (int64_t)nx * ny * nz; ++p) {
      if (W->windex[p] <= 0) continue;
      const int i = (int)(p / ((int64_t)ny * nz)), j = (int)((p / nz) % ny), k = (int)(p % nz);
      const int64_t t = tile_of(i, j, k);
      if (tmap[t] < 0) tmap[t] = (int32_t)n_all++;
    }
  }
  c->n_all_tiles = n_all;
  const int64_t ns_all = n_all * ZF_TC;
  a.ns_all = ns_all;
  std::vector<uint8_t> code(ns_all, ZF_CODE_SOLID);
  ZF_CUDA(cudaMemcpy(code.data(), c->d_code, c->ns, cudaMemcpyDeviceToHost));
  std::vector<int32_t> windex(ns_all, 0);
  std::vector<float4> wnode(ns_all, make_float4(0.f, 0.f, 0.f, -1.f));
  std::vector<float> uvoid(3 * ns_all, 0.f);
  std::vector<uint8_t> twall(n_all, 0);
  if (W) {
    auto slot = [&](int64_t p) {
      const int i = (int)(p / ((int64_t)ny * nz)), j = (int)((p / nz) % ny), k = (int)(p % nz);
      return (int64_t)tmap[tile_of(i, j, k)] * ZF_TC + (i % ZF_TS) + ZF_TS * (j % ZF_TS) +
             ZF_TS * ZF_TS * (k % ZF_TS);
    };
    for (int64_t p = 0; p < (int64_t)nx * ny * nz; ++p) {
      if (W->windex[p] <= 0) continue;
      const int64_t s = slot(p);
      windex[s] = W->windex[p];
      const int m = W->windex[p] - 1;
      wnode[s] = make_float4(W->xyz[m], W->xyz[(size_t)W->nw + m], W->xyz[2 * (size_t)W->nw + m], W->rad[m]);
      twall[s / ZF_TC] = 1;
    }
    for (const VoidPoint& v : W->uvoid) {
      const int64_t s = slot(v.p);
      for (int d = 0; d < 3; ++d) uvoid[(size_t)d * ns_all + s] = v.u[d];
    }
  }
  auto& own = c->wall_allocs;
  int rc;
  // the tile map of the LBM tables keeps population tiles only; the IB view
  // gets its own map that also names the auxiliary tiles
  if ((rc = dalloc<int32_t>(c, own, const_cast<int32_t**>(&a.tile_map), tmap.size(), tmap.data())))
    return rc;
  if ((rc = dalloc<uint8_t>(c, own, const_cast<uint8_t**>(&a.code), code.size(), code.data()))) return rc;
  if ((rc = dalloc<int32_t>(c, own, const_cast<int32_t**>(&a.windex), windex.size(), windex.data())))
    return rc;
  if ((rc = dalloc<float4>(c, own, const_cast<float4**>(&a.wnode), wnode.size(), wnode.data()))) return rc;
  if ((rc = dalloc<float>(c, own, const_cast<float**>(&a.uvoid), uvoid.size(), uvoid.data()))) return rc;
  if ((rc = dalloc<uint8_t>(c, own, const_cast<uint8_t**>(&a.tile_wall), twall.size(), twall.data())))
    return rc;
  if (W) {
    a.nw = W->nw;
    a.mt = W->mt;
    a.wcap = W->cap;
    if ((rc = dalloc<float>(c, own, const_cast<float**>(&a.wxyz), W->xyz.size(), W->xyz.data()))) return rc;
    if ((rc = dalloc<int32_t>(c, own, const_cast<int32_t**>(&a.wtri), W->tri.size(), W->tri.data()))) return rc;
    if ((rc = dalloc<float>(c, own, const_cast<float**>(&a.wnrm), W->nrm.size(), W->nrm.data()))) return rc;
    if ((rc = dalloc<float>(c, own, const_cast<float**>(&a.wcen), W->cen.size(), W->cen.data()))) return rc;
    if ((rc = dalloc<int32_t>(c, own, const_cast<int32_t**>(&a.wntri), W->ntri.size(), W->ntri.data())))
      return rc;
    if ((rc = dalloc<float>(c, own, const_cast<float**>(&a.wrad), W->rad.size(), W->rad.data()))) return rc;
    if ((rc = dalloc<int32_t>(c, own, const_cast<int32_t**>(&a.wcand_off), W->cand_off.size(),
                              W->cand_off.data())))
      return rc;
    if ((rc = dalloc<float4>(c, own, const_cast<float4**>(&a.wcand), W->cand.size(), W->cand.data()))) return rc;
    if ((rc = dalloc<float>(c, own, const_cast<float**>(&a.wnnrm), W->nnrm.size(), W->nnrm.data())))
      return rc;
    if ((rc = wall_rel_build(c, own))) return rc;
  } else {
    a.nw = a.mt = a.wcap = 0;
    a.wxyz = a.wnrm = a.wcen = a.wrad = a.wnnrm = nullptr;
    a.wcand_off = nullptr;
    a.wcand = nullptr;
    a.wrel_cnt = a.wrel_off = a.wrel = nullptr;
    a.wtri = a.wntri = nullptr;
  }
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

// cell list and nucleus list buffers, sized by the lattice and the cells
int ib_buffers(zf_ctx* c) {
  free_list(c->ib_allocs);
  IbArgs& a = c->ib;
  const CellArgs& cl = c->cells;
  const int64_t ntri = (int64_t)cl.n_cells * cl.nt;
  const int64_t nscan = c->ns + 1;
  const int64_t nb = (nscan + 1023) / 1024;
  // [off: ns+1][counts: ns+1][tri_bin: ntri][bsum: nb+1]
  int32_t* buf = nullptr;
  int rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &buf, 2 * nscan + ntri + nb + 1))) return rc;
  a.bin_off = buf;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, const_cast<int32_t**>(&a.bin_tri), ntri))) return rc;
  if ((rc = dalloc<float4>(c, c->ib_allocs, &a.bin_rec, 2 * ntri))) return rc;
  if ((rc = dalloc<float4>(c, c->ib_allocs, &a.bin_v, 3 * ntri))) return rc;
  if ((rc = dalloc<uint8_t>(c, c->ib_allocs, &a.bin_kk, ntri))) return rc;
  // node-tile lists
  const int64_t nnodes = (int64_t)cl.n_cells * (cl.nn + cl.nnn);
  a.ngrid = (int64_t)c->ntx * c->nty * c->ntz;
  const int64_t ng1 = a.ngrid + 1;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.node_gt, nnodes))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.node_cnt, ng1))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.node_off, ng1))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.node_sorted, nnodes))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.wall_walk, nnodes))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.wall_walk_ctr, 4))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.wall_tri, nnodes))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.tile_list, std::min(a.ngrid, nnodes)))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.tile_ctr, 4))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.node_bsum, (ng1 + 1023) / 1024 + 1))) return rc;
  a.nuc_cap = std::max(1, c->p.nuc_list_max);
  const int64_t nnuc = (int64_t)cl.n_cells * cl.nnn;
  if ((rc = dalloc<uint16_t>(c, c->ib_allocs, &a.nuc_list, nnuc * a.nuc_cap))) return rc;
  if ((rc = dalloc<int32_t>(c, c->ib_allocs, &a.nuc_cnt, nnuc))) return rc;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

}  // namespace

namespace zf {

// (Re)builds what the IB kernels need once lattice and cells exist.
int ib_prepare(zf_ctx* c) {
  if (!c->lattice_set) return ZF_OK;
  int rc;
  if (!c->wall_set && c->wall_allocs.empty())
    if ((rc = build_view(c, nullptr))) return rc;
  if (c->cells_set)
    if ((rc = ib_buffers(c))) return rc;
  c->nuc_lists_valid = false;
  c->node_tiles_valid = false;
  return ZF_OK;
}

void ib_free(zf_ctx* c) {
  free_list(c->wall_allocs);
  free_list(c->ib_allocs);
  c->wall_set = false;
}

}  // namespace zf

#define NEED_IB(fn)                                                    \
  if (!c) return ZF_ERR_ARG;                                           \
  if (!c->lattice_set || !c->cells_set) {                              \
    set_error(fn ": lattice and cells must be set");                   \
    return ZF_ERR_STATE;                                               \
  }                                                                    \
  ZF_CUDA(cudaSetDevice(c->device));                                   \
  if (c->ib_allocs.empty()) {                                          \
    int rc_ = ib_prepare(c);                                           \
    if (rc_) return rc_;                                               \
  }

extern "C" {

int zf_set_wall(zf_ctx* c, int n_node_w, const float* xyz, int n_tri_w, const int32_t* tri,
                const float* normals) {
  if (!c || n_node_w <= 0 || n_tri_w <= 0 || !xyz || !tri || !normals) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_set_wall: lattice not set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  WallHost W;
  int rc = wall_build(c, n_node_w, xyz, n_tri_w, tri, normals, W);
  if (rc) return rc;
  if ((rc = build_view(c, &W))) return rc;
  c->wall_set = true;
  return ZF_OK;
}

int zf_get_wall_index(zf_ctx* c, int32_t* windex, float* uvoid) {
  if (!c) return ZF_ERR_ARG;
  if (!c->lattice_set || c->wall_allocs.empty()) {
    set_error("zf_get_wall_index: lattice and wall must be set");
    return ZF_ERR_STATE;
  }
  // dense [nx][ny][nz] outputs from the tiled view
  const IbArgs& a = c->ib;
  std::vector<int32_t> wi(a.ns_all), tm((size_t)c->ntx * c->nty * c->ntz);
  std::vector<float> uv(3 * a.ns_all);
  ZF_CUDA(cudaMemcpy(wi.data(), a.windex, wi.size() * 4, cudaMemcpyDeviceToHost));
  ZF_CUDA(cudaMemcpy(uv.data(), a.uvoid, uv.size() * 4, cudaMemcpyDeviceToHost));
  ZF_CUDA(cudaMemcpy(tm.data(), a.tile_map, tm.size() * 4, cudaMemcpyDeviceToHost));
  const int nx = c->p.nx, ny = c->p.ny, nz = c->p.nz;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int64_t p = ((int64_t)i * ny + j) * nz + k;
        const int t = tm[((int64_t)(k / 4) * c->nty + j / 4) * c->ntx + i / 4];
        const int64_t s = t < 0 ? -1 : (int64_t)t * 64 + (i % 4) + 4 * (j % 4) + 16 * (k % 4);
        if (windex) windex[p] = s < 0 ? 0 : wi[s];
        if (uvoid)
          for (int d = 0; d < 3; ++d) uvoid[(size_t)d * nx * ny * nz + p] = s < 0 ? 0.f : uv[(size_t)d * a.ns_all + s];
      }
  return ZF_OK;
}

int zf_wss(zf_ctx* c, const float* node_normals, double pgauge, float* wss, float* pressure,
           int32_t* valid) {
  if (!c || !wss) return ZF_ERR_ARG;
  if (!c->lattice_set || c->wall_allocs.empty() || c->ib.nw == 0) {
    set_error("zf_wss: lattice and wall must be set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  const size_t nw = (size_t)c->ib.nw;
  // [normals 3 nw][wss 3 nw][pressure nw][valid nw]
  void* buf = nullptr;
  int rc = dev_alloc(c, &buf, 8 * nw * sizeof(float));
  if (rc) return rc;
  float* d_nrm = (float*)buf;
  float* d_wss = d_nrm + 3 * nw;
  float* d_press = d_wss + 3 * nw;
  int32_t* d_valid = (int32_t*)(d_press + nw);
  cudaError_t e = cudaSuccess;
  if (node_normals)
    e = cudaMemcpyAsync(d_nrm, node_normals, 3 * nw * sizeof(float), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) rc = wss_launch(c, node_normals ? d_nrm : nullptr, pgauge, d_wss, d_press, d_valid);
  if (e == cudaSuccess && rc == ZF_OK)
    e = cudaMemcpyAsync(wss, d_wss, 3 * nw * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && rc == ZF_OK && pressure)
    e = cudaMemcpyAsync(pressure, d_press, nw * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && rc == ZF_OK && valid)
    e = cudaMemcpyAsync(valid, d_valid, nw * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(buf);
  c->device_bytes -= (int64_t)(8 * nw * sizeof(float));
  ZF_CUDA(e);
  return rc;
}

int zf_get_cell_list_counts(zf_ctx* c, int32_t* counts) {
  if (!c || !counts) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_get_cell_list_counts: lattice not set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  const int64_t n = c->n_listed;
  for (int64_t l = 0; l < n; ++l) counts[l] = 0;
  if (!c->cells_set || c->ib_allocs.empty() || !c->ib.bin_off) return ZF_OK;
  std::vector<int32_t> off((size_t)c->ns + 1), slot((size_t)n);
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  ZF_CUDA(cudaMemcpy(off.data(), c->ib.bin_off, off.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
  ZF_CUDA(cudaMemcpy(slot.data(), c->d_dom_slot, slot.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
  for (int64_t l = 0; l < n; ++l) {
    const int64_t s = slot[(size_t)l], cc = s & 63;
    // the cell list is keyed with z fastest inside a tile (k_bin_assign)
    const int64_t key = (s & ~(int64_t)63) | (((cc >> 4) & 3) + 4 * ((cc >> 2) & 3) + 16 * (cc & 3));
    counts[l] = off[(size_t)key + 1] - off[(size_t)key];
  }
  return ZF_OK;
}

int zf_set_ib_slab(zf_ctx* c, int k_lo, int k_hi, double lz) {
  if (!c) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_set_ib_slab: lattice not set");
    return ZF_ERR_STATE;
  }
  if (c->p.periodic[2] || k_lo < 8 || k_hi > c->p.nz - 8 || k_hi <= k_lo || lz < 0.0) {
    set_error("zf_set_ib_slab: needs a lattice not periodic in z, owned planes [%d, %d) with 8 planes of halo "
              "on either side (nz %d), lz >= 0",
              k_lo, k_hi, c->p.nz);
    return ZF_ERR_ARG;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  c->ib_slab = true;
  c->ib_k0 = k_lo;
  c->ib_k1 = k_hi;
  c->ib_lz = lz;
  IbArgs& a = c->ib;
  a.own_k0 = k_lo;
  a.own_k1 = k_hi;
  a.kmin = 0;
  a.kmax = c->p.nz - 1;
  a.LZ = (float)lz;
  c->node_tiles_valid = false;
  return ZF_OK;
}

int zf_cells_reduce_size(zf_ctx* c, int64_t* n) {
  if (!c || !n) return ZF_ERR_ARG;
  *n = c->cells_set ? 3 * (int64_t)c->cells.n_cells * (2 * c->cells.nn + c->cells.nnn) : 0;
  return ZF_OK;
}

int zf_cells_reduce_buffer(zf_ctx* c, int dir, void* dev_buf) {
  if (!c || (dir != 0 && dir != 1) || !dev_buf) return ZF_ERR_ARG;
  if (!c->cells_set) {
    set_error("zf_cells_reduce_buffer: cells not set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  return ib_kin_buffer_launch(c, (double*)dev_buf, dir);
}

int zf_ibm_interp(zf_ctx* c) {
  NEED_IB("zf_ibm_interp");
  return ib_interp_launch(c);
}

int zf_nuc_memb_repulsion(zf_ctx* c, int rebuild_lists) {
  NEED_IB("zf_nuc_memb_repulsion");
  const int rb = rebuild_lists || !c->nuc_lists_valid;
  int rc = ib_nuc_memb_launch(c, rb);
  if (rc == ZF_OK) c->nuc_lists_valid = true;
  return rc;
}

int zf_rbc_rbc_repulsion(zf_ctx* c) {
  NEED_IB("zf_rbc_rbc_repulsion");
  int rc = ib_bins_launch(c);
  if (rc) return rc;
  return ib_rbc_rbc_launch(c);
}

int zf_ibm_spread(zf_ctx* c) {
  NEED_IB("zf_ibm_spread");
  return ib_spread_launch(c);
}

int zf_update_positions(zf_ctx* c) {
  NEED_IB("zf_update_positions");
  return ib_update_launch(c);
}

// One or more iterations of the reference time loop, ZebraflowWT.c:5646-12190.
static int step_impl(zf_ctx* c, int nsteps, double* mass_last) {
  if (!c) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("zf_step: lattice not set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  const bool cells = c->cells_set && c->cells.n_cells > 0;
  if (cells && c->ib_allocs.empty()) {
    int rc = ib_prepare(c);
    if (rc) return rc;
  }
  // LBM profiling: one event pair around each run of consecutive plain LBM
  // steps (events around single launches would also time the host's enqueue)
  auto close_run = [&]() -> int {
    if (!c->prof_open) return ZF_OK;
    ZF_CUDA(cudaEventRecord(c->prof_ev[2 * c->prof_lbm + 1], c->stream));
    c->prof_run_n.push_back(c->prof_open_n);
    c->prof_lbm++;
    c->prof_open = false;
    return ZF_OK;
  };
  for (int s = 0; s < nsteps; ++s) {
    const int64_t iter = c->status.iter + 1;
    const bool membrane = cells && (iter % c->p.stagger == 0);  // RBCSOLVERFLAG, :5650-5652
    const bool last = s == nsteps - 1;
    int rc;
    if (membrane && (rc = close_run())) return rc;
    // on profiled membrane iterations an event precedes each stage and one
    // follows the last: [forces][LBM][interp][nucleus][bins][RBC-RBC][spread][update]
    const bool pm = c->profiling && membrane && c->prof_mem < c->prof_cap;
    auto mark = [&](int k) -> int {
      if (pm) ZF_CUDA(cudaEventRecord(c->prof_ev[2 * (size_t)c->prof_cap + ZF_PROF_MARKS * (size_t)c->prof_mem + k],
                                      c->stream));
      return ZF_OK;
    };
    if ((rc = mark(0))) return rc;
    if (membrane && (rc = cells_membrane_launch(c))) return rc;
    if ((rc = mark(1))) return rc;
    if (!membrane && c->profiling && !c->prof_open && c->prof_lbm < c->prof_cap) {
      ZF_CUDA(cudaEventRecord(c->prof_ev[2 * c->prof_lbm], c->stream));
      c->prof_open = true;
      c->prof_open_n = 0;
    }
    if ((rc = lbm_launch(c, membrane, membrane, (last && mass_last) ? mass_last : nullptr)))
      return rc;
    if (c->prof_open) c->prof_open_n++;
    if (membrane) {
      const bool rebuild = !c->nuc_lists_valid || (iter % c->p.nuc_list_period == 0);
      if ((rc = mark(2)) || (rc = ib_interp_launch(c))) return rc;
      if ((rc = mark(3)) || (rc = ib_nuc_memb_launch(c, rebuild))) return rc;
      c->nuc_lists_valid = true;
      if ((rc = mark(4)) || (rc = ib_bins_launch(c))) return rc;
      if ((rc = mark(5)) || (rc = ib_rbc_rbc_launch(c))) return rc;
      if ((rc = mark(6)) || (rc = ib_spread_launch(c))) return rc;
      if ((rc = mark(7)) || (rc = ib_update_launch(c))) return rc;
      if ((rc = mark(8))) return rc;
      if (pm) c->prof_mem++;
    }
    c->status.iter = iter;
  }
  return close_run();
}

int zf_step(zf_ctx* c, int nsteps) { return step_impl(c, nsteps, nullptr); }

int zf_step_mass(zf_ctx* c, double* mass) {
  if (!mass) return ZF_ERR_ARG;
  return step_impl(c, 1, mass);
}

int zf_launch_count(zf_ctx* c, int64_t* n) {
  if (!c || !n) return ZF_ERR_ARG;
  *n = c->launches;
  return ZF_OK;
}

int zf_profile(zf_ctx* c, int enable, int capacity) {
  if (!c) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  c->prof_ev.clear();
  c->prof_cap = c->prof_lbm = c->prof_mem = 0;
  c->prof_open = false;
  c->prof_run_n.clear();
  c->profiling = enable != 0;
  if (!enable) return ZF_OK;
  c->prof_cap = capacity > 0 ? capacity : 4096;
  // [LBM run pairs: 2 per run][membrane iterations: ZF_PROF_MARKS per block]
  c->prof_ev.resize((2 + ZF_PROF_MARKS) * (size_t)c->prof_cap);
  for (auto& e : c->prof_ev) ZF_CUDA(cudaEventCreate(&e));
  return ZF_OK;
}

// Summed device time (ms) of each stage of the profiled membrane iterations.
static int stage_times(zf_ctx* c, float* st) {
  for (int k = 0; k < ZF_PROF_STAGES; ++k) st[k] = 0.f;
  for (int i = 0; i < c->prof_mem; ++i) {
    const size_t b = 2 * (size_t)c->prof_cap + ZF_PROF_MARKS * (size_t)i;
    for (int k = 0; k < ZF_PROF_STAGES; ++k) {
      float ms = 0.f;
      ZF_CUDA(cudaEventElapsedTime(&ms, c->prof_ev[b + k], c->prof_ev[b + k + 1]));
      st[k] += ms;
    }
  }
  return ZF_OK;
}

int zf_profile_read(zf_ctx* c, float* lbm_ms, int* lbm_count, float* membrane_ms, int* membrane_count) {
  if (!c) return ZF_ERR_ARG;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  float tl = 0.f;
  int runs_n = 0;
  for (int i = 0; i < c->prof_lbm; ++i) {
    runs_n += c->prof_run_n[i];
    float ms = 0.f;
    ZF_CUDA(cudaEventElapsedTime(&ms, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]));
    tl += ms;
  }
  float st[ZF_PROF_STAGES];
  int rc = stage_times(c, st);
  if (rc) return rc;
  float tm = 0.f;
  for (int k = 0; k < ZF_PROF_STAGES; ++k)
    if (k != 1) tm += st[k];  // the membrane iteration's own LBM launch is not part of the block
  if (lbm_ms) *lbm_ms = tl;
  if (lbm_count) *lbm_count = runs_n;
  if (membrane_ms) *membrane_ms = tm;
  if (membrane_count) *membrane_count = c->prof_mem;
  return ZF_OK;
}

int zf_profile_stages(zf_ctx* c, float* stage_ms, int* blocks) {
  if (!c || !stage_ms) return ZF_ERR_ARG;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  int rc = stage_times(c, stage_ms);
  if (rc) return rc;
  if (blocks) *blocks = c->prof_mem;
  return ZF_OK;
}

int zf_step_timed(zf_ctx* c, int nsteps, float* ms) {
  if (!c || !ms) return ZF_ERR_ARG;
  ZF_CUDA(cudaEventRecord(c->ev0, c->stream));
  int rc = zf_step(c, nsteps);
  if (rc) return rc;
  ZF_CUDA(cudaEventRecord(c->ev1, c->stream));
  ZF_CUDA(cudaEventSynchronize(c->ev1));
  ZF_CUDA(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return ZF_OK;
}

int zf_iteration(zf_ctx* c, int64_t* iter) {
  if (!c || !iter) return ZF_ERR_ARG;
  *iter = c->status.iter;
  return ZF_OK;
}

int zf_set_iteration(zf_ctx* c, int64_t iter) {
  if (!c || iter < 0) return ZF_ERR_ARG;
  c->status.iter = iter;
  return ZF_OK;
}

}  // extern "C"

// Hand-written adjoint of the coupled step for a wall-shear-stress objective
// or a flux-split objective, with checkpointing and recomputation
// (zf_wss_objective / zf_wss_adjoint, zf_flux_objective / zf_flux_adjoint).
//
// The differentiated forward starts from the context's populations f_0 and
// its cells, whose positions stay fixed over the window:
//   BODYFORCE = S(x) F_total(x; Es, kb) + F_b           (spreading :10737-10990
//                                                        of the membrane forces
//                                                        :5704-7535, plus a field)
//   f_t = LBM(f_{t-1}; tau, BODYFORCE),   t = 1..N       (:6100-6145, bounce-back)
//   J = 1/(t1-t0+1) sum_{t=t0..t1} 1/|P| sum_{m in P} |WSS_m(f_t)|   (W:319-369)
//   or J = 1/(t1-t0+1) sum_{t=t0..t1} Q_0(f_t) / (Q_0(f_t) + Q_1(f_t)),
//      Q_s = sum over the points of set s of U.n_s (outlet fluxes)
// Gradients: dJ/dF_b (per listed point, the same as dJ/dBODYFORCE), dJ/dtau,
// and dJ/dEs, dJ/dkb through the membrane forces: F_total = Es A(x) +
// kb B(x) + C(x) at fixed positions (the springs' coefficients are
// proportional to Es at the calibration's fixed point, bending is linear in
// kb), so dJ/dEs = sum_nodes (S^T dJ/dBODYFORCE) . A with A from one force
// evaluation at 2 Es, and likewise for kb.
//
// Populations of every K-th step are kept; the backward pass recomputes each
// segment of K steps from its checkpoint, keeps its states, and walks it
// backwards with the adjoint kernel.  With 16-bit population storage the
// forward and its recomputation round identically (step t always draws the
// same stochastic-rounding bits), and the adjoint linearises the fp32
// arithmetic around the stored states: the rounding itself is passed through
// as the identity.
#include <algorithm>
#include <cmath>
#include <vector>

#include "zf_internal.h"

using namespace zf;

namespace {

struct DevBuf {
  zf_ctx* c = nullptr;
  void* p = nullptr;
  size_t bytes = 0;
  int alloc(zf_ctx* ctx, size_t b) {
    c = ctx;
    bytes = b;
    return dev_alloc(ctx, &p, b);
  }
  ~DevBuf() {
    if (p) {
      cudaFree(p);
      c->device_bytes -= (int64_t)bytes;
    }
  }
};

enum Kind { kWss, kFlux };

struct Setup {
  zf_ctx* c = nullptr;
  Kind kind = kWss;
  size_t pop_bytes = 0;        // one population state
  uint32_t step0 = 0;          // step number of the first forward step
  double weight = 0.0;         // WSS: 1 / (window x patch size); flux: 1 / window
  DevBuf nrm, patch, acc;      // WSS normals [3][nw], patch ids; FP64 accumulator
  DevBuf U;                    // velocities at the compact points [3][nu]
  DevBuf set, q;               // flux: set of each compact point, the two fluxes
  float nrm6[6] = {};          // flux: the two sets' unit normals
  PatchStencil ps;             // the objective's compact points (and WSS stencils)
  std::vector<std::pair<void*, size_t>> ps_bufs;
  std::vector<float> bf_save;  // BODYFORCE at entry (listed order)
  ~Setup() {
    for (auto& b : ps_bufs) {
      cudaFree(b.first);
      c->device_bytes -= (int64_t)b.second;
    }
  }
};

// what both objectives need: the window, the flow model, a lattice
int check_common(zf_ctx* c, int nsteps, int t0, int t1) {
  if (!c || nsteps < 1 || t0 < 1 || t1 < t0 || t1 > nsteps) return ZF_ERR_ARG;
  if (!c->lattice_set) {
    set_error("adjoint: the lattice must be set");
    return ZF_ERR_STATE;
  }
  if (c->p.wall_mode != ZF_WALL_HALFWAY_BB || c->p.tau_from_phase) {
    set_error("adjoint: needs halfway bounce-back walls and a uniform tau");
    return ZF_ERR_ARG;
  }
  return ZF_OK;
}

int check_args(zf_ctx* c, int nsteps, int t0, int t1, const int32_t* patch, int n_patch) {
  int rc = check_common(c, nsteps, t0, t1);
  if (rc) return rc;
  if (!patch || n_patch < 1) return ZF_ERR_ARG;
  if (c->wall_allocs.empty() || c->ib.nw == 0) {
    set_error("WSS objective: lattice and wall must be set");
    return ZF_ERR_STATE;
  }
  for (int i = 0; i < n_patch; ++i)
    if (patch[i] < 0 || patch[i] >= c->ib.nw) {
      set_error("WSS objective: patch node %d out of range", patch[i]);
      return ZF_ERR_ARG;
    }
  return ZF_OK;
}

// BODYFORCE := S F_total(x) + F_b, saved first; the accumulator and velocities
int setup_common(zf_ctx* c, const float* fb, Setup& S) {
  const size_t esz = c->p.storage == ZF_STORE_F32 || c->p.storage == ZF_STORE_F32_DEV ? 4 : 2;
  const size_t nl = (size_t)c->n_listed;
  S.pop_bytes = (size_t)ZF_Q * c->ns * esz;
  S.step0 = (uint32_t)c->status.iter;
  int rc;
  if ((rc = S.acc.alloc(c, sizeof(double)))) return rc;
  if ((rc = S.U.alloc(c, 3 * (size_t)std::max(S.ps.nu, 1) * sizeof(float)))) return rc;
  S.bf_save.resize(3 * nl);
  if ((rc = lbm_gather_listed(c, c->d_force, 3, S.bf_save.data()))) return rc;
  ZF_CUDA(cudaMemsetAsync(c->d_force, 0, 3 * c->ns * sizeof(float), c->stream));
  if (c->cells_set && c->cells.n_cells > 0) {
    if (c->ib_allocs.empty() && (rc = ib_prepare(c))) return rc;
    if ((rc = cells_membrane_launch(c))) return rc;  // forces at the current positions
    if ((rc = ib_spread_launch(c))) return rc;       // BODYFORCE += S F_total
  }
  if (fb) {
    std::vector<float> bf(3 * nl);
    if ((rc = lbm_gather_listed(c, c->d_force, 3, bf.data()))) return rc;
    for (size_t i = 0; i < bf.size(); ++i) bf[i] += fb[i];
    if ((rc = lbm_scatter_listed(c, bf.data(), 3, c->d_force))) return rc;
  }
  return ZF_OK;
}

// WSS objective: normals, patch and its stencils
int setup(zf_ctx* c, int t0, int t1, const int32_t* patch, int n_patch, const float* normals,
          const float* fb, Setup& S) {
  S.c = c;
  S.kind = kWss;
  S.weight = 1.0 / ((double)(t1 - t0 + 1) * n_patch);
  const size_t nw = (size_t)c->ib.nw;
  int rc;
  if ((rc = S.nrm.alloc(c, 3 * nw * sizeof(float)))) return rc;
  if ((rc = S.patch.alloc(c, (size_t)n_patch * sizeof(int32_t)))) return rc;
  ZF_CUDA(cudaMemcpyAsync(S.nrm.p, normals ? normals : c->ib.wnnrm, 3 * nw * sizeof(float),
                          normals ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->stream));
  ZF_CUDA(cudaMemcpyAsync(S.patch.p, patch, (size_t)n_patch * sizeof(int32_t), cudaMemcpyHostToDevice,
                          c->stream));
  if ((rc = wss_patch_stencil(c, (const float*)S.nrm.p, (const int32_t*)S.patch.p, n_patch, S.ps, S.ps_bufs)))
    return rc;
  return setup_common(c, fb, S);
}

// flux objective: the two point sets (listed ids, fluid points only, disjoint)
// as compact points with their set, and the normals
int setup_flux(zf_ctx* c, int t0, int t1, const int32_t* pts0, int n0, const float* nrm0, const int32_t* pts1,
               int n1, const float* nrm1, const float* fb, Setup& S) {
  S.c = c;
  S.kind = kFlux;
  S.weight = 1.0 / (double)(t1 - t0 + 1);
  if (!pts0 || !pts1 || n0 < 1 || n1 < 1 || !nrm0 || !nrm1) return ZF_ERR_ARG;
  for (int v = 0; v < 3; ++v) {
    S.nrm6[v] = nrm0[v];
    S.nrm6[3 + v] = nrm1[v];
  }
  const int64_t nl = c->n_listed;
  std::vector<std::pair<int32_t, uint8_t>> pts;
  pts.reserve((size_t)n0 + n1);
  for (int s = 0; s < 2; ++s) {
    const int32_t* p = s ? pts1 : pts0;
    const int n = s ? n1 : n0;
    for (int i = 0; i < n; ++i) {
      const int32_t l = p[i];
      if (l < 0 || l >= nl) {
        set_error("flux objective: point %d out of range", l);
        return ZF_ERR_ARG;
      }
      const int64_t d = ((int64_t)c->domlist[3 * l] * c->p.ny + c->domlist[3 * l + 1]) * c->p.nz +
                        c->domlist[3 * l + 2];
      const int32_t code = c->b_index[d];
      if (code < 1 || code > 9) {
        set_error("flux objective: point %d is not a fluid point", l);
        return ZF_ERR_ARG;
      }
      pts.emplace_back(l, (uint8_t)s);
    }
  }
  std::sort(pts.begin(), pts.end());
  for (size_t i = 1; i < pts.size(); ++i)
    if (pts[i].first == pts[i - 1].first) {
      set_error("flux objective: point %d listed twice", pts[i].first);
      return ZF_ERR_ARG;
    }
  // slots of the listed points, in the sorted order
  std::vector<int32_t> dom(nl);
  ZF_CUDA(cudaMemcpyAsync(dom.data(), c->d_dom_slot, nl * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  const int nu = (int)pts.size();
  std::vector<int32_t> uslot(nu);
  std::vector<uint8_t> set(nu);
  for (int u = 0; u < nu; ++u) {
    uslot[u] = dom[pts[u].first];
    set[u] = pts[u].second;
  }
  int rc;
  void* d_us = nullptr;
  if ((rc = dev_alloc(c, &d_us, (size_t)nu * sizeof(int32_t)))) return rc;
  S.ps_bufs.emplace_back(d_us, (size_t)nu * sizeof(int32_t));
  if ((rc = S.set.alloc(c, (size_t)nu)) || (rc = S.q.alloc(c, 2 * sizeof(double)))) return rc;
  ZF_CUDA(cudaMemcpyAsync(d_us, uslot.data(), (size_t)nu * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  ZF_CUDA(cudaMemcpyAsync(S.set.p, set.data(), (size_t)nu, cudaMemcpyHostToDevice, c->stream));
  S.ps = PatchStencil{};
  S.ps.nu = nu;
  S.ps.uslot = (const int32_t*)d_us;
  return setup_common(c, fb, S);
}

// BODYFORCE back as it was, and the moment planes of the context's populations
int restore(zf_ctx* c, Setup& S) {
  int rc = lbm_scatter_listed(c, S.bf_save.data(), 3, c->d_force);
  if (rc) return rc;
  if ((rc = lbm_moments_launch(c))) return rc;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

// J of the state f (adds into S.acc)
int objective_of(zf_ctx* c, const void* f, Setup& S) {
  int rc = lbm_moments_at(c, f, S.ps, (float*)S.U.p);
  if (rc) return rc;
  if (S.kind == kFlux)
    return flux_objective_launch(c, S.ps, (const uint8_t*)S.set.p, S.nrm6, (const float*)S.U.p, S.weight,
                                 (double*)S.q.p, (double*)S.acc.p);
  return wss_patch_launch(c, S.ps, (const float*)S.nrm.p, (const float*)S.U.p, S.weight, (double*)S.acc.p);
}

// lam += dJ_t/df_t for the state f of a step in the window (gU: scratch of
// 3 nu floats, zero on entry and on return)
int objective_seed(zf_ctx* c, const void* f, Setup& S, float* gU, float* lam) {
  int rc = lbm_moments_at(c, f, S.ps, (float*)S.U.p);
  if (rc) return rc;
  if (S.kind == kFlux)
    rc = flux_adj_launch(c, S.ps, (const uint8_t*)S.set.p, S.nrm6, (const float*)S.U.p, S.weight, (double*)S.q.p,
                         gU);
  else
    rc = wss_patch_adj_launch(c, S.ps, (const float*)S.nrm.p, (const float*)S.U.p, S.weight, gU);
  if (rc) return rc;
  return lbm_seed_at(c, f, S.ps, gU, lam);
}

// the forward from the context's populations: J over the window
int run_objective(zf_ctx* c, int nsteps, int t0, int t1, Setup& S, double* J) {
  int rc;
  DevBuf a, b;
  if ((rc = a.alloc(c, S.pop_bytes)) || (rc = b.alloc(c, S.pop_bytes))) return rc;
  ZF_CUDA(cudaMemcpyAsync(a.p, c->d_f[c->cur], S.pop_bytes, cudaMemcpyDeviceToDevice, c->stream));
  ZF_CUDA(cudaMemsetAsync(S.acc.p, 0, sizeof(double), c->stream));
  void* fin = a.p;
  void* fout = b.p;
  for (int t = 1; t <= nsteps; ++t) {
    if ((rc = lbm_step_buffers(c, fin, fout, S.step0 + (uint32_t)(t - 1)))) return rc;
    std::swap(fin, fout);
    if (t >= t0 && t <= t1 && (rc = objective_of(c, fin, S))) return rc;
  }
  ZF_CUDA(cudaMemcpyAsync(J, S.acc.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return restore(c, S);
}

int run_adjoint(zf_ctx* c, int nsteps, int t0, int t1, int K, Setup& S, double* J, float* dJ_dfb,
                double* dJ_dtau, double* dJ_dEs, double* dJ_dkb);
bool cells_active(zf_ctx* c);
int run_objective_coupled(zf_ctx* c, int nsteps, int t0, int t1, const float* fb, Setup& S, double* J);
int run_adjoint_coupled(zf_ctx* c, int nsteps, int t0, int t1, int K, const float* fb, Setup& S, double* J,
                        float* dJ_dfb, double* dJ_dtau, double* dJ_dEs, double* dJ_dkb);

// the forward the context's adjoint mode names
int objective(zf_ctx* c, int nsteps, int t0, int t1, const float* fb, Setup& S, double* J) {
  if (c->adj_move_cells && cells_active(c)) return run_objective_coupled(c, nsteps, t0, t1, fb, S, J);
  return run_objective(c, nsteps, t0, t1, S, J);
}
int adjoint(zf_ctx* c, int nsteps, int t0, int t1, int K, const float* fb, Setup& S, double* J, float* dJ_dfb,
            double* dJ_dtau, double* dJ_dEs, double* dJ_dkb) {
  if (c->adj_move_cells && cells_active(c))
    return run_adjoint_coupled(c, nsteps, t0, t1, K, fb, S, J, dJ_dfb, dJ_dtau, dJ_dEs, dJ_dkb);
  return run_adjoint(c, nsteps, t0, t1, K, S, J, dJ_dfb, dJ_dtau, dJ_dEs, dJ_dkb);
}

}  // namespace

extern "C" {

int zf_wss_objective(zf_ctx* c, int nsteps, int t0, int t1, const int32_t* patch, int n_patch,
                     const float* node_normals, const float* fb, double* J) {
  int rc = check_args(c, nsteps, t0, t1, patch, n_patch);
  if (rc) return rc;
  if (!J) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  Setup S;
  if ((rc = setup(c, t0, t1, patch, n_patch, node_normals, fb, S))) return rc;
  return objective(c, nsteps, t0, t1, fb, S, J);
}

int zf_wss_adjoint(zf_ctx* c, int nsteps, int t0, int t1, const int32_t* patch, int n_patch,
                   const float* node_normals, const float* fb, int checkpoint_interval, double* J,
                   float* dJ_dfb, double* dJ_dtau, double* dJ_dEs, double* dJ_dkb) {
  int rc = check_args(c, nsteps, t0, t1, patch, n_patch);
  if (rc) return rc;
  if (checkpoint_interval < 1) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  Setup S;
  if ((rc = setup(c, t0, t1, patch, n_patch, node_normals, fb, S))) return rc;
  return adjoint(c, nsteps, t0, t1, checkpoint_interval, fb, S, J, dJ_dfb, dJ_dtau, dJ_dEs, dJ_dkb);
}

int zf_flux_objective(zf_ctx* c, int nsteps, int t0, int t1, const int32_t* pts0, int n0, const float* nrm0,
                      const int32_t* pts1, int n1, const float* nrm1, const float* fb, double* J) {
  int rc = check_common(c, nsteps, t0, t1);
  if (rc) return rc;
  if (!J) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  Setup S;
  if ((rc = setup_flux(c, t0, t1, pts0, n0, nrm0, pts1, n1, nrm1, fb, S))) return rc;
  return objective(c, nsteps, t0, t1, fb, S, J);
}

int zf_flux_adjoint(zf_ctx* c, int nsteps, int t0, int t1, const int32_t* pts0, int n0, const float* nrm0,
                    const int32_t* pts1, int n1, const float* nrm1, const float* fb, int checkpoint_interval,
                    double* J, float* dJ_dfb, double* dJ_dtau, double* dJ_dEs, double* dJ_dkb) {
  int rc = check_common(c, nsteps, t0, t1);
  if (rc) return rc;
  if (checkpoint_interval < 1) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  Setup S;
  if ((rc = setup_flux(c, t0, t1, pts0, n0, nrm0, pts1, n1, nrm1, fb, S))) return rc;
  return adjoint(c, nsteps, t0, t1, checkpoint_interval, fb, S, J, dJ_dfb, dJ_dtau, dJ_dEs, dJ_dkb);
}

}  // extern "C"

namespace {

int run_adjoint(zf_ctx* c, int nsteps, int t0, int t1, int K, Setup& S, double* J, float* dJ_dfb,
                double* dJ_dtau, double* dJ_dEs, double* dJ_dkb) {
  int rc;
  const int nseg = (nsteps + K - 1) / K;
  const size_t PB = S.pop_bytes;
  // checkpoints f_0, f_K, ...; the states of one segment; adjoint fields
  DevBuf ck, seg, lam, lam2, gF, gU, gw;
  if ((rc = ck.alloc(c, (size_t)nseg * PB))) return rc;
  if ((rc = seg.alloc(c, (size_t)(K + 1) * PB))) return rc;
  const size_t fl = (size_t)ZF_Q * c->ns * sizeof(float);
  if ((rc = lam.alloc(c, fl)) || (rc = lam2.alloc(c, fl))) return rc;
  if ((rc = gF.alloc(c, 3 * c->ns * sizeof(float))) ||
      (rc = gU.alloc(c, 3 * (size_t)std::max(S.ps.nu, 1) * sizeof(float))))
    return rc;
  const int nb = lbm_adj_blocks(c);
  if ((rc = gw.alloc(c, (size_t)std::max(nb, 1) * sizeof(double)))) return rc;
  char* CK = (char*)ck.p;
  char* SG = (char*)seg.p;
  // forward: objective and checkpoints
  ZF_CUDA(cudaMemcpyAsync(CK, c->d_f[c->cur], PB, cudaMemcpyDeviceToDevice, c->stream));
  ZF_CUDA(cudaMemcpyAsync(SG, CK, PB, cudaMemcpyDeviceToDevice, c->stream));
  ZF_CUDA(cudaMemsetAsync(S.acc.p, 0, sizeof(double), c->stream));
  {
    void* fin = SG;
    void* fout = SG + PB;
    for (int t = 1; t <= nsteps; ++t) {
      if ((rc = lbm_step_buffers(c, fin, fout, S.step0 + (uint32_t)(t - 1)))) return rc;
      std::swap(fin, fout);
      if (t >= t0 && t <= t1 && (rc = objective_of(c, fin, S))) return rc;
      if (t % K == 0 && t / K < nseg)
        ZF_CUDA(cudaMemcpyAsync(CK + (size_t)(t / K) * PB, fin, PB, cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  if (J) ZF_CUDA(cudaMemcpyAsync(J, S.acc.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  // backward
  ZF_CUDA(cudaMemsetAsync(lam.p, 0, fl, c->stream));
  ZF_CUDA(cudaMemsetAsync(lam2.p, 0, fl, c->stream));
  ZF_CUDA(cudaMemsetAsync(gF.p, 0, 3 * c->ns * sizeof(float), c->stream));
  ZF_CUDA(cudaMemsetAsync(gU.p, 0, gU.bytes, c->stream));  // k_seed_at clears it after each use
  ZF_CUDA(cudaMemsetAsync(gw.p, 0, (size_t)std::max(nb, 1) * sizeof(double), c->stream));
  float* L = (float*)lam.p;
  float* Lp = (float*)lam2.p;
  for (int s = nseg - 1; s >= 0; --s) {
    const int base = s * K, len = std::min(K, nsteps - base);
    // states f_base .. f_{base+len} of this segment
    ZF_CUDA(cudaMemcpyAsync(SG, CK + (size_t)s * PB, PB, cudaMemcpyDeviceToDevice, c->stream));
    for (int i = 1; i <= len; ++i)
      if ((rc = lbm_step_buffers(c, SG + (size_t)(i - 1) * PB, SG + (size_t)i * PB,
                                 S.step0 + (uint32_t)(base + i - 1))))
        return rc;
    for (int i = len; i >= 1; --i) {
      const int t = base + i;
      const char* ft = SG + (size_t)i * PB;
      if (t >= t0 && t <= t1 && (rc = objective_seed(c, ft, S, (float*)gU.p, L))) return rc;  // dJ_t/df_t
      if ((rc = lbm_adj_launch(c, SG + (size_t)(i - 1) * PB, L, Lp, (float*)gF.p, (double*)gw.p)))
        return rc;
      std::swap(L, Lp);
    }
  }
  // parameter gradients
  if (dJ_dfb && (rc = lbm_gather_listed(c, (const float*)gF.p, 3, dJ_dfb))) return rc;
  if (dJ_dtau) {
    std::vector<double> h(std::max(nb, 1));
    ZF_CUDA(cudaMemcpyAsync(h.data(), gw.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ZF_CUDA(cudaStreamSynchronize(c->stream));
    double sw = 0.0;
    for (double v : h) sw += v;
    const double om = 1.0 / (double)c->p.tau;
    *dJ_dtau = -om * om * sw;
  }
  if (dJ_dEs) *dJ_dEs = 0.0;
  if (dJ_dkb) *dJ_dkb = 0.0;
  const CellArgs& cl = c->cells;
  if ((dJ_dEs || dJ_dkb) && c->cells_set && cl.n_cells > 0) {
    const size_t nm = 3 * (size_t)cl.n_cells * cl.nn, nn_ = 3 * (size_t)cl.n_cells * cl.nnn;
    DevBuf gm, gn;
    if ((rc = gm.alloc(c, nm * sizeof(float))) || (rc = gn.alloc(c, std::max(nn_, (size_t)1) * sizeof(float))))
      return rc;
    if ((rc = spread_adj_launch(c, (const float*)gF.p, (float*)gm.p, (float*)gn.p))) return rc;
    std::vector<float> hgm(nm), hgn(nn_), F0m(nm), F0n(nn_), F1m(nm), F1n(nn_);
    std::vector<int32_t> status(cl.n_cells);
    std::vector<unsigned long long> counters(4);
    ZF_CUDA(cudaMemcpyAsync(hgm.data(), gm.p, nm * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    if (nn_) ZF_CUDA(cudaMemcpyAsync(hgn.data(), gn.p, nn_ * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    ZF_CUDA(cudaMemcpyAsync(status.data(), cl.status, status.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            c->stream));
    ZF_CUDA(cudaMemcpyAsync(counters.data(), cl.counters, 4 * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, c->stream));
    auto forces = [&](std::vector<float>& m, std::vector<float>& n) -> int {
      int r = cells_membrane_launch(c);
      if (r) return r;
      ZF_CUDA(cudaMemcpyAsync(m.data(), cl.ftot, nm * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      if (nn_) ZF_CUDA(cudaMemcpyAsync(n.data(), cl.ftot_n, nn_ * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      ZF_CUDA(cudaStreamSynchronize(c->stream));
      return ZF_OK;
    };
    auto dot = [&](const std::vector<float>& m1, const std::vector<float>& n1, double scale) {
      double acc = 0.0;
      for (size_t i = 0; i < nm; ++i) acc += (double)hgm[i] * ((double)m1[i] - F0m[i]);
      for (size_t i = 0; i < nn_; ++i) acc += (double)hgn[i] * ((double)n1[i] - F0n[i]);
      return acc / scale;
    };
    if ((rc = forces(F0m, F0n))) return rc;
    if (dJ_dEs) {  // F(2 Es) - F(Es) = Es A
      if ((rc = scale_springs_launch(c, 2.f))) return rc;
      rc = forces(F1m, F1n);
      const int rc2 = scale_springs_launch(c, 0.5f);
      if (rc || (rc = rc2)) return rc;
      *dJ_dEs = dot(F1m, F1n, c->p.Es);
    }
    if (dJ_dkb) {  // F(2 kb) - F(kb) = kb B
      const float kb = c->cells.kbend;
      c->cells.kbend = 2.f * kb;
      rc = forces(F1m, F1n);
      c->cells.kbend = kb;
      if (rc) return rc;
      *dJ_dkb = dot(F1m, F1n, c->p.kbend);
    }
    // the force evaluations ran at the same positions: put back the state they
    // may have touched (forces, removal bookkeeping)
    if ((rc = cells_membrane_launch(c))) return rc;
    ZF_CUDA(cudaMemcpyAsync(cl.status, status.data(), status.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            c->stream));
    ZF_CUDA(cudaMemcpyAsync(cl.counters, counters.data(), 4 * sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, c->stream));
  }
  return restore(c, S);
}

}  // namespace

// ---- the coupled forward: the cells move -----------------------------------------
//
// With zf_adjoint_move_cells(ctx, 1) the differentiated forward is the
// reference's time loop (ZebraflowWT.c:5646-12190) over the window, iteration
// iter0 + t for t = 1..N:
//   BF_0 = S(x_0) F(x_0) + F_b                     (as with held cells)
//   f_t  = LBM(f_{t-1}; tau, BF)                   every iteration
//   at membrane iterations ((iter0 + t) % stagger == 0), with x the positions:
//     F = F(x; Es, kb) (before the LBM step), then after it
//     u = I(x, U(f_t)) + repulsion velocities, BF = S(x) (gamma_p wrep + F) + F_b,
//     x <- x + dt_stagger u
// The adjoint walks the window backwards: at each membrane iteration the
// transposed update, spreading and interpolation (k_ib_vjp) and the membrane
// forces' vector-Jacobian product (k_membrane_vjp) carry the adjoint of the
// positions, the spread field's dJ/dBF turns into dJ/dF, and the interpolation
// seeds dJ/dU into the populations' adjoint, and the repulsion velocities'
// adjoint goes through the transposed wall, nucleus-membrane and RBC-RBC
// repulsions (k_wall_vjp, k_nuc_vjp, k_rbc_vjp) at the iteration's positions:
// the backward re-forms the iteration's geometry, cell list, wall triangles
// and nucleus-membrane lists there.  Positions, spread forces and the spread
// field of every membrane iteration are kept (M + 1 snapshots for M membrane
// iterations).

namespace {

struct Event {
  int t = 0;             // window step of the membrane iteration (0: the window start)
  size_t off = 0;        // offset of its snapshot
};

struct Coupled {
  zf_ctx* c = nullptr;
  size_t nxm = 0, nxn = 0;     // doubles of the membrane and nucleus positions
  size_t bf_bytes = 0, snap_bytes = 0;
  std::vector<Event> ev;
  std::vector<char> rebuilt;   // the forward rebuilt the nucleus-membrane lists at event k
  DevBuf snaps;                // per event: x, xn (double), ftot, ftot_n, wrep, wrep_n (float), BF
  DevBuf fbdev;                // F_b in slot layout [3][ns]
  DevBuf save_x;               // positions at entry
  DevBuf save_lists;           // nucleus-membrane lists at entry
  size_t list_bytes = 0, cnt_bytes = 0;
  std::vector<int32_t> status;
  std::vector<unsigned long long> counters;
  bool lists_valid = false;
  double* X(int k) { return (double*)((char*)snaps.p + ev[k].off); }
  float* F(int k) { return (float*)(X(k) + nxm + nxn); }  // ftot [nxm], ftot_n [nxn], wrep, wrep_n
  float* BF(int k) { return F(k) + 2 * (nxm + nxn); }
};

bool cells_active(zf_ctx* c) { return c->cells_set && c->cells.n_cells > 0; }

// membrane iterations of the window and the snapshot buffers
int coupled_setup(zf_ctx* c, int nsteps, const float* fb, bool keep, Coupled& P) {
  P.c = c;
  const CellArgs& cl = c->cells;
  P.nxm = 3 * (size_t)cl.n_cells * cl.nn;
  P.nxn = 3 * (size_t)cl.n_cells * cl.nnn;
  P.bf_bytes = 3 * (size_t)c->ns * sizeof(float);
  P.snap_bytes = (P.nxm + P.nxn) * (sizeof(double) + 2 * sizeof(float)) + P.bf_bytes;
  P.snap_bytes = (P.snap_bytes + 255) & ~(size_t)255;
  const int64_t iter0 = c->status.iter;
  P.ev.push_back(Event{0, 0});
  for (int t = 1; t <= nsteps; ++t)
    if ((iter0 + t) % c->p.stagger == 0) P.ev.push_back(Event{t, 0});
  for (size_t k = 0; k < P.ev.size(); ++k) P.ev[k].off = k * P.snap_bytes;
  P.rebuilt.assign(P.ev.size(), 0);
  int rc;
  if (keep && (rc = P.snaps.alloc(c, P.ev.size() * P.snap_bytes))) return rc;
  if ((rc = P.fbdev.alloc(c, P.bf_bytes))) return rc;
  ZF_CUDA(cudaMemsetAsync(P.fbdev.p, 0, P.bf_bytes, c->stream));
  if (fb && (rc = lbm_scatter_listed(c, fb, 3, (float*)P.fbdev.p))) return rc;
  if ((rc = P.save_x.alloc(c, (P.nxm + P.nxn) * sizeof(double)))) return rc;
  ZF_CUDA(cudaMemcpyAsync(P.save_x.p, cl.x, P.nxm * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (P.nxn)
    ZF_CUDA(cudaMemcpyAsync((double*)P.save_x.p + P.nxm, cl.xn, P.nxn * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
  P.list_bytes = (size_t)cl.n_cells * cl.nnn * c->ib.nuc_cap * sizeof(uint16_t);
  P.cnt_bytes = (size_t)cl.n_cells * cl.nnn * sizeof(int32_t);
  if (P.list_bytes && c->ib.nuc_list) {
    if ((rc = P.save_lists.alloc(c, P.list_bytes + P.cnt_bytes))) return rc;
    ZF_CUDA(cudaMemcpyAsync(P.save_lists.p, c->ib.nuc_list, P.list_bytes, cudaMemcpyDeviceToDevice, c->stream));
    ZF_CUDA(cudaMemcpyAsync((char*)P.save_lists.p + P.list_bytes, c->ib.nuc_cnt, P.cnt_bytes,
                            cudaMemcpyDeviceToDevice, c->stream));
  }
  P.lists_valid = c->nuc_lists_valid;
  P.status.resize(cl.n_cells);
  P.counters.resize(4);
  ZF_CUDA(cudaMemcpyAsync(P.status.data(), cl.status, P.status.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                          c->stream));
  ZF_CUDA(cudaMemcpyAsync(P.counters.data(), cl.counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

// snapshot k: positions now, the forces the spreading used, the spread field
int snap(zf_ctx* c, Coupled& P, int k) {
  const CellArgs& cl = c->cells;
  const cudaStream_t s = c->stream;
  double* X = P.X(k);
  float* F = P.F(k);
  ZF_CUDA(cudaMemcpyAsync(X, cl.x, P.nxm * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ZF_CUDA(cudaMemcpyAsync(F, cl.ftot, P.nxm * sizeof(float), cudaMemcpyDeviceToDevice, s));
  ZF_CUDA(cudaMemcpyAsync(F + P.nxm + P.nxn, cl.wrep, P.nxm * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (P.nxn) {
    ZF_CUDA(cudaMemcpyAsync(X + P.nxm, cl.xn, P.nxn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ZF_CUDA(cudaMemcpyAsync(F + P.nxm, cl.ftot_n, P.nxn * sizeof(float), cudaMemcpyDeviceToDevice, s));
    ZF_CUDA(cudaMemcpyAsync(F + 2 * P.nxm + P.nxn, cl.wrep_n, P.nxn * sizeof(float), cudaMemcpyDeviceToDevice, s));
  }
  ZF_CUDA(cudaMemcpyAsync(P.BF(k), c->d_force, P.bf_bytes, cudaMemcpyDeviceToDevice, s));
  return ZF_OK;
}

// positions of snapshot k into the cells
int put_positions(zf_ctx* c, Coupled& P, const double* X) {
  const CellArgs& cl = c->cells;
  int rc = cells_write_fence(c);
  if (rc) return rc;
  ZF_CUDA(cudaMemcpyAsync(cl.x, X, P.nxm * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (P.nxn) ZF_CUDA(cudaMemcpyAsync(cl.xn, X + P.nxm, P.nxn * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  c->node_tiles_valid = false;
  return ZF_OK;
}

// the cells as they were at entry
int coupled_restore(zf_ctx* c, Coupled& P) {
  const CellArgs& cl = c->cells;
  int rc = put_positions(c, P, (const double*)P.save_x.p);
  if (rc) return rc;
  if (P.save_lists.p) {
    ZF_CUDA(cudaMemcpyAsync(c->ib.nuc_list, P.save_lists.p, P.list_bytes, cudaMemcpyDeviceToDevice, c->stream));
    ZF_CUDA(cudaMemcpyAsync(c->ib.nuc_cnt, (char*)P.save_lists.p + P.list_bytes, P.cnt_bytes,
                            cudaMemcpyDeviceToDevice, c->stream));
  }
  c->nuc_lists_valid = P.lists_valid;
  ZF_CUDA(cudaMemcpyAsync(cl.status, P.status.data(), P.status.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                          c->stream));
  ZF_CUDA(cudaMemcpyAsync(cl.counters, P.counters.data(), 4 * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                          c->stream));
  return ZF_OK;
}

// the forward over the window from the populations in buffer f0 (left at the
// last state in *fend); with keep, snapshots and every K-th state into CK
int coupled_forward(zf_ctx* c, int nsteps, int t0, int t1, int K, Setup& S, Coupled& P, bool keep, char* CK,
                    void* bufa, void* bufb) {
  int rc;
  const size_t PB = S.pop_bytes;
  const int64_t iter0 = c->status.iter;
  if (keep && (rc = snap(c, P, 0))) return rc;
  ZF_CUDA(cudaMemsetAsync(S.acc.p, 0, sizeof(double), c->stream));
  void* fin = bufa;
  void* fout = bufb;
  size_t k = 1;
  for (int t = 1; t <= nsteps; ++t) {
    const bool membrane = k < P.ev.size() && P.ev[k].t == t;
    if (membrane && (rc = cells_membrane_launch(c))) return rc;
    if ((rc = lbm_step_buffers(c, fin, fout, S.step0 + (uint32_t)(t - 1)))) return rc;
    std::swap(fin, fout);
    if (membrane) {
      const int64_t iter = iter0 + t;
      const bool rebuild = !c->nuc_lists_valid || (iter % c->p.nuc_list_period == 0);
      P.rebuilt[k] = rebuild;
      ZF_CUDA(cudaMemsetAsync(c->d_force, 0, P.bf_bytes, c->stream));
      if ((rc = lbm_moments_of(c, fin)) || (rc = ib_interp_launch(c)) || (rc = ib_nuc_memb_launch(c, rebuild)))
        return rc;
      c->nuc_lists_valid = true;
      if ((rc = ib_bins_launch(c)) || (rc = ib_rbc_rbc_launch(c)) || (rc = ib_spread_launch(c))) return rc;
      if ((rc = add_launch(c, c->d_force, (const float*)P.fbdev.p, 3 * c->ns))) return rc;
      if (keep && (rc = snap(c, P, (int)k))) return rc;
      if ((rc = ib_update_launch(c))) return rc;
      ++k;
    }
    if (t >= t0 && t <= t1 && (rc = objective_of(c, fin, S))) return rc;
    if (keep && t % K == 0 && t / K < (nsteps + K - 1) / K)
      ZF_CUDA(cudaMemcpyAsync(CK + (size_t)(t / K) * PB, fin, PB, cudaMemcpyDeviceToDevice, c->stream));
  }
  return ZF_OK;
}

int run_objective_coupled(zf_ctx* c, int nsteps, int t0, int t1, const float* fb, Setup& S, double* J) {
  Coupled P;
  int rc;
  if ((rc = coupled_setup(c, nsteps, fb, false, P))) return rc;
  DevBuf a, b;
  if ((rc = a.alloc(c, S.pop_bytes)) || (rc = b.alloc(c, S.pop_bytes))) return rc;
  ZF_CUDA(cudaMemcpyAsync(a.p, c->d_f[c->cur], S.pop_bytes, cudaMemcpyDeviceToDevice, c->stream));
  if ((rc = coupled_forward(c, nsteps, t0, t1, 1, S, P, false, nullptr, a.p, b.p))) return rc;
  ZF_CUDA(cudaMemcpyAsync(J, S.acc.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if ((rc = coupled_restore(c, P))) return rc;
  return restore(c, S);
}

int run_adjoint_coupled(zf_ctx* c, int nsteps, int t0, int t1, int K, const float* fb, Setup& S, double* J,
                        float* dJ_dfb, double* dJ_dtau, double* dJ_dEs, double* dJ_dkb) {
  int rc;
  Coupled P;
  if ((rc = coupled_setup(c, nsteps, fb, true, P))) return rc;
  const int nseg = (nsteps + K - 1) / K;
  const size_t PB = S.pop_bytes;
  const size_t fl = (size_t)ZF_Q * c->ns * sizeof(float);
  const size_t nx = P.nxm + P.nxn;
  DevBuf ck, seg, lam, lam2, gFc, gFb, gU, gw, lx, gFn, GU, gpar, allslots, lw;
  if ((rc = ck.alloc(c, (size_t)nseg * PB)) || (rc = seg.alloc(c, (size_t)(K + 1) * PB))) return rc;
  if ((rc = lam.alloc(c, fl)) || (rc = lam2.alloc(c, fl))) return rc;
  if ((rc = gFc.alloc(c, P.bf_bytes)) || (rc = gFb.alloc(c, P.bf_bytes)) || (rc = GU.alloc(c, P.bf_bytes)))
    return rc;
  if ((rc = gU.alloc(c, 3 * (size_t)std::max(S.ps.nu, 1) * sizeof(float)))) return rc;
  const int nb = lbm_adj_blocks(c);
  if ((rc = gw.alloc(c, (size_t)std::max(nb, 1) * sizeof(double)))) return rc;
  if ((rc = lx.alloc(c, nx * sizeof(float))) || (rc = gFn.alloc(c, nx * sizeof(float)))) return rc;
  if ((rc = gpar.alloc(c, 2 * sizeof(double))) || (rc = lw.alloc(c, P.nxm * sizeof(float)))) return rc;
  // the seed of dJ/dU at every slot: a stencil of all slots
  PatchStencil all;
  {
    if ((rc = allslots.alloc(c, (size_t)c->ns * sizeof(int32_t)))) return rc;
    std::vector<int32_t> id((size_t)c->ns);
    for (int64_t s = 0; s < c->ns; ++s) id[(size_t)s] = (int32_t)s;
    ZF_CUDA(cudaMemcpy(allslots.p, id.data(), id.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    all.nu = (int)c->ns;
    all.uslot = (const int32_t*)allslots.p;
  }
  char* CK = (char*)ck.p;
  char* SG = (char*)seg.p;
  ZF_CUDA(cudaMemcpyAsync(CK, c->d_f[c->cur], PB, cudaMemcpyDeviceToDevice, c->stream));
  ZF_CUDA(cudaMemcpyAsync(SG, CK, PB, cudaMemcpyDeviceToDevice, c->stream));
  if ((rc = coupled_forward(c, nsteps, t0, t1, K, S, P, true, CK, SG, SG + PB))) return rc;
  if (J) ZF_CUDA(cudaMemcpyAsync(J, S.acc.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));

  // backward
  ZF_CUDA(cudaMemsetAsync(lam.p, 0, fl, c->stream));
  ZF_CUDA(cudaMemsetAsync(lam2.p, 0, fl, c->stream));
  ZF_CUDA(cudaMemsetAsync(gFc.p, 0, P.bf_bytes, c->stream));
  ZF_CUDA(cudaMemsetAsync(gFb.p, 0, P.bf_bytes, c->stream));
  ZF_CUDA(cudaMemsetAsync(GU.p, 0, P.bf_bytes, c->stream));  // k_seed_at clears it after each use
  ZF_CUDA(cudaMemsetAsync(gU.p, 0, gU.bytes, c->stream));
  ZF_CUDA(cudaMemsetAsync(gw.p, 0, (size_t)std::max(nb, 1) * sizeof(double), c->stream));
  ZF_CUDA(cudaMemsetAsync(lx.p, 0, nx * sizeof(float), c->stream));
  ZF_CUDA(cudaMemsetAsync(gpar.p, 0, 2 * sizeof(double), c->stream));
  float* L = (float*)lam.p;
  float* Lp = (float*)lam2.p;
  float* LX = (float*)lx.p;
  float* LXn = LX + P.nxm;
  float* GFm = (float*)gFn.p;
  float* GFn = GFm + P.nxm;
  // the spread field in effect at step t: that of the last membrane iteration before t
  int bf_loaded = -1;
  auto load_bf = [&](int t) -> int {
    int k = 0;
    while (k + 1 < (int)P.ev.size() && P.ev[k + 1].t < t) ++k;
    if (k != bf_loaded) {
      ZF_CUDA(cudaMemcpyAsync(c->d_force, P.BF(k), P.bf_bytes, cudaMemcpyDeviceToDevice, c->stream));
      bf_loaded = k;
    }
    return ZF_OK;
  };
  // transposed membrane iteration k (spreading, forces; with interp: also
  // interpolation and update) at its positions
  // nucleus-membrane lists as the forward used them at event k: built at the
  // last rebuild event r <= k (at its positions), else the lists at entry
  int lists_of = -2;  // event whose lists are loaded (-1: the entry lists)
  auto load_lists = [&](int k) -> int {
    int r = -1;
    for (int i = k; i >= 1; --i)
      if (P.rebuilt[i]) {
        r = i;
        break;
      }
    if (r == lists_of) return ZF_OK;
    int e;
    if (r < 0) {
      if (P.save_lists.p) {
        ZF_CUDA(cudaMemcpyAsync(c->ib.nuc_list, P.save_lists.p, P.list_bytes, cudaMemcpyDeviceToDevice,
                                c->stream));
        ZF_CUDA(cudaMemcpyAsync(c->ib.nuc_cnt, (char*)P.save_lists.p + P.list_bytes, P.cnt_bytes,
                                cudaMemcpyDeviceToDevice, c->stream));
      }
    } else {
      if ((e = put_positions(c, P, P.X(r))) || (e = cells_membrane_launch(c)) || (e = ib_nuc_memb_launch(c, 1)))
        return e;
    }
    lists_of = r;
    return ZF_OK;
  };
  auto event_adj = [&](int k, const void* ft) -> int {
    int r;
    const float* F = P.F(k);
    const bool interp = k > 0;
    if (interp) {
      // the iteration's geometry, wall triangles and cell list at its positions
      if ((r = load_lists(k)) || (r = put_positions(c, P, P.X(k))) || (r = cells_membrane_launch(c)) ||
          (r = lbm_moments_of(c, ft)) || (r = ib_interp_launch(c)) || (r = ib_bins_launch(c)))
        return r;
    } else if ((r = put_positions(c, P, P.X(k)))) {
      return r;
    }
    if ((r = ib_vjp_launch(c, (const float*)gFc.p, interp ? LX : nullptr, interp ? LXn : nullptr, LX, LXn, GFm,
                           GFn, interp ? (float*)GU.p : nullptr, interp ? (float*)lw.p : nullptr, F, F + P.nxm,
                           F + P.nxm + P.nxn, F + 2 * P.nxm + P.nxn)))
      return r;
    if ((r = membrane_vjp_launch(c, GFm, GFn, LX, LXn, (double*)gpar.p))) return r;
    if (interp && (r = repulsion_vjp_launch(c, (const float*)lw.p, LX, LXn))) return r;
    if ((r = add_launch(c, (float*)gFb.p, (const float*)gFc.p, 3 * c->ns))) return r;
    ZF_CUDA(cudaMemsetAsync(gFc.p, 0, P.bf_bytes, c->stream));
    if (interp && (r = lbm_seed_at(c, ft, all, (float*)GU.p, L))) return r;
    return ZF_OK;
  };
  int ke = (int)P.ev.size() - 1;  // next membrane iteration to meet going backwards
  for (int s = nseg - 1; s >= 0; --s) {
    const int base = s * K, len = std::min(K, nsteps - base);
    ZF_CUDA(cudaMemcpyAsync(SG, CK + (size_t)s * PB, PB, cudaMemcpyDeviceToDevice, c->stream));
    for (int i = 1; i <= len; ++i) {
      if ((rc = load_bf(base + i))) return rc;
      if ((rc = lbm_step_buffers(c, SG + (size_t)(i - 1) * PB, SG + (size_t)i * PB,
                                 S.step0 + (uint32_t)(base + i - 1))))
        return rc;
    }
    for (int i = len; i >= 1; --i) {
      const int t = base + i;
      const char* ft = SG + (size_t)i * PB;
      if (ke > 0 && P.ev[ke].t == t) {
        if ((rc = event_adj(ke, ft))) return rc;
        --ke;
      }
      if (t >= t0 && t <= t1 && (rc = objective_seed(c, ft, S, (float*)gU.p, L))) return rc;
      if ((rc = load_bf(t))) return rc;
      if ((rc = lbm_adj_launch(c, SG + (size_t)(i - 1) * PB, L, Lp, (float*)gFc.p, (double*)gw.p))) return rc;
      std::swap(L, Lp);
    }
  }
  if ((rc = event_adj(0, nullptr))) return rc;  // BF_0 = S(x_0) F(x_0) + F_b

  // outputs
  if (dJ_dfb && (rc = lbm_gather_listed(c, (const float*)gFb.p, 3, dJ_dfb))) return rc;
  std::vector<double> h(std::max(nb, 1));
  double gp[2] = {0.0, 0.0};
  c->adj_gx.resize(P.nxm);
  c->adj_gxn.resize(P.nxn);
  ZF_CUDA(cudaMemcpyAsync(h.data(), gw.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaMemcpyAsync(gp, gpar.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaMemcpyAsync(c->adj_gx.data(), LX, P.nxm * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if (P.nxn)
    ZF_CUDA(cudaMemcpyAsync(c->adj_gxn.data(), LXn, P.nxn * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  if (dJ_dtau) {
    double sw = 0.0;
    for (double v : h) sw += v;
    const double om = 1.0 / (double)c->p.tau;
    *dJ_dtau = -om * om * sw;
  }
  if (dJ_dEs) *dJ_dEs = gp[0];
  if (dJ_dkb) *dJ_dkb = gp[1];
  if ((rc = coupled_restore(c, P))) return rc;
  return restore(c, S);
}

}  // namespace

extern "C" {

int zf_adjoint_move_cells(zf_ctx* c, int move) {
  if (!c) return ZF_ERR_ARG;
  c->adj_move_cells = move != 0;
  return ZF_OK;
}

int zf_adjoint_position_gradient(zf_ctx* c, float* dJ_dx, float* dJ_dxn) {
  if (!c) return ZF_ERR_ARG;
  if (c->adj_gx.empty()) {
    set_error("no adjoint with moving cells has run since the cells were set");
    return ZF_ERR_STATE;
  }
  if (dJ_dx) std::copy(c->adj_gx.begin(), c->adj_gx.end(), dJ_dx);
  if (dJ_dxn) std::copy(c->adj_gxn.begin(), c->adj_gxn.end(), dJ_dxn);
  return ZF_OK;
}

int zf_repulsion_vjp(zf_ctx* c, const float* lam_w, float* dx, float* dxn) {
  if (!c || !lam_w) return ZF_ERR_ARG;
  if (!c->cells_set || !c->lattice_set) {
    set_error("zf_repulsion_vjp: lattice and cells must be set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  const CellArgs& cl = c->cells;
  const size_t nm = 3 * (size_t)cl.n_cells * cl.nn, nn_ = 3 * (size_t)cl.n_cells * cl.nnn;
  int rc;
  if (c->ib_allocs.empty() && (rc = ib_prepare(c))) return rc;
  DevBuf b;
  const size_t bytes = (2 * nm + nn_) * sizeof(float);
  if ((rc = b.alloc(c, bytes))) return rc;
  float* dl = (float*)b.p;
  float* g = dl + nm;
  float* gn = g + nm;
  ZF_CUDA(cudaMemsetAsync(b.p, 0, bytes, c->stream));
  ZF_CUDA(cudaMemcpyAsync(dl, lam_w, nm * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  // the membrane iteration's geometry, wall triangles, lists and cell list at
  // the current positions (forces, velocities and repulsions are overwritten)
  if ((rc = cells_membrane_launch(c)) || (rc = lbm_moments_launch(c)) || (rc = ib_interp_launch(c)) ||
      (rc = ib_nuc_memb_launch(c, 1)) || (rc = ib_bins_launch(c)))
    return rc;
  c->nuc_lists_valid = true;
  if ((rc = repulsion_vjp_launch(c, dl, g, gn))) return rc;
  if (dx) ZF_CUDA(cudaMemcpyAsync(dx, g, nm * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if (dxn && nn_) ZF_CUDA(cudaMemcpyAsync(dxn, gn, nn_ * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int zf_membrane_vjp(zf_ctx* c, const float* lam, const float* lam_n, float* dx, float* dxn, double* dEs,
                    double* dkb) {
  if (!c || !lam) return ZF_ERR_ARG;
  if (!c->cells_set) {
    set_error("zf_membrane_vjp: cells not set");
    return ZF_ERR_STATE;
  }
  ZF_CUDA(cudaSetDevice(c->device));
  const CellArgs& cl = c->cells;
  const size_t nm = 3 * (size_t)cl.n_cells * cl.nn, nn_ = 3 * (size_t)cl.n_cells * cl.nnn;
  DevBuf b;
  int rc;
  const size_t bytes = 2 * (nm + nn_) * sizeof(float) + 2 * sizeof(double);
  if ((rc = b.alloc(c, bytes))) return rc;
  float* dl = (float*)b.p;
  float* dln = dl + nm;
  float* g = dln + nn_;
  float* gn = g + nm;
  double* gp = (double*)(gn + nn_);
  ZF_CUDA(cudaMemsetAsync(b.p, 0, bytes, c->stream));
  ZF_CUDA(cudaMemcpyAsync(dl, lam, nm * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if (lam_n && nn_) ZF_CUDA(cudaMemcpyAsync(dln, lam_n, nn_ * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = membrane_vjp_launch(c, dl, dln, g, gn, gp))) return rc;
  double h[2];
  if (dx) ZF_CUDA(cudaMemcpyAsync(dx, g, nm * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if (dxn && nn_) ZF_CUDA(cudaMemcpyAsync(dxn, gn, nn_ * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaMemcpyAsync(h, gp, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  if (dEs) *dEs = h[0];
  if (dkb) *dkb = h[1];
  return ZF_OK;
}

}  // extern "C"

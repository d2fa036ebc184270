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
  return run_objective(c, nsteps, t0, t1, S, J);
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
  return run_adjoint(c, nsteps, t0, t1, checkpoint_interval, S, J, dJ_dfb, dJ_dtau, dJ_dEs, dJ_dkb);
}

int zf_flux_objective(zf_ctx* c, int nsteps, int t0, int t1, const int32_t* pts0, int n0, const float* nrm0,
                      const int32_t* pts1, int n1, const float* nrm1, const float* fb, double* J) {
  int rc = check_common(c, nsteps, t0, t1);
  if (rc) return rc;
  if (!J) return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  Setup S;
  if ((rc = setup_flux(c, t0, t1, pts0, n0, nrm0, pts1, n1, nrm1, fb, S))) return rc;
  return run_objective(c, nsteps, t0, t1, S, J);
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
  return run_adjoint(c, nsteps, t0, t1, checkpoint_interval, S, J, dJ_dfb, dJ_dtau, dJ_dEs, dJ_dkb);
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

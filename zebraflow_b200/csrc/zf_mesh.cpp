// Membrane mesh set-up on the host: topology, spring calibration and rest
// metrics shared by every cell.
//
// Reference behaviour restated here (ZebraflowWT.c):
//  - edge list and 4-node rhombus (n1,n2 edge; n3,n4 opposite vertices;
//    tri1, tri2) in the order CGSM_ZFISHRBC_DATA_GEN builds them, :1640-1805.
//    The reference scans all edges per triangle and all triangles per edge
//    (O(E*T)); a hash of node pairs gives the same order in O(T).
//  - WLC persistence length and POW coefficient by fixed-point iteration,
//    CGSM_FILAMENT_PARAMETERS :1930-2053, run `calib_passes` times (:2339-2346)
//  - LMAX, rest dihedral angles: CGSM_EQUILIBRIUM_METRICS :2056-2223
//  - rest triangle areas TRI_AREA_eq: :2387-2460
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <unordered_map>
#include <vector>

#include "zf_internal.h"
#include "zf_mesh.h"

namespace zf {

uint64_t pair_key(int a, int b) {
  if (a > b) std::swap(a, b);
  return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
}

int mesh_build(MeshHost& m, const zf_params& P) {
  const int nn = m.n_node, nt = m.n_tri;
  // 1) edges in first-appearance order over triangles, (v1v2, v2v3, v3v1)
  std::unordered_map<uint64_t, int> eid;
  eid.reserve((size_t)nt * 2);
  m.edge.clear();
  for (int t = 0; t < nt; ++t) {
    const int v[3] = {m.tri[3 * t], m.tri[3 * t + 1], m.tri[3 * t + 2]};
    for (int s = 0; s < 3; ++s) {
      const int a = v[s], b = v[(s + 1) % 3];
      const uint64_t k = pair_key(a, b);
      if (eid.count(k)) continue;
      eid[k] = (int)(m.edge.size() / 6);
      const int e6[6] = {a, b, -1, -1, -1, -1};
      m.edge.insert(m.edge.end(), e6, e6 + 6);
    }
  }
  m.n_edge = (int)(m.edge.size() / 6);
  // 2) rhombus: the first triangle (in index order) holding the edge gives
  //    n3/tri1, the second n4/tri2
  for (int t = 0; t < nt; ++t) {
    const int v[3] = {m.tri[3 * t], m.tri[3 * t + 1], m.tri[3 * t + 2]};
    for (int s = 0; s < 3; ++s) {
      const int a = v[s], b = v[(s + 1) % 3], opp = v[(s + 2) % 3];
      int* e = &m.edge[6 * eid[pair_key(a, b)]];
      if (e[2] < 0) {
        e[2] = opp;
        e[4] = t;
      } else if (e[3] < 0) {
        e[3] = opp;
        e[5] = t;
      }
    }
  }
  for (int e = 0; e < m.n_edge; ++e)
    if (m.edge[6 * e + 3] < 0) {
      set_error("zf_set_mesh: edge %d (%d,%d) borders one triangle; the membrane must be closed",
                e, m.edge[6 * e], m.edge[6 * e + 1]);
      return ZF_ERR_ARG;
    }
  // 3) first visitor of each triangle's area/volume terms (AREA_UPDATE,
  //    ZebraflowWT.c:7127-7128, :7250-7251: edges in order, tri1 before tri2)
  m.area_first.assign(m.n_edge, 0);
  {
    std::vector<uint8_t> seen(nt, 0);
    for (int e = 0; e < m.n_edge; ++e) {
      const int t1 = m.edge[6 * e + 4], t2 = m.edge[6 * e + 5];
      if (!seen[t1]) {
        seen[t1] = 1;
        m.area_first[e] |= 1;
      }
      if (!seen[t2]) {
        seen[t2] = 1;
        m.area_first[e] |= 2;
      }
    }
  }

  // 4) calibration and rest metrics (the reference keeps these in float)
  const double x0 = P.e_ratio_eq;
  const float beta = (float)(0.5 * x0 / ((1. - x0) * (1. - x0) * (1. - x0)) -
                             0.25 / ((1. - x0) * (1. - x0)) + 0.25);
  const double wlc0 = x0 - 0.25 + 1. / (4. * (1. - x0) * (1. - x0));
  auto calibrate = [&](const std::vector<double>& X, const std::vector<int32_t>& E, int stride,
                       int ne, double Es_local, std::vector<float>& lmax,
                       std::vector<float>& plen, std::vector<float>& kp) {
    lmax.assign(ne, 0.f);
    plen.assign(ne, 1.e-9f);
    kp.assign(ne, 0.f);
    for (int e = 0; e < ne; ++e) {
      const int a = E[stride * e], b = E[stride * e + 1];
      const float dx = (float)(X[3 * a] - X[3 * b]), dy = (float)(X[3 * a + 1] - X[3 * b + 1]),
                  dz = (float)(X[3 * a + 2] - X[3 * b + 2]);
      const float l = sqrtf(dx * dx + dy * dy + dz * dz);
      const float alpha = (float)(sqrtf(3.f) * 0.25 * P.kT / (l * 1.e-006));
      const float eta = (float)(sqrtf(3.f) * 0.25 * (2. + 1.) / ((double)(l * l * l) * 1.e-018));
      float P_ = 1.e-9f, k_ = 0.f;
      for (int pass = 0; pass < P.calib_passes; ++pass) {
        k_ = ((float)Es_local - alpha * beta / P_) / eta;
        P_ = (float)((double)(l * l) * 1.e-012 * P.kT * wlc0 / k_);
      }
      plen[e] = P_;
      kp[e] = k_;
      lmax[e] = (float)(1.e-006 * l / x0);
    }
  };
  calibrate(m.rest, m.edge, 6, m.n_edge, P.Es, m.lmax, m.plength, m.kp);
  calibrate(m.rest_n, m.edge_n, 2, m.n_edge_n, P.Es * P.Es_nucleus_ratio, m.lmax_n, m.plength_n,
            m.kp_n);

  // rest dihedral angles from Heron areas and vector-area normals, :2073-2221
  m.sin0.assign(m.n_edge, 0.f);
  m.cos0.assign(m.n_edge, 0.f);
  const std::vector<double>& X = m.rest;
  for (int e = 0; e < m.n_edge; ++e) {
    const int n1 = m.edge[6 * e], n2 = m.edge[6 * e + 1], n3 = m.edge[6 * e + 2],
              n4 = m.edge[6 * e + 3];
    auto nrm = [&](int a, int b, int c, float* out, float* cen) {
      // vector area of the polygon a->b->c over its Heron area
      const int v[3] = {a, b, c};
      float len[3];
      for (int s = 0; s < 3; ++s) {
        const int p = v[s], q = v[(s + 1) % 3];
        const float dx = (float)(X[3 * p] - X[3 * q]), dy = (float)(X[3 * p + 1] - X[3 * q + 1]),
                    dz = (float)(X[3 * p + 2] - X[3 * q + 2]);
        len[s] = sqrtf(dx * dx + dy * dy + dz * dz);
      }
      const float sp = 0.5f * (len[0] + len[1] + len[2]);
      const float area =
          (float)(sqrtf(sp * (sp - len[0]) * (sp - len[1]) * (sp - len[2])) * 1.e-12);
      float ax = 0, ay = 0, az = 0;
      for (int s = 0; s < 3; ++s) {
        const int p = v[s], q = v[(s + 1) % 3];
        const float dxp = (float)(X[3 * p] - X[3 * q]), dyp = (float)(X[3 * p + 1] - X[3 * q + 1]),
                    dzp = (float)(X[3 * p + 2] - X[3 * q + 2]);
        const float sx = (float)(X[3 * p] + X[3 * q]), sy = (float)(X[3 * p + 1] + X[3 * q + 1]),
                    sz = (float)(X[3 * p + 2] + X[3 * q + 2]);
        ax += dyp * sz;
        ay += dzp * sx;
        az += dxp * sy;
      }
      out[0] = (float)(0.5 * ax * 1.e-12 / area);
      out[1] = (float)(0.5 * ay * 1.e-12 / area);
      out[2] = (float)(0.5 * az * 1.e-12 / area);
      for (int s = 0; s < 3; ++s) cen[s] = (float)((X[3 * a + s] + X[3 * b + s] + X[3 * c + s]) / 3.);
    };
    float t1n[3], t2n[3], c1[3], c2[3];
    nrm(n1, n2, n3, t1n, c1);
    nrm(n2, n1, n4, t2n, c2);
    float cs = t1n[0] * t2n[0] + t1n[1] * t2n[1] + t1n[2] * t2n[2];
    cs = cs > 1.f ? 1.f : (cs < -1.f ? -1.f : cs);
    float chk = 0;
    for (int s = 0; s < 3; ++s) chk += (t1n[s] - t2n[s]) * (float)((c1[s] - c2[s]) * 1.e-006);
    const float sn = chk >= 0 ? sqrtf(1.f - cs * cs) : -sqrtf(1.f - cs * cs);
    m.sin0[e] = sn;
    m.cos0[e] = cs;
  }

  // rest triangle areas (cross-product form), :2398-2423; rest cell area and volume
  m.tri_area_eq.assign(nt, 0.f);
  double A = 0, V = 0;
  for (int t = 0; t < nt; ++t) {
    const int a = m.tri[3 * t], b = m.tri[3 * t + 1], c = m.tri[3 * t + 2];
    float p1[3], p2[3], p3[3];
    for (int s = 0; s < 3; ++s) {
      p1[s] = (float)X[3 * a + s];
      p2[s] = (float)X[3 * b + s];
      p3[s] = (float)X[3 * c + s];
    }
    const float e1[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
    const float e3[3] = {p1[0] - p3[0], p1[1] - p3[1], p1[2] - p3[2]};
    const float Ax = (float)(0.5 * (e1[1] * e3[2] - e1[2] * e3[1]) * 1.e-012);
    const float Ay = (float)(0.5 * (e1[2] * e3[0] - e1[0] * e3[2]) * 1.e-012);
    const float Az = (float)(0.5 * (e1[0] * e3[1] - e1[1] * e3[0]) * 1.e-012);
    const float ar = sqrtf(Ax * Ax + Ay * Ay + Az * Az);
    m.tri_area_eq[t] = ar;
    A += ar;
    const double cx = (p1[0] + p2[0] + p3[0]) / 3., cy = (p1[1] + p2[1] + p3[1]) / 3.,
                 cz = (p1[2] + p2[2] + p3[2]) / 3.;
    V += ar * (cx * (-Ax / ar) + cy * (-Ay / ar) + cz * (-Az / ar)) * 1.e-006;
  }
  m.area0 = P.area0 > 0 ? P.area0 : A;
  m.volume0 = P.volume0 > 0 ? P.volume0 : V / 3.;
  return ZF_OK;
}

}  // namespace zf

// ---- C ABI: mesh and cells -------------------------------------------------

using namespace zf;

namespace {

template <typename T>
int upload(zf_ctx* c, std::vector<void*>& owned, T** dst, const T* src, size_t n) {
  void* p = nullptr;
  int rc = dev_alloc(c, &p, (n ? n : 1) * sizeof(T));
  if (rc) return rc;
  owned.push_back(p);
  if (n && src) ZF_CUDA(cudaMemcpyAsync(p, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  if (!src) ZF_CUDA(cudaMemsetAsync(p, 0, (n ? n : 1) * sizeof(T), c->stream));
  *dst = (T*)p;
  return ZF_OK;
}

void free_owned(std::vector<void*>& v) {
  for (void* p : v) cudaFree(p);
  v.clear();
}

}  // namespace

namespace zf {
void cells_free(zf_ctx* c) {
  free_owned(c->cell_allocs);
  free_owned(c->mesh_allocs);
  delete (MeshHost*)c->mesh_host;
  c->mesh_host = nullptr;
  c->mesh_set = c->cells_set = false;
  c->cells = CellArgs{};
}
}  // namespace zf

#define NEED(cond, fn, msg)            \
  if (!(cond)) {                       \
    set_error(fn ": " msg);            \
    return ZF_ERR_STATE;               \
  }

namespace zf {

int cells_write_fence(zf_ctx* c) {
  if (c->copy_pending) {
    ZF_CUDA(cudaStreamWaitEvent(c->stream, c->ev_copied, 0));
    c->copy_pending = false;
  }
  return ZF_OK;
}

int cells_copy_wait_host(zf_ctx* c) {
  if (c->copy_stream) ZF_CUDA(cudaStreamSynchronize(c->copy_stream));
  c->copy_pending = false;
  return ZF_OK;
}

}  // namespace zf

extern "C" {

int zf_set_mesh(zf_ctx* c, int n_node, int n_tri, const int32_t* tri, const double* rest,
                int n_node_n, int n_edge_n, const int32_t* edge_n, const double* rest_n) {
  if (!c || !tri || !rest || n_node < 4 || n_tri < 4 || n_node_n < 0 || n_edge_n < 0 ||
      (n_edge_n > 0 && (!edge_n || !rest_n)))
    return ZF_ERR_ARG;
  ZF_CUDA(cudaSetDevice(c->device));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  cells_free(c);
  MeshHost* m = new MeshHost();
  c->mesh_host = m;
  m->n_node = n_node;
  m->n_tri = n_tri;
  m->tri.resize(3 * (size_t)n_tri);
  for (size_t i = 0; i < m->tri.size(); ++i) {
    m->tri[i] = tri[i] - 1;
    if (m->tri[i] < 0 || m->tri[i] >= n_node) {
      set_error("zf_set_mesh: triangle node %d out of range 1..%d", tri[i], n_node);
      return ZF_ERR_ARG;
    }
  }
  m->rest.assign(rest, rest + 3 * (size_t)n_node);
  m->n_node_n = n_node_n;
  m->n_edge_n = n_edge_n;
  m->edge_n.resize(2 * (size_t)n_edge_n);
  for (size_t i = 0; i < m->edge_n.size(); ++i) {
    m->edge_n[i] = edge_n[i] - 1;
    if (m->edge_n[i] < 0 || m->edge_n[i] >= n_node_n) {
      set_error("zf_set_mesh: nucleus edge node %d out of range 1..%d", edge_n[i], n_node_n);
      return ZF_ERR_ARG;
    }
  }
  if (n_node_n) m->rest_n.assign(rest_n, rest_n + 3 * (size_t)n_node_n);
  int rc = mesh_build(*m, c->p);
  if (rc) return rc;

  CellArgs& a = c->cells;
  a.nn = m->n_node;
  a.nt = m->n_tri;
  a.ne = m->n_edge;
  a.nnn = m->n_node_n;
  a.nen = m->n_edge_n;
  std::vector<float> epar(5 * (size_t)a.ne), epar_n(3 * (size_t)a.nen);
  for (int e = 0; e < a.ne; ++e) {
    epar[e] = m->lmax[e];
    epar[a.ne + e] = m->plength[e];
    epar[2 * a.ne + e] = m->kp[e];
    epar[3 * a.ne + e] = m->sin0[e];
    epar[4 * a.ne + e] = m->cos0[e];
  }
  for (int e = 0; e < a.nen; ++e) {
    epar_n[e] = m->lmax_n[e];
    epar_n[a.nen + e] = m->plength_n[e];
    epar_n[2 * a.nen + e] = m->kp_n[e];
  }
  auto& own = c->mesh_allocs;
  if ((rc = upload(c, own, (int32_t**)&a.tri, m->tri.data(), m->tri.size()))) return rc;
  if ((rc = upload(c, own, (int32_t**)&a.edge, m->edge.data(), m->edge.size()))) return rc;
  if ((rc = upload(c, own, (uint8_t**)&a.area_first, m->area_first.data(), m->area_first.size())))
    return rc;
  if ((rc = upload(c, own, (float**)&a.epar, epar.data(), epar.size()))) return rc;
  if ((rc = upload(c, own, (float**)&a.tri_area_eq, m->tri_area_eq.data(), m->tri_area_eq.size())))
    return rc;
  if ((rc = upload(c, own, (int32_t**)&a.edge_n, m->edge_n.data(), m->edge_n.size()))) return rc;
  if ((rc = upload(c, own, (float**)&a.epar_n, epar_n.data(), epar_n.size()))) return rc;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  a.kT = (float)c->p.kT;
  a.kbend = (float)c->p.kbend;
  a.kd = (float)c->p.kd;
  a.ka = (float)c->p.ka;
  a.kv = (float)c->p.kv;
  a.area0 = (float)m->area0;
  a.volume0 = (float)m->volume0;
  a.remove_count = c->p.remove_count;
  c->mesh_set = true;
  return ZF_OK;
}

int zf_mesh_info(zf_ctx* c, int32_t* n_edge, double* area0, double* volume0) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->mesh_set, "zf_mesh_info", "mesh not set");
  const MeshHost* m = (const MeshHost*)c->mesh_host;
  if (n_edge) *n_edge = m->n_edge;
  if (area0) *area0 = m->area0;
  if (volume0) *volume0 = m->volume0;
  return ZF_OK;
}

int zf_get_edges(zf_ctx* c, int32_t* edges, uint8_t* area_first) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->mesh_set, "zf_get_edges", "mesh not set");
  const MeshHost* m = (const MeshHost*)c->mesh_host;
  if (edges)
    for (size_t i = 0; i < m->edge.size(); ++i) edges[i] = m->edge[i] + 1;
  if (area_first) std::memcpy(area_first, m->area_first.data(), m->area_first.size());
  return ZF_OK;
}

int zf_get_edge_params(zf_ctx* c, float* epar, float* epar_n, float* tri_area_eq) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->mesh_set, "zf_get_edge_params", "mesh not set");
  const MeshHost* m = (const MeshHost*)c->mesh_host;
  const int ne = m->n_edge, nen = m->n_edge_n;
  if (epar) {
    std::memcpy(epar, m->lmax.data(), ne * sizeof(float));
    std::memcpy(epar + ne, m->plength.data(), ne * sizeof(float));
    std::memcpy(epar + 2 * ne, m->kp.data(), ne * sizeof(float));
    std::memcpy(epar + 3 * ne, m->sin0.data(), ne * sizeof(float));
    std::memcpy(epar + 4 * ne, m->cos0.data(), ne * sizeof(float));
  }
  if (epar_n && nen) {
    std::memcpy(epar_n, m->lmax_n.data(), nen * sizeof(float));
    std::memcpy(epar_n + nen, m->plength_n.data(), nen * sizeof(float));
    std::memcpy(epar_n + 2 * nen, m->kp_n.data(), nen * sizeof(float));
  }
  if (tri_area_eq) std::memcpy(tri_area_eq, m->tri_area_eq.data(), m->n_tri * sizeof(float));
  return ZF_OK;
}

int zf_set_cells(zf_ctx* c, int n_cells, const double* x, const double* xn) {
  if (!c || n_cells < 0 || (n_cells > 0 && !x)) return ZF_ERR_ARG;
  NEED(c->mesh_set, "zf_set_cells", "mesh not set");
  ZF_CUDA(cudaSetDevice(c->device));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  int rc0 = cells_copy_wait_host(c);  // a zf_get_cells_async copy may still read the old buffers
  if (rc0) return rc0;
  free_owned(c->cell_allocs);
  c->adj_gx.clear();  // a position gradient belongs to the cells it was taken for
  c->adj_gxn.clear();
  CellArgs& a = c->cells;
  a.n_cells = n_cells;
  const size_t nc = n_cells, nn = a.nn, nnn = a.nnn, nt = a.nt;
  auto& own = c->cell_allocs;
  int rc;
  if ((rc = upload<double>(c, own, &a.x, x, 3 * nc * nn))) return rc;
  if ((rc = upload<double>(c, own, &a.xn, (nnn && xn) ? xn : nullptr, 3 * nc * nnn))) return rc;
  if ((rc = upload<double>(c, own, &a.vel, nullptr, 3 * nc * nn))) return rc;
  if ((rc = upload<double>(c, own, &a.vel_n, nullptr, 3 * nc * nnn))) return rc;
  if ((rc = upload<float>(c, own, &a.ftot, nullptr, 3 * nc * nn))) return rc;
  if ((rc = upload<float>(c, own, &a.ftot_n, nullptr, 3 * nc * nnn))) return rc;
  if ((rc = upload<float>(c, own, &a.wrep, nullptr, 3 * nc * nn))) return rc;
  if ((rc = upload<float>(c, own, &a.wrep_n, nullptr, 3 * nc * nnn))) return rc;
  if ((rc = upload<float>(c, own, &a.node_normal, nullptr, 3 * nc * nn))) return rc;
  if ((rc = upload<float>(c, own, &a.tri_c, nullptr, 3 * nc * nt))) return rc;
  if ((rc = upload<float>(c, own, &a.tri_nrm, nullptr, 3 * nc * nt))) return rc;
  if ((rc = upload<float>(c, own, &a.tri_a, nullptr, nc * nt))) return rc;
  if ((rc = upload<float>(c, own, &a.cell_f, nullptr, 8 * nc))) return rc;
  std::vector<int32_t> st(nc, 1);
  if ((rc = upload<int32_t>(c, own, &a.status, st.data(), nc))) return rc;
  if ((rc = upload<int32_t>(c, own, &a.caps_remove, nullptr, nc))) return rc;
  if ((rc = upload<unsigned long long>(c, own, &a.counters, nullptr, 4))) return rc;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  c->cells_set = true;
  return ib_prepare(c);  // cell list and nucleus lists sized for these cells
}

int zf_put_cells(zf_ctx* c, const double* x, const double* xn, const int32_t* status) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->cells_set, "zf_put_cells", "cells not set");
  ZF_CUDA(cudaSetDevice(c->device));
  int rc = cells_write_fence(c);  // a pending asynchronous copy still reads the positions
  if (rc) return rc;
  const CellArgs& a = c->cells;
  const size_t nc = a.n_cells;
  if (x) ZF_CUDA(cudaMemcpyAsync(a.x, x, 3 * nc * a.nn * 8, cudaMemcpyHostToDevice, c->stream));
  if (xn && a.nnn) ZF_CUDA(cudaMemcpyAsync(a.xn, xn, 3 * nc * a.nnn * 8, cudaMemcpyHostToDevice, c->stream));
  if (status) ZF_CUDA(cudaMemcpyAsync(a.status, status, nc * 4, cudaMemcpyHostToDevice, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  c->node_tiles_valid = false;  // positions changed
  c->nuc_lists_valid = false;
  return ZF_OK;
}

int zf_get_cells(zf_ctx* c, double* x, double* xn, int32_t* status) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->cells_set, "zf_get_cells", "cells not set");
  const CellArgs& a = c->cells;
  const size_t nc = a.n_cells;
  if (x) ZF_CUDA(cudaMemcpyAsync(x, a.x, 3 * nc * a.nn * 8, cudaMemcpyDeviceToHost, c->stream));
  if (xn && a.nnn)
    ZF_CUDA(cudaMemcpyAsync(xn, a.xn, 3 * nc * a.nnn * 8, cudaMemcpyDeviceToHost, c->stream));
  if (status) ZF_CUDA(cudaMemcpyAsync(status, a.status, nc * 4, cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}


int zf_get_cells_async(zf_ctx* c, double* x, double* xn, int32_t* status) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->cells_set, "zf_get_cells_async", "cells not set");
  if (!c->copy_stream) {
    ZF_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    ZF_CUDA(cudaEventCreateWithFlags(&c->ev_ready, cudaEventDisableTiming));
    ZF_CUDA(cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming));
  }
  const CellArgs& a = c->cells;
  const size_t nc = a.n_cells;
  ZF_CUDA(cudaEventRecord(c->ev_ready, c->stream));
  ZF_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_ready, 0));
  if (x) ZF_CUDA(cudaMemcpyAsync(x, a.x, 3 * nc * a.nn * 8, cudaMemcpyDeviceToHost, c->copy_stream));
  if (xn && a.nnn)
    ZF_CUDA(cudaMemcpyAsync(xn, a.xn, 3 * nc * a.nnn * 8, cudaMemcpyDeviceToHost, c->copy_stream));
  if (status) ZF_CUDA(cudaMemcpyAsync(status, a.status, nc * 4, cudaMemcpyDeviceToHost, c->copy_stream));
  ZF_CUDA(cudaEventRecord(c->ev_copied, c->copy_stream));
  c->copy_pending = true;
  return ZF_OK;
}

int zf_wait_cells(zf_ctx* c) {
  if (!c) return ZF_ERR_ARG;
  if (c->copy_stream) ZF_CUDA(cudaEventSynchronize(c->ev_copied));
  return ZF_OK;
}

int zf_get_cell_forces(zf_ctx* c, float* ftot, float* ftot_n) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->cells_set, "zf_get_cell_forces", "cells not set");
  const CellArgs& a = c->cells;
  const size_t nc = a.n_cells;
  if (ftot) ZF_CUDA(cudaMemcpyAsync(ftot, a.ftot, 3 * nc * a.nn * 4, cudaMemcpyDeviceToHost, c->stream));
  if (ftot_n && a.nnn)
    ZF_CUDA(cudaMemcpyAsync(ftot_n, a.ftot_n, 3 * nc * a.nnn * 4, cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int zf_get_cell_kinematics(zf_ctx* c, double* vel, double* vel_n, float* wrep, float* wrep_n) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->cells_set, "zf_get_cell_kinematics", "cells not set");
  const CellArgs& a = c->cells;
  const size_t nc = a.n_cells;
  if (vel) ZF_CUDA(cudaMemcpyAsync(vel, a.vel, 3 * nc * a.nn * 8, cudaMemcpyDeviceToHost, c->stream));
  if (vel_n && a.nnn)
    ZF_CUDA(cudaMemcpyAsync(vel_n, a.vel_n, 3 * nc * a.nnn * 8, cudaMemcpyDeviceToHost, c->stream));
  if (wrep) ZF_CUDA(cudaMemcpyAsync(wrep, a.wrep, 3 * nc * a.nn * 4, cudaMemcpyDeviceToHost, c->stream));
  if (wrep_n && a.nnn)
    ZF_CUDA(cudaMemcpyAsync(wrep_n, a.wrep_n, 3 * nc * a.nnn * 4, cudaMemcpyDeviceToHost, c->stream));
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int zf_get_cell_geometry(zf_ctx* c, float* tri_area, float* tri_normal, float* tri_centroid,
                         float* node_normal, float* cell_f) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->cells_set, "zf_get_cell_geometry", "cells not set");
  const CellArgs& a = c->cells;
  const size_t nc = a.n_cells;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (dst) ZF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    return ZF_OK;
  };
  int rc;
  if ((rc = cp(tri_area, a.tri_a, nc * a.nt * 4))) return rc;
  if ((rc = cp(tri_normal, a.tri_nrm, 3 * nc * a.nt * 4))) return rc;
  if ((rc = cp(tri_centroid, a.tri_c, 3 * nc * a.nt * 4))) return rc;
  if ((rc = cp(node_normal, a.node_normal, 3 * nc * a.nn * 4))) return rc;
  if ((rc = cp(cell_f, a.cell_f, 8 * nc * 4))) return rc;
  ZF_CUDA(cudaStreamSynchronize(c->stream));
  return ZF_OK;
}

int zf_cgsm_forces(zf_ctx* c) {
  if (!c) return ZF_ERR_ARG;
  NEED(c->cells_set, "zf_cgsm_forces", "cells not set");
  ZF_CUDA(cudaSetDevice(c->device));
  return cells_membrane_launch(c);
}

}  // extern "C"

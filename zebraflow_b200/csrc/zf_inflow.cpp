// Periodic parent segments and cell cloning (the inflow of the reference,
// ZebraflowWT.c:11926-11960 and :12193-12403), as host-side steps between
// membrane iterations.
//
// A parent segment is a periodic stretch of vessel [z0, z1) upstream (flow
// +z, leaving at z1) or downstream-facing (flow -z, leaving at z0) of the
// region of interest, with its own cells ("parents"), run as its own context.
// After every membrane iteration of both contexts:
//   zf_inflow_slaves   the region's clones still slaved to their parent: nodes
//                      not yet 5 DX past the segment's exit plane move with
//                      the parent's node velocity instead of their own; a
//                      clone whose nodes have all passed the exit plane is
//                      released (:11926-11960)
//   zf_inflow_parents  the parents' positions (already moved by the update)
//                      folded back into [z0, z1); a parent in the interior
//                      (status 2) whose node crosses the exit plane is marked
//                      for cloning unless it has regressed; a parent that was
//                      cloned (status 4) is re-armed (status 2) once it lies
//                      inside the segment's window again (:12196-12340)
//   zf_inflow_clone    each marked parent, in order, is copied into the first
//                      free slot of the region (status -5000) with its nodes
//                      made contiguous across the exit plane, and becomes
//                      status 4 (:12347-12403)
// Statuses follow the reference (:256-263): 2 parent in the interior, 4
// parent after cloning; in the region, -(p + 1) a clone slaved to parent p,
// 1 an independent cell, -5000 a free slot.  Positions are [3][cells][nodes]
// in um, as everywhere at the boundary.
#include <cmath>
#include <vector>

#include "zf_internal.h"

namespace {

bool seg_ok(const zf_inflow_segment* s) {
  return s && s->z1 > s->z0 && (s->direction == 1 || s->direction == -1) && s->dx > 0.0;
}

// fold one node's z back into the segment; returns whether it crossed the exit
// plane in the flow direction (:12207-12270)
bool fold(const zf_inflow_segment& s, double& z) {
  const double L = s.z1 - s.z0;
  if (s.direction > 0) {
    if (z >= s.z1) {
      z -= L;
      return true;
    }
    if (z < s.z0) z += L;  // moved backwards across the entry
  } else {
    if (z <= s.z0) {
      z += L;
      return true;
    }
    if (z > s.z1) z -= L;
  }
  return false;
}

}  // namespace

extern "C" {

int zf_inflow_parents(const zf_inflow_segment* seg, int n_parents, int nn, int nnn, double* x, double* xn,
                      int32_t* status, int32_t* regress, int32_t* clone) {
  if (!seg_ok(seg) || n_parents < 0 || nn <= 0 || nnn < 0 || !x || (nnn && !xn) || !status || !regress || !clone)
    return ZF_ERR_ARG;
  const zf_inflow_segment& s = *seg;
  const double L = s.z1 - s.z0;
  const size_t np = (size_t)n_parents;
  for (size_t p = 0; p < np; ++p) {
    clone[p] = 0;
    if (status[p] == 2) {  // :12202-12272
      for (int node = 0; node < nn; ++node)
        if (fold(s, x[(2 * np + p) * nn + node]) && regress[p] == 0) clone[p] = 1;
      for (int node = 0; node < nnn; ++node)
        if (fold(s, xn[(2 * np + p) * nnn + node]) && regress[p] == 0) clone[p] = 1;
    } else if (status[p] == 4) {  // :12274-12337
      regress[p] = 1;
      double zmin = 5000.0, zmax = -5000.0;
      for (int node = 0; node < nn; ++node) {
        double& z = x[(2 * np + p) * nn + node];
        fold(s, z);
        zmax = std::max(zmax, z);
        zmin = std::min(zmin, z);
      }
      for (int node = 0; node < nnn; ++node) fold(s, xn[(2 * np + p) * nnn + node]);
      const bool inside = s.direction > 0 ? (zmin > s.z0 + 5.0 && zmax < s.z0 + 0.75 * L)
                                          : (zmax < s.z1 - 5.0 && zmin > s.z1 - 0.75 * L);
      if (inside) status[p] = 2;
    }
  }
  return ZF_OK;
}

int zf_inflow_clone(const zf_inflow_segment* seg, int n_parents, int nn, int nnn, const double* xp, const double* xnp,
                    int32_t* status_p, int32_t* regress_p, int32_t* clone, int n_slots, double* xr, double* xnr,
                    int32_t* status_r, int32_t* cloned_into) {
  if (!seg_ok(seg) || n_parents < 0 || n_slots < 0 || nn <= 0 || nnn < 0 || !xp || !status_p || !regress_p ||
      !clone || !xr || !status_r || (nnn && (!xnp || !xnr)))
    return ZF_ERR_ARG;
  const zf_inflow_segment& s = *seg;
  const double L = s.z1 - s.z0, mid = 0.5 * (s.z0 + s.z1);
  const size_t np = (size_t)n_parents, nr = (size_t)n_slots;
  // the clone's nodes on the entry side of the middle go one period on, so the
  // clone is whole across the exit plane (:12361-12387)
  auto place = [&](double z) {
    if (s.direction > 0 && z < mid) return z + L;
    if (s.direction < 0 && z > mid) return z - L;
    return z;
  };
  for (size_t p = 0; p < np; ++p) {
    if (cloned_into) cloned_into[p] = -1;
    if (clone[p] <= 0) continue;
    for (size_t m = 0; m < nr; ++m) {
      if (status_r[m] != -5000) continue;
      status_r[m] = -(int32_t)(p + 1);
      for (int c = 0; c < 3; ++c)
        for (int node = 0; node < nn; ++node) {
          const double v = xp[((size_t)c * np + p) * nn + node];
          xr[((size_t)c * nr + m) * nn + node] = c == 2 ? place(v) : v;
        }
      for (int c = 0; c < 3; ++c)
        for (int node = 0; node < nnn; ++node) {
          const double v = xnp[((size_t)c * np + p) * nnn + node];
          xnr[((size_t)c * nr + m) * nnn + node] = c == 2 ? place(v) : v;
        }
      if (cloned_into) cloned_into[p] = (int32_t)m;
      break;
    }
    // the parent is marked cloned even when no slot was free (:12398-12400)
    status_p[p] = 4;
    clone[p] = 0;
    regress_p[p] = 1;
  }
  return ZF_OK;
}

int zf_inflow_slaves(const zf_inflow_segment* seg, double dt_stagger, int n_slots, int nn, int nnn, double* xr,
                     double* xnr, const double* vr, const double* vnr, int32_t* status_r, int n_parents,
                     const double* vp, const double* vnp) {
  if (!seg_ok(seg) || n_slots < 0 || n_parents < 0 || nn <= 0 || nnn < 0 || !xr || !vr || !status_r || !vp ||
      (nnn && (!xnr || !vnr || !vnp)))
    return ZF_ERR_ARG;
  const zf_inflow_segment& s = *seg;
  const size_t nr = (size_t)n_slots, np = (size_t)n_parents;
  // a node 5 DX past the exit plane moves with its own velocity (:11937-11940)
  auto past = [&](double z) {
    return s.direction > 0 ? z > s.z1 + 5.0 * s.dx : z < s.z0 - 5.0 * s.dx;
  };
  for (size_t m = 0; m < nr; ++m) {
    if (!(status_r[m] < 0 && status_r[m] > -4998)) continue;
    const size_t p = (size_t)(-status_r[m] - 1);
    if (p >= np) return ZF_ERR_ARG;
    double zmin = 5000.0, zmax = -5000.0;
    // the region's update moved every node with its own velocity; a node that
    // was not yet past the plane takes its parent's instead.  The reference
    // tests the position before the move; x - v dt recovers it.
    for (int node = 0; node < nn; ++node) {
      const double z_old = xr[(2 * nr + m) * nn + node] - vr[(2 * nr + m) * nn + node] * dt_stagger;
      if (!past(z_old))
        for (int c = 0; c < 3; ++c) {
          const size_t g = ((size_t)c * nr + m) * nn + node;
          xr[g] += (vp[((size_t)c * np + p) * nn + node] - vr[g]) * dt_stagger;
        }
      const double z = xr[(2 * nr + m) * nn + node];
      zmax = std::max(zmax, z);
      zmin = std::min(zmin, z);
    }
    for (int node = 0; node < nnn; ++node) {
      const double z_old = xnr[(2 * nr + m) * nnn + node] - vnr[(2 * nr + m) * nnn + node] * dt_stagger;
      if (!past(z_old))
        for (int c = 0; c < 3; ++c) {
          const size_t g = ((size_t)c * nr + m) * nnn + node;
          xnr[g] += (vnp[((size_t)c * np + p) * nnn + node] - vnr[g]) * dt_stagger;
        }
    }
    // released once every node has crossed the exit plane (:11958-11960)
    if (s.direction > 0 ? zmin > s.z1 : zmax < s.z0) status_r[m] = 1;
  }
  return ZF_OK;
}

}  // extern "C"

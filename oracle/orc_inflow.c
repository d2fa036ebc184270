/* ORACLE — test infrastructure only.  The reference's inflow steps restated
 * in C for one parent segment (ZebraflowWT.c:11926-11960, :12193-12403), in
 * the reference's own order within each step: the position update x += v DT
 * SOLVERSTAGGER is part of each block, as there.  The reference hard-codes
 * three segments by cell-id range (1-188 flowing +z and leaving at ZM_1,
 * 189-329 and 330-344 flowing -z and leaving at Z0_2, Z0_3); here one segment
 * [z0, z1) with its direction stands for any of them.  Layouts [3][cells][nodes]
 * (0-based), fp64 as NODECOORD.  Statuses as the reference's (:256-263). */
#include <stddef.h>
#include <stdint.h>

#define V3(a, n, c, cell, node, nc) (a)[((size_t)(c) * (nc) + (cell)) * (n) + (node)]

/* ROI update of the clones still slaved to their parent (:11926-11960) and of
 * the independent cells (:11962-, the plain update only).  Slave m belongs to
 * parent -status[m] - 1. */
void orc_inflow_roi_update(double z0, double z1, int dir, double dx, double dt, int nr, int nn, int nnn, double* x,
                           double* xn, const double* v, const double* vn, int32_t* status, int np,
                           const double* vp, const double* vnp) {
  for (int m = 0; m < nr; ++m) {
    if (status[m] < 0 && status[m] > -4998) {
      const int p = -status[m] - 1;
      double nzmax = -5000., nzmin = 5000.;
      for (int node = 0; node < nn; ++node) {
        int check = 0;
        if (dir > 0 && V3(x, nn, 2, m, node, nr) > z1 + 5. * dx) check = 1;
        if (dir < 0 && V3(x, nn, 2, m, node, nr) < z0 - 5. * dx) check = 1;
        for (int i = 0; i <= 2; ++i) {
          const double vel = check == 0 ? V3(vp, nn, i, p, node, np) : V3(v, nn, i, m, node, nr);
          V3(x, nn, i, m, node, nr) += vel * dt;
        }
        if (V3(x, nn, 2, m, node, nr) > nzmax) nzmax = V3(x, nn, 2, m, node, nr);
        if (V3(x, nn, 2, m, node, nr) < nzmin) nzmin = V3(x, nn, 2, m, node, nr);
      }
      for (int node = 0; node < nnn; ++node) {
        int check = 0;
        if (dir > 0 && V3(xn, nnn, 2, m, node, nr) > z1 + 5. * dx) check = 1;
        if (dir < 0 && V3(xn, nnn, 2, m, node, nr) < z0 - 5. * dx) check = 1;
        for (int i = 0; i <= 2; ++i) {
          const double vel = check == 0 ? V3(vnp, nnn, i, p, node, np) : V3(vn, nnn, i, m, node, nr);
          V3(xn, nnn, i, m, node, nr) += vel * dt;
        }
      }
      /* fully across the cloning line (:11958-11960; the line is the exit plane) */
      if (dir > 0 ? nzmin > z1 : nzmax < z0) status[m] = 1;
    } else if (status[m] == 1) {
      for (int i = 0; i <= 2; ++i) {
        for (int node = 0; node < nn; ++node) V3(x, nn, i, m, node, nr) += V3(v, nn, i, m, node, nr) * dt;
        for (int node = 0; node < nnn; ++node) V3(xn, nnn, i, m, node, nr) += V3(vn, nnn, i, m, node, nr) * dt;
      }
    }
  }
}

/* parent update with the periodic fold and the clone flags (:12196-12340) */
static void orc_fold(double z0, double z1, int dir, double* z, int* crossed) {
  const double L = z1 - z0;
  *crossed = 0;
  if (dir > 0) {
    if (*z >= z1) {
      *crossed = 1;
      *z = *z - L;
    } else if (*z < z0) {
      *z = *z + L;
    }
  } else {
    if (*z <= z0) {
      *crossed = 1;
      *z = *z + L;
    } else if (*z > z1) {
      *z = *z - L;
    }
  }
}

void orc_inflow_parent_update(double z0, double z1, int dir, double dt, int np, int nn, int nnn, double* x,
                              double* xn, const double* v, const double* vn, int32_t* status, int32_t* regress,
                              int32_t* cloneflag) {
  const double L = z1 - z0;
  for (int p = 0; p < np; ++p) {
    cloneflag[p] = 0;
    if (status[p] == 2) {
      for (int node = 0; node < nn; ++node) {
        for (int i = 0; i <= 2; ++i) V3(x, nn, i, p, node, np) += V3(v, nn, i, p, node, np) * dt;
        int crossed;
        orc_fold(z0, z1, dir, &V3(x, nn, 2, p, node, np), &crossed);
        if (crossed && regress[p] == 0) cloneflag[p] = 1;
      }
      for (int node = 0; node < nnn; ++node) {
        for (int i = 0; i <= 2; ++i) V3(xn, nnn, i, p, node, np) += V3(vn, nnn, i, p, node, np) * dt;
        int crossed;
        orc_fold(z0, z1, dir, &V3(xn, nnn, 2, p, node, np), &crossed);
        if (crossed && regress[p] == 0) cloneflag[p] = 1;
      }
    } else if (status[p] == 4) {
      double nzmax = -5000., nzmin = 5000.;
      regress[p] = 1;
      for (int node = 0; node < nn; ++node) {
        for (int i = 0; i <= 2; ++i) V3(x, nn, i, p, node, np) += V3(v, nn, i, p, node, np) * dt;
        int crossed;
        orc_fold(z0, z1, dir, &V3(x, nn, 2, p, node, np), &crossed);
        if (V3(x, nn, 2, p, node, np) > nzmax) nzmax = V3(x, nn, 2, p, node, np);
        if (V3(x, nn, 2, p, node, np) < nzmin) nzmin = V3(x, nn, 2, p, node, np);
      }
      for (int node = 0; node < nnn; ++node) {
        for (int i = 0; i <= 2; ++i) V3(xn, nnn, i, p, node, np) += V3(vn, nnn, i, p, node, np) * dt;
        int crossed;
        orc_fold(z0, z1, dir, &V3(xn, nnn, 2, p, node, np), &crossed);
      }
      if (dir > 0) {
        if (nzmin > (z0 + 5.) && nzmax < (z0 + 0.75 * L)) status[p] = 2;
      } else {
        if (nzmax < (z1 - 5.) && nzmin > (z1 - 0.75 * L)) status[p] = 2;
      }
    }
  }
}

/* serial cloning into the first free slot (:12347-12403) */
void orc_inflow_clone(double z0, double z1, int dir, int np, int nn, int nnn, const double* xp, const double* xnp,
                      int32_t* status_p, int32_t* regress_p, int32_t* cloneflag, int nr, double* xr, double* xnr,
                      int32_t* status_r) {
  const double L = z1 - z0, mid = 0.5 * (z0 + z1);
  for (int p = 0; p < np; ++p) {
    if (cloneflag[p] > 0) {
      for (int m = 0; m < nr; ++m) {
        if (status_r[m] == -5000) {
          status_r[m] = -(p + 1);
          for (int node = 0; node < nn; ++node) {
            for (int i = 0; i <= 2; ++i) V3(xr, nn, i, m, node, nr) = V3(xp, nn, i, p, node, np);
            if (dir > 0 && V3(xr, nn, 2, m, node, nr) < mid) V3(xr, nn, 2, m, node, nr) += L;
            else if (dir < 0 && V3(xr, nn, 2, m, node, nr) > mid) V3(xr, nn, 2, m, node, nr) += -L;
          }
          for (int node = 0; node < nnn; ++node) {
            for (int i = 0; i <= 2; ++i) V3(xnr, nnn, i, m, node, nr) = V3(xnp, nnn, i, p, node, np);
            if (dir > 0 && V3(xnr, nnn, 2, m, node, nr) < mid) V3(xnr, nnn, 2, m, node, nr) += L;
            else if (dir < 0 && V3(xnr, nnn, 2, m, node, nr) > mid) V3(xnr, nnn, 2, m, node, nr) += -L;
          }
          break;
        }
      }
      status_p[p] = 4;
      cloneflag[p] = 0;
      regress_p[p] = 1;
    }
  }
}

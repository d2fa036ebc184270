"""Periodic parent segments feeding cells into the region of interest (the
reference's inflow, ZebraflowWT.c:11926-11960 and :12193-12403).

A parent segment is its own context: a periodic stretch of vessel holding the
parent cells, stepped with the region's context in lockstep.  After every
membrane iteration of both, the host steps of include/zf.h
(zf_inflow_slaves, zf_inflow_parents, zf_inflow_clone) run in the reference's
order: the region's slaved clones take their parent's velocity, the parents
are folded back into their segment (a parent crossing the exit plane is marked
for cloning), and each marked parent is copied into a free slot of the region.
Slaved clones are ordinary active cells on the GPU (forces, IB coupling,
repulsions); only their motion near the exit plane follows the parent.
"""
import ctypes as C

import numpy as np

from . import lib, _check, _ptr


class Segment(C.Structure):
    """zf_inflow_segment: periodic over [z0, z1) um, flow leaving at z1
    (direction +1) or z0 (-1), lattice spacing dx um."""
    _fields_ = [("z0", C.c_double), ("z1", C.c_double), ("direction", C.c_int32), ("dx", C.c_double)]


def _f64(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a


def _i32(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a


def slaves(seg, dt_stagger, xr, xnr, vr, vnr, status_r, vp, vnp):
    """zf_inflow_slaves on host arrays (in place: xr, xnr, status_r)."""
    nr, nn = xr.shape[1], xr.shape[2]
    nnn = xnr.shape[2] if xnr is not None else 0
    _check(lib().zf_inflow_slaves(C.byref(seg), float(dt_stagger), nr, nn, nnn, _ptr(_f64(xr)),
                                  _ptr(None if xnr is None else _f64(xnr)), _ptr(_f64(vr)),
                                  _ptr(None if vnr is None else _f64(vnr)), _ptr(_i32(status_r)), vp.shape[1],
                                  _ptr(_f64(vp)), _ptr(None if vnp is None else _f64(vnp))))


def parents(seg, x, xn, status, regress, clone):
    """zf_inflow_parents on host arrays (in place)."""
    np_, nn = x.shape[1], x.shape[2]
    nnn = xn.shape[2] if xn is not None else 0
    _check(lib().zf_inflow_parents(C.byref(seg), np_, nn, nnn, _ptr(_f64(x)), _ptr(None if xn is None else _f64(xn)),
                                   _ptr(_i32(status)), _ptr(_i32(regress)), _ptr(_i32(clone))))


def clone(seg, xp, xnp, status_p, regress_p, clone_p, xr, xnr, status_r):
    """zf_inflow_clone on host arrays (in place); returns cloned_into [parents]."""
    np_, nn = xp.shape[1], xp.shape[2]
    nnn = xnp.shape[2] if xnp is not None else 0
    into = np.empty(np_, np.int32)
    _check(lib().zf_inflow_clone(C.byref(seg), np_, nn, nnn, _ptr(_f64(xp)), _ptr(None if xnp is None else _f64(xnp)),
                                 _ptr(_i32(status_p)), _ptr(_i32(regress_p)), _ptr(_i32(clone_p)), xr.shape[1],
                                 _ptr(_f64(xr)), _ptr(None if xnr is None else _f64(xnr)), _ptr(_i32(status_r)),
                                 _ptr(into)))
    return into


class Inflow:
    """A parent-segment context feeding a region context.

    parent, region: Contexts with the same membrane mesh and stagger; the
    parents are all cells of `parent` (host status 2 at the start), the
    region's cells are slots (host status 1 for cells, -5000 for free slots,
    `free`: a boolean mask of the free ones).  seg: the parent segment in the
    frame both contexts share."""

    def __init__(self, parent, region, seg, free, dt_stagger):
        self.parent, self.region, self.seg, self.dt = parent, region, seg, float(dt_stagger)
        self.status_p = np.full(parent.nc, 2, np.int32)
        self.regress_p = np.zeros(parent.nc, np.int32)
        self.clone_p = np.zeros(parent.nc, np.int32)
        self.status_r = np.where(np.asarray(free, bool), -5000, 1).astype(np.int32)
        self.stagger = parent.params.stagger
        region.put_cells(status=self._gpu_status())
        self.clones = 0

    def _gpu_status(self):
        return np.where(self.status_r == -5000, -5000, 1).astype(np.int32)

    def after_membrane(self):
        """The host steps after a membrane iteration of both contexts."""
        P, R = self.parent, self.region
        xp, xnp, _ = P.cells()
        vp, vnp, _, _ = P.cell_kinematics()
        xr, xnr, st = R.cells()
        vr, vnr, _, _ = R.cell_kinematics()
        self.status_r[st <= -5000] = -5000  # removed on the GPU (screening, speed check)
        slaves(self.seg, self.dt, xr, xnr, vr, vnr, self.status_r, vp, vnp)
        parents(self.seg, xp, xnp, self.status_p, self.regress_p, self.clone_p)
        into = clone(self.seg, xp, xnp, self.status_p, self.regress_p, self.clone_p, xr, xnr, self.status_r)
        self.clones += int((into >= 0).sum())
        P.put_cells(xp, xnp)
        R.put_cells(xr, xnr, self._gpu_status())

    def step(self, n):
        """n iterations of both contexts, the host steps after each membrane
        iteration."""
        for _ in range(n):
            self.parent.step(1)
            self.region.step(1)
            if self.parent.iteration() % self.stagger == 0:
                self.after_membrane()

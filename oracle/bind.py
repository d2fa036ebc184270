"""ORACLE — test infrastructure only: ctypes binding of oracle/liboracle.so.

Each function cites the C restatement it wraps; the restatement cites the
reference lines it follows (ZebraflowWT.c).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        for s in ("_f32", "_f64"):
            g = lambda n: getattr(L, n + s)  # noqa: E731
            g("orc_lbm_create").restype = C.c_void_p
            g("orc_lbm_create").argtypes = [C.c_int, C.c_int, C.c_int, _i32p, C.c_int, _i32p,
                                            C.c_double, C.c_int, C.c_double, _f64p, C.c_int]
            g("orc_lbm_destroy").argtypes = [C.c_void_p]
            g("orc_lbm_n_listed").restype = C.c_int64
            g("orc_lbm_n_listed").argtypes = [C.c_void_p]
            for n in ("orc_lbm_set_f", "orc_lbm_get_f", "orc_lbm_set_bodyforce",
                      "orc_lbm_get_bodyforce"):
                g(n).argtypes = [C.c_void_p, _f64p]
            g("orc_lbm_get_moments").argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p]
            g("orc_lbm_step").argtypes = [C.c_void_p, C.c_int]
            g("orc_lbm_mass").restype = C.c_double
            g("orc_lbm_mass").argtypes = [C.c_void_p, C.c_int]
            g("orc_lbm_set_storage_emulation").argtypes = [C.c_void_p, C.c_int, C.c_double,
                                                           C.c_double]
            g("orc_lbm_get_dom").argtypes = [C.c_void_p, _i32p, _i32p]
            g("orc_lbm_time_steps").restype = C.c_double
            g("orc_lbm_time_steps").argtypes = [C.c_void_p, C.c_int]
            g("orc_cells_create").restype = C.c_void_p
            g("orc_cells_create").argtypes = [C.c_int, C.c_int, _i32p, _f64p, C.c_int, C.c_int,
                                              _i32p, _f64p, _f64p]
            g("orc_cells_num_edges").restype = C.c_int
            g("orc_cells_num_edges").argtypes = [C.c_void_p]
            g("orc_cells_topology").argtypes = [C.c_void_p, _i32p, _f64p, _f64p, _f64p, _f64p]
            g("orc_cells_set").argtypes = [C.c_void_p, C.c_int, _f64p, _f64p]
            g("orc_cells_forces").argtypes = [C.c_void_p]
            g("orc_cells_get").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
            g("orc_cells_geometry").argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p]
            g("orc_cells_destroy").argtypes = [C.c_void_p]
            g("orc_world_create").restype = C.c_void_p
            g("orc_world_create").argtypes = [C.c_void_p, C.c_void_p, _f64p, C.c_double, _f64p]
            g("orc_world_set_wall").argtypes = [C.c_void_p, C.c_int, _f32p, C.c_int, _i32p, _f32p,
                                                C.c_int]
            g("orc_world_get_wall").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
            for n in ("orc_world_interp", "orc_world_rbc_rbc", "orc_world_spread",
                      "orc_world_update", "orc_world_destroy"):
                g(n).argtypes = [C.c_void_p]
            g("orc_world_nuc_memb").argtypes = [C.c_void_p, C.c_int]
            g("orc_world_set_exact").argtypes = [C.c_void_p, C.c_int]
            g("orc_world_step").argtypes = [C.c_void_p, C.c_int]
            g("orc_world_kinematics").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p]
            g("orc_world_wss").argtypes = [C.c_void_p, _f32p, C.c_double, _f64p, C.c_void_p,
                                           C.c_void_p]
            g("orc_lbm_moments_from_f").argtypes = [C.c_void_p]
            g("orc_lbm_set_iter").argtypes = [C.c_void_p, C.c_int64]
        # the inflow steps (one precision: fp64 positions, as the reference's)
        L.orc_inflow_roi_update.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int,
                                            C.c_int, C.c_int] + [C.c_void_p] * 5 + [C.c_int] + [C.c_void_p] * 2
        L.orc_inflow_parent_update.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int,
                                               C.c_int] + [C.c_void_p] * 7
        L.orc_inflow_clone.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int] + \
            [C.c_void_p] * 5 + [C.c_int] + [C.c_void_p] * 3
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_inputs = None


def inputs():
    """The workload generators and reference parameter defaults compiled into
    this library (orc_gen.cpp), with the interface of zebraflow_b200.inputs():
    a CPU run builds the same inputs as the GPU library without loading it."""
    global _inputs
    if _inputs is None:
        import sys
        root = os.path.dirname(_HERE)
        if root not in sys.path:
            sys.path.insert(0, root)
        from zebraflow_b200 import Inputs  # the ctypes binding class only; libzf.so is not loaded
        _inputs = Inputs(lib(), "orc_")
    return _inputs


class OracleCells:
    """Reference membrane set-up and membrane step (ZebraflowWT.c:1592-2460,
    :5704-7535) restated in C; see oracle/orc_cells.inc."""

    def __init__(self, rest, tri1, rest_n, edge_n1, params, precision="f64"):
        """params: a zebraflow_b200 Params (moduli, kT, e_ratio_eq, area0/volume0,
        calibration passes, removal count are read from it)."""
        self.sfx = "_f32" if precision == "f32" else "_f64"
        self._fn = lambda n: getattr(lib(), n + self.sfx)  # noqa: E731
        rest = np.ascontiguousarray(rest, np.float64).ravel()
        tri1 = np.ascontiguousarray(tri1, np.int32).ravel()
        rest_n = np.ascontiguousarray(rest_n, np.float64).ravel()
        edge_n1 = np.ascontiguousarray(edge_n1, np.int32).ravel()
        self.nn, self.nt = rest.size // 3, tri1.size // 3
        self.nnn, self.nen = rest_n.size // 3, edge_n1.size // 2
        P = params
        par = np.array([P.Es, P.Es_nucleus_ratio, P.kbend, P.kd, P.ka, P.kv, P.kT, P.e_ratio_eq,
                        P.area0, P.volume0, P.calib_passes, P.remove_count], np.float64)
        self._h = self._fn("orc_cells_create")(self.nn, self.nt, tri1, rest, self.nnn, self.nen,
                                                edge_n1, rest_n, par)
        self.ne = int(self._fn("orc_cells_num_edges")(self._h))
        self.nc = 0

    def topology(self):
        e = np.empty(6 * self.ne, np.int32)
        ep = np.empty(5 * self.ne)
        epn = np.empty(max(3 * self.nen, 1))
        ae = np.empty(self.nt)
        av = np.empty(2)
        self._fn("orc_cells_topology")(self._h, e, ep, epn, ae, av)
        return (e.reshape(self.ne, 6), ep.reshape(5, self.ne),
                epn[:3 * self.nen].reshape(3, self.nen), ae, av)

    def set_cells(self, x, xn):
        x = np.ascontiguousarray(x, np.float64)
        self.nc = x.shape[1]
        self._fn("orc_cells_set")(self._h, self.nc, x.ravel(),
                                  np.ascontiguousarray(xn, np.float64).ravel())

    def forces(self):
        self._fn("orc_cells_forces")(self._h)

    def get(self):
        x = np.empty((3, self.nc, self.nn))
        xn = np.empty((3, self.nc, self.nnn))
        f = np.empty((3, self.nc, self.nn))
        fn = np.empty((3, self.nc, self.nnn))
        cf = np.empty((self.nc, 8))
        st = np.empty(self.nc, np.int32)
        cnt = np.zeros(2, np.int64)
        self._fn("orc_cells_get")(self._h, _p(x), _p(xn), _p(f), _p(fn), _p(cf), _p(st), _p(cnt))
        return dict(x=x, xn=xn, ftot=f, ftot_n=fn, cell=cf, status=st, counters=cnt)

    def geometry(self):
        ta = np.empty((self.nc, self.nt))
        tn = np.empty((3, self.nc, self.nt))
        tc = np.empty((3, self.nc, self.nt))
        nn_ = np.empty((3, self.nc, self.nn))
        self._fn("orc_cells_geometry")(self._h, ta, tn, tc, nn_)
        return ta, tn, tc, nn_

    def close(self):
        if self._h:
            self._fn("orc_cells_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleLBM:
    """The reference LBM step (ZebraflowWT.c:6100-6145, :6290-6315, :6599-6626)
    restated in C with fp32 (``precision='f32'``) or fp64 arithmetic."""

    def __init__(self, b_index, wall_mode=0, periodic=(0, 0, 0), tau=0.9, tau_from_phase=False,
                 dt=0.5, g=(0.0, 0.0, 0.0), precision="f64", faithful=False):
        b = np.ascontiguousarray(b_index, np.int32)
        nx, ny, nz = b.shape
        self.sfx = "_f32" if precision == "f32" else "_f64"
        self._fn = lambda n: getattr(lib(), n + self.sfx)  # noqa: E731
        self._h = self._fn("orc_lbm_create")(
            nx, ny, nz, b.ravel(), int(wall_mode), np.asarray(periodic, np.int32), float(tau),
            int(tau_from_phase), float(dt), np.asarray(g, np.float64), int(faithful))
        self.n = int(self._fn("orc_lbm_n_listed")(self._h))

    def close(self):
        if self._h:
            self._fn("orc_lbm_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_f(self, f):
        self._fn("orc_lbm_set_f")(self._h, np.ascontiguousarray(f, np.float64).ravel())

    def get_f(self):
        out = np.empty(19 * self.n)
        self._fn("orc_lbm_get_f")(self._h, out)
        return out.reshape(19, self.n)

    def set_bodyforce(self, bf):
        self._fn("orc_lbm_set_bodyforce")(self._h, np.ascontiguousarray(bf, np.float64).ravel())

    def get_bodyforce(self):
        out = np.empty(3 * self.n)
        self._fn("orc_lbm_get_bodyforce")(self._h, out)
        return out.reshape(3, self.n)

    def moments_from_f(self):
        """Recomputes D, U, V, W from the current populations."""
        self._fn("orc_lbm_moments_from_f")(self._h)

    def set_iter(self, it):
        """Completed steps; the next step is iteration it + 1 (pressure inlets' time)."""
        self._fn("orc_lbm_set_iter")(self._h, int(it))

    def moments(self):
        outs = [np.empty(self.n) for _ in range(4)]
        self._fn("orc_lbm_get_moments")(self._h, *outs)
        return outs

    def step(self, rbc_flag=False):
        self._fn("orc_lbm_step")(self._h, int(rbc_flag))

    def dom(self):
        """(listed points [n][3] 0-based, designated neighbour per point or -1)."""
        d = np.empty(3 * self.n, np.int32)
        nb = np.empty(self.n, np.int32)
        self._fn("orc_lbm_get_dom")(self._h, d, nb)
        return d.reshape(self.n, 3), nb

    def set_storage_emulation(self, mode, scale=65536.0, rho_ref=1.0):
        """Rounds the stored populations after every step as a storage form
        would: 0 none, 1 raw fp32, 2 fp32 deviation, 3 fp16 deviation,
        4 bf16 deviation (deviation d = f/w - rho_ref, stored as scale*d)."""
        self._fn("orc_lbm_set_storage_emulation")(self._h, int(mode), float(scale), float(rho_ref))

    def mass(self, include_walls=False):
        return float(self._fn("orc_lbm_mass")(self._h, int(include_walls)))

    def time_steps(self, n):
        return float(self._fn("orc_lbm_time_steps")(self._h, int(n)))


class OracleWorld:
    """The reference IB coupling and time loop (ZebraflowWT.c:5646-12190) over an
    OracleLBM and an OracleCells of the same precision; see oracle/orc_ib.inc."""

    def __init__(self, lbm: OracleLBM, cells, params):
        """cells may be None for wall-only use (set_wall, wss)."""
        assert cells is None or lbm.sfx == cells.sfx
        self.lbm, self.cells, self.sfx = lbm, cells, lbm.sfx
        self._fn = lambda n: getattr(lib(), n + self.sfx)  # noqa: E731
        P = params
        par = np.array([P.gamma_p, P.unit_mass, P.bforce_scale, P.vel_scale, P.dt, P.vmax_remove,
                        P.stagger, P.nuc_list_period, P.nuc_list_max], np.float64)
        self._h = self._fn("orc_world_create")(lbm._h, cells._h if cells is not None else None,
                                               np.asarray(P.origin[:], np.float64), float(P.dx), par)
        self.wall_cap = P.wall_list_max

    def set_wall(self, xyz, tri, nrm):
        xyz = np.ascontiguousarray(xyz, np.float32)
        tri = np.ascontiguousarray(tri, np.int32)
        nrm = np.ascontiguousarray(nrm, np.float32)
        self._fn("orc_world_set_wall")(self._h, xyz.shape[1], xyz.ravel(), tri.shape[1], tri.ravel(),
                                       nrm.ravel(), int(self.wall_cap))

    def wall_index(self, shape):
        n = int(np.prod(shape))
        wi = np.empty(n, np.int32)
        uv = np.empty(3 * n, np.float32)
        self._fn("orc_world_get_wall")(self._h, _p(wi), _p(uv))
        return wi.reshape(shape), uv.reshape((3,) + tuple(shape))

    def set_exact(self, on=True):
        """Interpolation and spreading weights from the fp64 positions instead of
        the reference's fp32 ones: the forward becomes smooth in the positions
        below fp32 resolution, as finite-difference checks of position
        derivatives need."""
        self._fn("orc_world_set_exact")(self._h, int(bool(on)))

    def interp(self):
        self._fn("orc_world_interp")(self._h)

    def nuc_memb(self, rebuild=False):
        self._fn("orc_world_nuc_memb")(self._h, int(rebuild))

    def rbc_rbc(self):
        self._fn("orc_world_rbc_rbc")(self._h)

    def spread(self):
        self._fn("orc_world_spread")(self._h)

    def update(self):
        self._fn("orc_world_update")(self._h)

    def step(self, n=1):
        self._fn("orc_world_step")(self._h, int(n))

    def wss(self, node_normals, pgauge=120.0):
        """WSS [3][nw] (Pa), pressure [nw] (Pa) and valid flags [nw] from the
        LBM's current moments (PostProWSSandPressure.c:275-369)."""
        nrm = np.ascontiguousarray(node_normals, np.float32)
        nw = nrm.shape[1]
        wss = np.empty(3 * nw, np.float64)
        press = np.empty(nw, np.float64)
        valid = np.empty(nw, np.int32)
        self._fn("orc_world_wss")(self._h, nrm.ravel(), float(pgauge), wss, _p(press), _p(valid))
        return wss.reshape(3, nw), press, valid

    def kinematics(self):
        c = self.cells
        v = np.empty((3, c.nc, c.nn))
        vn = np.empty((3, c.nc, c.nnn))
        w = np.empty((3, c.nc, c.nn))
        wn = np.empty((3, c.nc, c.nnn))
        self._fn("orc_world_kinematics")(self._h, _p(v), _p(vn), _p(w), _p(wn))
        return v, vn, w, wn

    def close(self):
        if self._h:
            self._fn("orc_world_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

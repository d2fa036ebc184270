"""zebraflow_b200 — B200-native Zebraflow coupled LBM-IB-RBC time step.

The product is the C ABI of ``include/zf.h`` implemented by ``libzf.so``
(hand-written sm_100a CUDA kernels plus C++ host setup).  This module is a
thin ctypes mirror of that ABI for Python callers (tests, benchmarks); it
does no numerics of its own and raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzf.so")

ZF_OK, ZF_ERR_CUDA, ZF_ERR_ARG, ZF_ERR_OVERFLOW, ZF_ERR_NONFINITE, ZF_ERR_STATE, ZF_ERR_NOMEM = range(7)
WALL_HALFWAY_BB, WALL_REF_EQ = 0, 1
STORE_F32, STORE_F16, STORE_BF16, STORE_F32_DEV = 0, 1, 2, 3
Q = 19

# D3Q19 in the reference order (ZebraflowWT.c:2471-2497); slot q = reference c-1.
E = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [-1, -1, 0], [-1, 1, 0], [1, -1, 0], [1, 0, 1], [-1, 0, -1],
              [-1, 0, 1], [1, 0, -1], [0, 1, 1], [0, -1, -1], [0, -1, 1], [0, 1, -1],
              [0, 0, 0]], dtype=np.int32)
W = np.array([1 / 18] * 6 + [1 / 36] * 12 + [1 / 3])


class ZfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"zf error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("origin", C.c_double * 3), ("dx", C.c_double), ("dt", C.c_double),
        ("tau", C.c_float), ("tau_from_phase", C.c_int32), ("g", C.c_float * 3),
        ("wall_mode", C.c_int32), ("periodic", C.c_int32 * 3), ("storage", C.c_int32),
        ("rho_ref", C.c_float), ("stagger", C.c_int32),
        ("Es", C.c_double), ("Es_nucleus_ratio", C.c_double), ("kbend", C.c_double),
        ("kd", C.c_double), ("ka", C.c_double), ("kv", C.c_double),
        ("area0", C.c_double), ("volume0", C.c_double), ("kT", C.c_double),
        ("e_ratio_eq", C.c_double), ("calib_passes", C.c_int32), ("gamma_p", C.c_double),
        ("unit_mass", C.c_double), ("bforce_scale", C.c_double), ("vel_scale", C.c_double),
        ("vmax_remove", C.c_double), ("remove_count", C.c_int32),
        ("nuc_list_period", C.c_int32), ("nuc_list_max", C.c_int32),
        ("stochastic_round", C.c_int32), ("wall_list_max", C.c_int32),
    ]


class Status(C.Structure):
    _fields_ = [("screened_terms", C.c_int64), ("cells_removed", C.c_int64),
                ("list_overflows", C.c_int64), ("bc_no_neighbour", C.c_int64),
                ("iter", C.c_int64)]


_P = C.c_void_p
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")

# name -> (restype, argtypes)
_SIGS = {
    "zf_params_size": (C.c_size_t, []),
    "zf_create": (_P, [C.POINTER(Params), C.c_int]),
    "zf_destroy": (None, [_P]),
    "zf_last_error": (C.c_char_p, []),
    "zf_sync": (C.c_int, [_P]),
    "zf_get_status": (C.c_int, [_P, C.POINTER(Status)]),
    "zf_set_lattice": (C.c_int, [_P, _i32p]),
    "zf_num_listed": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "zf_get_domlist": (C.c_int, [_P, _i32p]),
    "zf_upload_populations": (C.c_int, [_P, _f32p]),
    "zf_download_populations": (C.c_int, [_P, _f32p]),
    "zf_upload_bodyforce": (C.c_int, [_P, _f32p]),
    "zf_download_bodyforce": (C.c_int, [_P, _f32p]),
    "zf_download_moments": (C.c_int, [_P, _f32p, _f32p, _f32p, _f32p]),
    "zf_lbm_step": (C.c_int, [_P, C.c_int, C.c_int]),
    "zf_lbm_steps": (C.c_int, [_P, C.c_int]),
    "zf_lbm_step_mass": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "zf_lbm_step_mass_noalloc": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "zf_set_uniform_force": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "zf_set_stream": (C.c_int, [_P, C.c_void_p]),
    "zf_mass": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double)]),
    "zf_lbm_steps_timed": (C.c_int, [_P, C.c_int, C.POINTER(C.c_float)]),
    "zf_device_bytes": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "zf_set_mesh": (C.c_int, [_P, C.c_int, C.c_int, _i32p, _f64p, C.c_int, C.c_int, _i32p, _f64p]),
    "zf_mesh_info": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                               C.POINTER(C.c_double)]),
    "zf_get_edges": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "zf_get_edge_params": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_set_cells": (C.c_int, [_P, C.c_int, _f64p, C.c_void_p]),
    "zf_get_cells": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_get_cells_async": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_set_slab": (C.c_int, [_P, C.c_int, C.c_int]),
    "zf_lbm_step_part": (C.c_int, [_P, C.c_int, C.c_int]),
    "zf_wait_cells": (C.c_int, [_P]),
    "zf_get_cell_forces": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "zf_get_cell_kinematics": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_get_cell_geometry": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "zf_cgsm_forces": (C.c_int, [_P]),
    "zf_set_wall": (C.c_int, [_P, C.c_int, _f32p, C.c_int, _i32p, _f32p]),
    "zf_get_wall_index": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "zf_ibm_interp": (C.c_int, [_P]),
    "zf_nuc_memb_repulsion": (C.c_int, [_P, C.c_int]),
    "zf_rbc_rbc_repulsion": (C.c_int, [_P]),
    "zf_ibm_spread": (C.c_int, [_P]),
    "zf_update_positions": (C.c_int, [_P]),
    "zf_step": (C.c_int, [_P, C.c_int]),
    "zf_step_timed": (C.c_int, [_P, C.c_int, C.POINTER(C.c_float)]),
    "zf_iteration": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "zf_step_mass": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "zf_launch_count": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "zf_profile": (C.c_int, [_P, C.c_int, C.c_int]),
    "zf_profile_read": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_int),
                                  C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "zf_read_bindex_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _f64p, C.c_double, _i32p,
                                     C.POINTER(C.c_int64)]),
    "zf_read_boundary_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _f64p, C.c_double, _i32p,
                                       C.POINTER(C.c_int64)]),
    "zf_write_fluid_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _f64p, C.c_double, _i32p, _f32p, _f32p,
                                     _f32p, _f32p, _f32p, C.c_void_p, C.c_void_p]),
    "zf_read_fluid_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _f64p, C.c_double, _i32p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_int64)]),
    "zf_equilibrium_populations": (C.c_int, [C.c_int64, _f32p, _f32p, _f32p, _f32p, _f32p]),
    "zf_write_membrane_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_void_p, _i32p, _f64p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "zf_write_nucleus_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_void_p, _i32p, _f64p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_write_nucleus_edges_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p, _i32p, _f64p,
                                             _i32p, _f32p]),
    "zf_append_volume_area": (C.c_int, [C.c_char_p, C.c_int64, C.c_int, C.c_void_p, _i32p, _f32p, C.c_void_p]),
    "zf_read_cells_csv": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_read_mesh_dat": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_int]),
    "zf_read_wall_mesh": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "zf_write_wall_vtk": (C.c_int, [C.c_char_p, C.c_int, _f32p, C.c_int, _i32p, _f32p, _f32p, _i32p]),
    "zf_profile_stages": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "zf_save_state": (C.c_int, [_P, C.c_char_p]),
    "zf_lbm_moments": (C.c_int, [_P]),
    "zf_set_iteration": (C.c_int, [_P, C.c_int64]),
    "zf_get_cell_list_counts": (C.c_int, [_P, _i32p]),
    "zf_load_state": (C.c_int, [_P, C.c_char_p]),
    "zf_wss": (C.c_int, [_P, C.c_void_p, C.c_double, _f32p, C.c_void_p, C.c_void_p]),
    "zf_wss_objective": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _i32p, C.c_int, C.c_void_p,
                                   C.c_void_p, C.POINTER(C.c_double)]),
    "zf_wss_adjoint": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _i32p, C.c_int, C.c_void_p,
                                 C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_void_p,
                                 C.POINTER(C.c_double), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]),
    "zf_plane_count": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int32)]),
    "zf_plane_pack": (C.c_int, [_P, C.c_int, C.c_int, C.c_void_p]),
    "zf_plane_unpack": (C.c_int, [_P, C.c_int, C.c_int, C.c_void_p]),
    "zf_flux_objective": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _i32p, C.c_int, _f32p, _i32p, C.c_int,
                                    _f32p, C.c_void_p, C.POINTER(C.c_double)]),
    "zf_flux_adjoint": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _i32p, C.c_int, _f32p, _i32p, C.c_int,
                                  _f32p, C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_void_p,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "zf_adjoint_move_cells": (C.c_int, [_P, C.c_int]),
    "zf_adjoint_position_gradient": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "zf_repulsion_vjp": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_set_ib_slab": (C.c_int, [_P, C.c_int, C.c_int, C.c_double]),
    "zf_put_cells": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p]),
    "zf_inflow_slaves": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "zf_inflow_parents": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]),
    "zf_inflow_clone": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    "zf_cells_reduce_size": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "zf_cells_reduce_buffer": (C.c_int, [_P, C.c_int, C.c_void_p]),
    "zf_lbm_step_part_mf": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    "zf_membrane_vjp": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]),
}


def _ptr(a):
    """Data pointer of a numpy array (or None)."""
    return None if a is None else a.ctypes.data_as(C.c_void_p)

_lib = None


def lib() -> C.CDLL:
    """Loads libzf.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C zebraflow_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.zf_params_size() != C.sizeof(Params):
            raise RuntimeError("zf_params layout mismatch between zf.h and the ctypes mirror")
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != ZF_OK:
        raise ZfError(rc, lib().zf_last_error().decode(errors="replace"))


_GEN_SIGS = {
    "params_default": (None, [C.POINTER(Params)]),
    "gen_tube": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _i32p]),
    "gen_bifurcation": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _i32p,
                                  C.c_void_p]),
    "gen_icosphere": (C.c_int, [C.c_int, _f64p, _i32p]),
    "gen_wall_tube": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int, _f64p,
                                C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_int, C.c_int]),
    "gen_wall_bifurcation": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _f64p,
                                       C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "gen_cells": (C.c_int, [_i32p, C.c_int, C.c_int, C.c_int, _f64p, C.c_double, C.c_int, C.c_int, C.c_int,
                            _f64p, C.c_int, _f64p, _f64p, C.c_double, C.c_double, C.c_uint64, _f64p, _f64p,
                            C.POINTER(C.c_int)]),
}


class Inputs:
    """Reference parameter defaults and the workload generators of
    zebraflow_b200/csrc/zf_gen.cpp, bound to a library that exports them under
    `prefix`: libzf.so ("zf_"), or the CPU arm's oracle/liboracle.so ("orc_"),
    which compiles the same source, so that a CPU run builds the same inputs
    without loading the GPU library."""

    def __init__(self, L: C.CDLL, prefix: str):
        self._L, self._pre = L, prefix
        for name, (res, args) in _GEN_SIGS.items():
            fn = getattr(L, prefix + name)
            fn.restype = res
            fn.argtypes = args

    def _fn(self, name):
        return getattr(self._L, self._pre + name)

    def _check(self, rc: int, what: str) -> None:
        if rc != ZF_OK:
            raise ZfError(rc, f"{self._pre}{what} failed")

    def default_params(self, **kw) -> Params:
        p = Params()
        self._fn("params_default")(C.byref(p))
        for k, v in kw.items():
            if k in ("origin", "g", "periodic"):
                arr = getattr(p, k)
                for i, x in enumerate(v):
                    arr[i] = x
            else:
                setattr(p, k, v)
        return p

    def gen_tube(self, nx, ny, nz, cx, cy, R, periodic_z=True) -> np.ndarray:
        b = np.empty(nx * ny * nz, np.int32)
        self._check(self._fn("gen_tube")(nx, ny, nz, cx, cy, R, int(periodic_z), b), "gen_tube")
        return b.reshape(nx, ny, nz)

    def gen_bifurcation(self, nx, ny, nz, Rp, Rd, half_angle_deg=20.0):
        b = np.empty(nx * ny * nz, np.int32)
        layout = (C.c_double * 6)()
        self._check(self._fn("gen_bifurcation")(nx, ny, nz, Rp, Rd, half_angle_deg, b,
                                                C.cast(layout, C.c_void_p)), "gen_bifurcation")
        return b.reshape(nx, ny, nz), list(layout)

    def gen_icosphere(self, level: int):
        """Unit icosphere: (xyz [n][3] float64, tri [m][3] int32 1-based)."""
        n, m = 10 * 4 ** level + 2, 20 * 4 ** level
        xyz = np.empty(3 * n)
        tri = np.empty(3 * m, np.int32)
        self._check(self._fn("gen_icosphere")(level, xyz, tri), "gen_icosphere")
        return xyz.reshape(n, 3), tri.reshape(m, 3)

    def _wall_out(self, name, *args):
        fn = self._fn(name)
        nn_, nt_ = C.c_int(), C.c_int()
        self._check(fn(*args, C.byref(nn_), C.byref(nt_), None, None, None, 0, 0), name)
        xyz = np.empty(3 * nn_.value, np.float32)
        tri = np.empty(3 * nt_.value, np.int32)
        nrm = np.empty(3 * nt_.value, np.float32)
        self._check(fn(*args, C.byref(nn_), C.byref(nt_), _ptr(xyz), _ptr(tri), _ptr(nrm), nn_.value,
                       nt_.value), name)
        return xyz.reshape(3, -1), tri.reshape(3, -1), nrm.reshape(3, -1)

    def gen_wall_tube(self, cx, cy, R, nz, origin=(0.0, 0.0, 0.0), dx=0.5, h=1.0, nseg=None):
        """Cylinder wall mesh in um: (xyz [3][n], tri [3][m] 1-based, normals [3][m])."""
        if nseg is None:
            nseg = max(12, int(round(2 * np.pi * R / h)))
        return self._wall_out("gen_wall_tube", cx, cy, R, nz, h, nseg, np.asarray(origin, np.float64), dx)

    def gen_wall_bifurcation(self, nx, ny, nz, Rp, Rd, half_angle_deg=20.0, origin=(0.0, 0.0, 0.0), dx=0.5):
        return self._wall_out("gen_wall_bifurcation", nx, ny, nz, Rp, Rd, half_angle_deg,
                              np.asarray(origin, np.float64), dx)

    def gen_cells(self, b, n_cells, rest, rest_n, axes, seed=1234, origin=(0.0, 0.0, 0.0), dx=0.5,
                  periodic_z=True, margin=0.25, wall_clear=0.0):
        """Seeded placement; returns (x [3][placed][n_node], xn [3][placed][n_node_n]).
        margin (um) inflates each cell's ellipsoid against the others; wall_clear
        (um) is the least lattice (Chebyshev) distance of every membrane node
        from a non-fluid point, at least one lattice unit."""
        b = np.ascontiguousarray(b, np.int32)
        nx, ny, nz = b.shape
        rest = np.ascontiguousarray(rest, np.float64)
        rest_n = np.ascontiguousarray(rest_n, np.float64)
        nn_, nnn = rest.shape[0], rest_n.shape[0]
        x = np.zeros(3 * n_cells * nn_)
        xn = np.zeros(max(3 * n_cells * nnn, 1))
        placed = C.c_int()
        self._check(self._fn("gen_cells")(b.ravel(), nx, ny, nz, np.asarray(origin, np.float64), dx,
                                          int(periodic_z), n_cells, nn_, rest.ravel(), nnn, rest_n.ravel(),
                                          np.asarray(axes, np.float64), margin, wall_clear, seed, x, xn,
                                          C.byref(placed)), "gen_cells")
        k = placed.value
        x = x.reshape(3, n_cells, nn_)[:, :k, :].copy()
        xn = xn[:3 * n_cells * nnn].reshape(3, n_cells, nnn)[:, :k, :].copy()
        return x, xn


_inputs = None


def inputs() -> Inputs:
    """The generators and parameter defaults of libzf.so."""
    global _inputs
    if _inputs is None:
        _inputs = Inputs(lib(), "zf_")
    return _inputs


def default_params(**kw) -> Params:
    return inputs().default_params(**kw)


def gen_tube(nx, ny, nz, cx, cy, R, periodic_z=True) -> np.ndarray:
    return inputs().gen_tube(nx, ny, nz, cx, cy, R, periodic_z)


def gen_bifurcation(nx, ny, nz, Rp, Rd, half_angle_deg=20.0):
    return inputs().gen_bifurcation(nx, ny, nz, Rp, Rd, half_angle_deg)


def gen_icosphere(level: int):
    return inputs().gen_icosphere(level)


def gen_wall_tube(cx, cy, R, nz, origin=(0.0, 0.0, 0.0), dx=0.5, h=1.0, nseg=None):
    return inputs().gen_wall_tube(cx, cy, R, nz, origin, dx, h, nseg)


def gen_wall_bifurcation(nx, ny, nz, Rp, Rd, half_angle_deg=20.0, origin=(0.0, 0.0, 0.0), dx=0.5):
    return inputs().gen_wall_bifurcation(nx, ny, nz, Rp, Rd, half_angle_deg, origin, dx)


def gen_cells(b, n_cells, rest, rest_n, axes, seed=1234, origin=(0.0, 0.0, 0.0), dx=0.5,
              periodic_z=True, margin=0.25, wall_clear=0.0):
    return inputs().gen_cells(b, n_cells, rest, rest_n, axes, seed, origin, dx, periodic_z, margin,
                              wall_clear)


def mesh_edges(tri1: np.ndarray) -> np.ndarray:
    """Unique edges of a triangle mesh, 1-based [n][2] (nucleus edge list)."""
    t = np.asarray(tri1) - 1
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    e = np.sort(e, axis=1)
    e = np.unique(e, axis=0)
    return (e + 1).astype(np.int32)


# ---- the reference's file formats (zf_io.cpp; host only) -------------------

def _path(p) -> bytes:
    return os.fsencode(p)


def _opt(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype)


def read_bindex_csv(path, dims, origin=(0.0, 0.0, 0.0), dx=0.5):
    nx, ny, nz = dims
    b = np.empty(nx * ny * nz, np.int32)
    rows = C.c_int64()
    _check(lib().zf_read_bindex_csv(_path(path), nx, ny, nz, np.asarray(origin, np.float64), dx, b,
                                    C.byref(rows)))
    return b.reshape(nx, ny, nz), rows.value


def read_boundary_csv(path, dims, origin=(0.0, 0.0, 0.0), dx=0.5):
    """A parent segment's boundary CSV ("Bindex","D","U","V","W","Points:0..2"):
    the B_index array it describes (-1 elsewhere) and the row count."""
    nx, ny, nz = dims
    b = np.empty(nx * ny * nz, np.int32)
    rows = C.c_int64()
    _check(lib().zf_read_boundary_csv(_path(path), nx, ny, nz, np.asarray(origin, np.float64), dx, b,
                                      C.byref(rows)))
    return b.reshape(nx, ny, nz), rows.value


def write_fluid_csv(path, b_index, D, U, V, W, bodyforce, eulneigh=None, windex=None, origin=(0.0, 0.0, 0.0),
                    dx=0.5):
    b = np.ascontiguousarray(b_index, np.int32)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
    en, wi = _opt(eulneigh, np.int32), _opt(windex, np.int32)
    _check(lib().zf_write_fluid_csv(_path(path), *b.shape, np.asarray(origin, np.float64), dx, b.ravel(), f32(D),
                                    f32(U), f32(V), f32(W), f32(bodyforce).ravel(), _ptr(en), _ptr(wi)))


def read_fluid_csv(path, b_index, origin=(0.0, 0.0, 0.0), dx=0.5):
    """(D, U, V, W [n], bodyforce [3][n], eulneigh [n] in DOMLIST order,
    windex [nx][ny][nz], rows)."""
    b = np.ascontiguousarray(b_index, np.int32)
    n = int((b >= 0).sum())
    D, U, V, W = (np.zeros(n, np.float32) for _ in range(4))
    bf = np.zeros((3, n), np.float32)
    en = np.zeros(n, np.int32)
    wi = np.zeros(b.shape, np.int32)
    rows = C.c_int64()
    _check(lib().zf_read_fluid_csv(_path(path), *b.shape, np.asarray(origin, np.float64), dx, b.ravel(), _ptr(D),
                                   _ptr(U), _ptr(V), _ptr(W), _ptr(bf), _ptr(en), _ptr(wi), C.byref(rows)))
    return D, U, V, W, bf, en, wi, rows.value


def equilibrium_populations(D, U, V, W):
    D, U, V, W = (np.ascontiguousarray(a, np.float32) for a in (D, U, V, W))
    f = np.empty((19, D.size), np.float32)
    _check(lib().zf_equilibrium_populations(D.size, D, U, V, W, f.ravel()))
    return f


def write_membrane_csv(path, status, x, vel=None, wall_tri=None, wrep=None, regress=None, area_ratio=None,
                       ftot=None, fvol=None, out_flag=None, cell_id=None):
    x = np.ascontiguousarray(x, np.float64)
    nc, nn = x.shape[1], x.shape[2]
    args = [_opt(cell_id, np.int32), np.ascontiguousarray(status, np.int32), x.ravel(), _opt(vel, np.float64),
            _opt(wall_tri, np.int32), _opt(wrep, np.float32), _opt(regress, np.int32),
            _opt(area_ratio, np.float32), _opt(ftot, np.float32), _opt(fvol, np.float32), _opt(out_flag, np.int32)]
    _check(lib().zf_write_membrane_csv(_path(path), nc, nn, _ptr(args[0]), args[1], args[2],
                                       *[_ptr(a) for a in args[3:]]))


def write_nucleus_csv(path, status, xn, vel_n=None, ftot_n=None, neigh=None, neigh_flag=None, cell_id=None):
    xn = np.ascontiguousarray(xn, np.float64)
    nc, nn = xn.shape[1], xn.shape[2]
    opt = [_opt(vel_n, np.float64), _opt(ftot_n, np.float32), _opt(neigh, np.int32), _opt(neigh_flag, np.int32)]
    cid = _opt(cell_id, np.int32)
    _check(lib().zf_write_nucleus_csv(_path(path), nc, nn, _ptr(cid), np.ascontiguousarray(status, np.int32),
                                      xn.ravel(), *[_ptr(a) for a in opt]))


def write_nucleus_edges_csv(path, status, xn, edge_n, lmax_n, cell_id=None):
    xn = np.ascontiguousarray(xn, np.float64)
    e = np.ascontiguousarray(edge_n, np.int32)
    cid = _opt(cell_id, np.int32)
    _check(lib().zf_write_nucleus_edges_csv(_path(path), xn.shape[1], xn.shape[2], e.shape[0], _ptr(cid),
                                            np.ascontiguousarray(status, np.int32), xn.ravel(), e.ravel(),
                                            np.ascontiguousarray(lmax_n, np.float32)))


def append_volume_area(path, it, status, cell_f, regress=None, cell_id=None):
    st = np.ascontiguousarray(status, np.int32)
    cid, rg = _opt(cell_id, np.int32), _opt(regress, np.int32)
    _check(lib().zf_append_volume_area(_path(path), it, st.size, _ptr(cid), st,
                                       np.ascontiguousarray(cell_f, np.float32).ravel(), _ptr(rg)))


def read_cells_csv(path, n_node, nucleus=False):
    """(cell_id [nc], status [nc], x, vel [3][nc][n_node] fp64, ftot [3][nc][n_node] fp32)."""
    nc = C.c_int()
    L = lib()
    _check(L.zf_read_cells_csv(_path(path), int(nucleus), n_node, 0, C.byref(nc), None, None, None, None, None))
    k = nc.value
    cid, st = np.empty(k, np.int32), np.empty(k, np.int32)
    x, vel = np.empty((3, k, n_node)), np.empty((3, k, n_node))
    ft = np.empty((3, k, n_node), np.float32)
    _check(L.zf_read_cells_csv(_path(path), int(nucleus), n_node, k, C.byref(nc), _ptr(cid), _ptr(st), _ptr(x),
                               _ptr(vel), _ptr(ft)))
    return cid, st, x, vel, ft


MESH_POINTS, MESH_CELLS, MESH_LINES = 0, 1, 2


def read_mesh_dat(path, kind):
    n = C.c_int()
    L = lib()
    _check(L.zf_read_mesh_dat(_path(path), kind, C.byref(n), None, 0))
    per = 2 if kind == MESH_LINES else 3
    v = np.empty(n.value * per)
    _check(L.zf_read_mesh_dat(_path(path), kind, C.byref(n), _ptr(v), n.value))
    v = v.reshape(n.value, per)
    return v if kind == MESH_POINTS else v.astype(np.int32)


def read_wall_mesh(nodes_path, cells_path, normals_path):
    """(xyz [3][n], tri [3][m] 1-based, normals [3][m]) as zf_set_wall takes them."""
    nn_, nt_ = C.c_int(), C.c_int()
    L = lib()
    paths = (_path(nodes_path), _path(cells_path), _path(normals_path))
    _check(L.zf_read_wall_mesh(*paths, C.byref(nn_), C.byref(nt_), None, None, None, 0, 0))
    xyz = np.empty((3, nn_.value), np.float32)
    tri = np.empty((3, nt_.value), np.int32)
    nrm = np.empty((3, nt_.value), np.float32)
    _check(L.zf_read_wall_mesh(*paths, C.byref(nn_), C.byref(nt_), _ptr(xyz), _ptr(tri), _ptr(nrm), nn_.value,
                               nt_.value))
    return xyz, tri, nrm


def write_wall_vtk(path, xyz, tri, pressure, wss, valid):
    xyz = np.ascontiguousarray(xyz, np.float32)
    tri = np.ascontiguousarray(tri, np.int32)
    _check(lib().zf_write_wall_vtk(_path(path), xyz.shape[1], xyz.ravel(), tri.shape[1], tri.ravel(),
                                   np.ascontiguousarray(pressure, np.float32),
                                   np.ascontiguousarray(wss, np.float32).ravel(),
                                   np.ascontiguousarray(valid, np.int32)))


class Context:
    """Owns one zf_ctx (one CUDA stream on one device)."""

    def __init__(self, params: Params, device: int = 0):
        self.params = params
        self._h = lib().zf_create(C.byref(params), device)
        if not self._h:
            raise ZfError(ZF_ERR_CUDA, lib().zf_last_error().decode(errors="replace"))
        self.n_listed = 0
        self.n_fluid = 0

    def close(self):
        if self._h:
            lib().zf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # lattice ---------------------------------------------------------------
    def set_lattice(self, b_index: np.ndarray):
        b = np.ascontiguousarray(b_index, np.int32).ravel()
        _check(lib().zf_set_lattice(self._h, b))
        nl, nf = C.c_int64(), C.c_int64()
        _check(lib().zf_num_listed(self._h, C.byref(nl), C.byref(nf)))
        self.n_listed, self.n_fluid = nl.value, nf.value

    def domlist(self) -> np.ndarray:
        out = np.empty(self.n_listed * 3, np.int32)
        _check(lib().zf_get_domlist(self._h, out))
        return out.reshape(-1, 3)

    # fields ----------------------------------------------------------------
    def upload_populations(self, f: np.ndarray):
        _check(lib().zf_upload_populations(self._h, np.ascontiguousarray(f, np.float32).ravel()))

    def download_populations(self) -> np.ndarray:
        out = np.empty(Q * self.n_listed, np.float32)
        _check(lib().zf_download_populations(self._h, out))
        return out.reshape(Q, self.n_listed)

    def upload_bodyforce(self, bf: np.ndarray):
        _check(lib().zf_upload_bodyforce(self._h, np.ascontiguousarray(bf, np.float32).ravel()))

    def download_bodyforce(self) -> np.ndarray:
        out = np.empty(3 * self.n_listed, np.float32)
        _check(lib().zf_download_bodyforce(self._h, out))
        return out.reshape(3, self.n_listed)

    def download_moments(self):
        outs = [np.empty(self.n_listed, np.float32) for _ in range(4)]
        _check(lib().zf_download_moments(self._h, *outs))
        return outs

    # steps -----------------------------------------------------------------
    def lbm_step(self, store_moments=True, zero_bodyforce=False):
        _check(lib().zf_lbm_step(self._h, int(store_moments), int(zero_bodyforce)))

    def set_slab(self, k_lo: int, k_hi: int):
        _check(lib().zf_set_slab(self._h, k_lo, k_hi))

    def lbm_step_part(self, part: int, finish: bool, store_moments=False, zero_bodyforce=False):
        _check(lib().zf_lbm_step_part_mf(self._h, part, int(finish), int(store_moments), int(zero_bodyforce)))

    def set_ib_slab(self, k_lo: int, k_hi: int, lz: float):
        """zf_set_ib_slab: owned planes [k_lo, k_hi) of this slab, z period lz (um)."""
        _check(lib().zf_set_ib_slab(self._h, k_lo, k_hi, float(lz)))

    def cells_reduce_size(self) -> int:
        n = C.c_int64()
        _check(lib().zf_cells_reduce_size(self._h, C.byref(n)))
        return n.value

    def cells_reduce_buffer(self, direction: int, dev_ptr):
        """zf_cells_reduce_buffer with a device buffer of fp64 at dev_ptr."""
        _check(lib().zf_cells_reduce_buffer(self._h, int(direction), C.c_void_p(dev_ptr)))

    def lbm_steps(self, n: int):
        _check(lib().zf_lbm_steps(self._h, n))

    def lbm_steps_timed(self, n: int) -> float:
        ms = C.c_float()
        _check(lib().zf_lbm_steps_timed(self._h, n, C.byref(ms)))
        return ms.value

    def mass(self, include_walls=False) -> float:
        m = C.c_double()
        _check(lib().zf_mass(self._h, int(include_walls), C.byref(m)))
        return m.value

    def sync(self):
        _check(lib().zf_sync(self._h))

    def status(self) -> Status:
        s = Status()
        _check(lib().zf_get_status(self._h, C.byref(s)))
        return s

    # membrane mesh and cells ---------------------------------------------
    def set_mesh(self, rest, tri1, rest_n=None, edge_n1=None):
        rest = np.ascontiguousarray(rest, np.float64).ravel()
        tri1 = np.ascontiguousarray(tri1, np.int32).ravel()
        rest_n = np.zeros(3) if rest_n is None else np.ascontiguousarray(rest_n, np.float64).ravel()
        edge_n1 = (np.zeros(2, np.int32) if edge_n1 is None
                   else np.ascontiguousarray(edge_n1, np.int32).ravel())
        self.nn, self.nt = rest.size // 3, tri1.size // 3
        self.nnn = 0 if rest_n.size == 3 and edge_n1.size == 2 and not edge_n1.any() else rest_n.size // 3
        nen = 0 if self.nnn == 0 else edge_n1.size // 2
        _check(lib().zf_set_mesh(self._h, self.nn, self.nt, tri1, rest, self.nnn, nen, edge_n1,
                                 rest_n))
        ne, a0, v0 = C.c_int32(), C.c_double(), C.c_double()
        _check(lib().zf_mesh_info(self._h, C.byref(ne), C.byref(a0), C.byref(v0)))
        self.ne, self.nen, self.area0, self.volume0 = ne.value, nen, a0.value, v0.value

    def edges(self):
        e = np.empty(6 * self.ne, np.int32)
        af = np.empty(self.ne, np.uint8)
        _check(lib().zf_get_edges(self._h, _ptr(e), _ptr(af)))
        return e.reshape(self.ne, 6), af

    def edge_params(self):
        ep = np.empty(5 * self.ne, np.float32)
        epn = np.empty(max(3 * self.nen, 1), np.float32)
        ae = np.empty(self.nt, np.float32)
        _check(lib().zf_get_edge_params(self._h, _ptr(ep), _ptr(epn), _ptr(ae)))
        return ep.reshape(5, self.ne), epn[:3 * self.nen].reshape(3, self.nen), ae

    def set_cells(self, x, xn=None):
        """x: [3][n_cells][n_node] um; xn: [3][n_cells][n_node_n]."""
        x = np.ascontiguousarray(x, np.float64)
        self.nc = x.shape[1]
        xn_ = None if xn is None else np.ascontiguousarray(xn, np.float64)
        _check(lib().zf_set_cells(self._h, self.nc, x.ravel(), _ptr(xn_)))

    def cells(self):
        x = np.empty((3, self.nc, self.nn))
        xn = np.empty((3, self.nc, self.nnn)) if self.nnn else None
        st = np.empty(self.nc, np.int32)
        _check(lib().zf_get_cells(self._h, _ptr(x), _ptr(xn), _ptr(st)))
        return x, xn, st

    def put_cells(self, x=None, xn=None, status=None):
        """zf_put_cells: overwrite positions and/or statuses of all cells."""
        x_ = None if x is None else np.ascontiguousarray(x, np.float64)
        xn_ = None if xn is None else np.ascontiguousarray(xn, np.float64)
        st = None if status is None else np.ascontiguousarray(status, np.int32)
        _check(lib().zf_put_cells(self._h, _ptr(x_), _ptr(xn_), _ptr(st)))

    def cells_async(self, x, xn, status):
        """Queue the copies of zf_get_cells into x [3][nc][nn], xn and status
        (pinned host arrays, or None) without waiting; they hold the values
        once wait_cells() returns."""
        _check(lib().zf_get_cells_async(self._h, _ptr(x), _ptr(xn), _ptr(status)))

    def wait_cells(self):
        _check(lib().zf_wait_cells(self._h))

    def cell_forces(self):
        f = np.empty((3, self.nc, self.nn), np.float32)
        fn = np.empty((3, self.nc, self.nnn), np.float32) if self.nnn else None
        _check(lib().zf_get_cell_forces(self._h, _ptr(f), _ptr(fn)))
        return f, fn

    def cell_kinematics(self):
        v = np.empty((3, self.nc, self.nn))
        vn = np.empty((3, self.nc, self.nnn)) if self.nnn else None
        w = np.empty((3, self.nc, self.nn), np.float32)
        wn = np.empty((3, self.nc, self.nnn), np.float32) if self.nnn else None
        _check(lib().zf_get_cell_kinematics(self._h, _ptr(v), _ptr(vn), _ptr(w), _ptr(wn)))
        return v, vn, w, wn

    def cell_geometry(self):
        ta = np.empty((self.nc, self.nt), np.float32)
        tn = np.empty((3, self.nc, self.nt), np.float32)
        tc = np.empty((3, self.nc, self.nt), np.float32)
        nn_ = np.empty((3, self.nc, self.nn), np.float32)
        cf = np.empty((self.nc, 8), np.float32)
        _check(lib().zf_get_cell_geometry(self._h, _ptr(ta), _ptr(tn), _ptr(tc), _ptr(nn_),
                                          _ptr(cf)))
        return ta, tn, tc, nn_, cf

    def cgsm_forces(self):
        _check(lib().zf_cgsm_forces(self._h))

    # wall and IB coupling ---------------------------------------------------
    def set_wall(self, xyz, tri, nrm):
        xyz = np.ascontiguousarray(xyz, np.float32)
        tri = np.ascontiguousarray(tri, np.int32)
        nrm = np.ascontiguousarray(nrm, np.float32)
        _check(lib().zf_set_wall(self._h, xyz.shape[1], xyz.ravel(), tri.shape[1], tri.ravel(),
                                 nrm.ravel()))
        self._nw = xyz.shape[1]

    def wall_index(self):
        p = self.params
        n = p.nx * p.ny * p.nz
        wi = np.empty(n, np.int32)
        uv = np.empty(3 * n, np.float32)
        _check(lib().zf_get_wall_index(self._h, _ptr(wi), _ptr(uv)))
        return wi.reshape(p.nx, p.ny, p.nz), uv.reshape(3, p.nx, p.ny, p.nz)

    def ibm_interp(self):
        _check(lib().zf_ibm_interp(self._h))

    def nuc_memb_repulsion(self, rebuild=False):
        _check(lib().zf_nuc_memb_repulsion(self._h, int(rebuild)))

    def rbc_rbc_repulsion(self):
        _check(lib().zf_rbc_rbc_repulsion(self._h))

    def ibm_spread(self):
        _check(lib().zf_ibm_spread(self._h))

    def update_positions(self):
        _check(lib().zf_update_positions(self._h))

    def step(self, n=1):
        _check(lib().zf_step(self._h, n))

    @staticmethod
    def _opt(a, dtype):
        if a is None:
            return None, None
        a = np.ascontiguousarray(a, dtype)
        return a, a.ctypes.data_as(C.c_void_p)

    def wss_objective(self, nsteps, t0, t1, patch, fb=None, node_normals=None) -> float:
        """J of zf_wss_objective (mean |WSS| over patch and steps t0..t1)."""
        patch = np.ascontiguousarray(patch, np.int32)
        _, pn = self._opt(node_normals, np.float32)
        _fb, pf = self._opt(fb, np.float32)
        J = C.c_double()
        _check(lib().zf_wss_objective(self._h, nsteps, t0, t1, patch, patch.size, pn, pf, C.byref(J)))
        return J.value

    def wss_adjoint(self, nsteps, t0, t1, patch, fb=None, node_normals=None, checkpoint=50):
        """(J, dJ/dfb [3][n_listed], dJ/dtau, dJ/dEs, dJ/dkb) of zf_wss_adjoint."""
        patch = np.ascontiguousarray(patch, np.int32)
        _, pn = self._opt(node_normals, np.float32)
        _fb, pf = self._opt(fb, np.float32)
        g = np.zeros((3, self.n_listed), np.float32)
        J, gt, ge, gk = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        _check(lib().zf_wss_adjoint(self._h, nsteps, t0, t1, patch, patch.size, pn, pf, checkpoint,
                                    C.byref(J), g.ctypes.data_as(C.c_void_p), C.byref(gt),
                                    C.byref(ge), C.byref(gk)))
        return J.value, g, gt.value, ge.value, gk.value

    def plane_count(self, k) -> int:
        """Listed points of lattice plane z = k (zf_plane_count)."""
        n = C.c_int32()
        _check(lib().zf_plane_count(self._h, int(k), C.byref(n)))
        return n.value

    def plane_pack(self, k, direction, dev_ptr):
        """zf_plane_pack into device memory at dev_ptr (an int address)."""
        _check(lib().zf_plane_pack(self._h, int(k), int(direction), C.c_void_p(dev_ptr)))

    def plane_unpack(self, k, direction, dev_ptr):
        """zf_plane_unpack from device memory at dev_ptr (an int address)."""
        _check(lib().zf_plane_unpack(self._h, int(k), int(direction), C.c_void_p(dev_ptr)))

    def flux_objective(self, nsteps, t0, t1, pts0, nrm0, pts1, nrm1, fb=None) -> float:
        """J of zf_flux_objective (mean share of the flux through set 0)."""
        p0, p1 = np.ascontiguousarray(pts0, np.int32), np.ascontiguousarray(pts1, np.int32)
        n0, n1 = np.ascontiguousarray(nrm0, np.float32), np.ascontiguousarray(nrm1, np.float32)
        _fb, pf = self._opt(fb, np.float32)
        J = C.c_double()
        _check(lib().zf_flux_objective(self._h, nsteps, t0, t1, p0, p0.size, n0, p1, p1.size, n1, pf,
                                       C.byref(J)))
        return J.value

    def flux_adjoint(self, nsteps, t0, t1, pts0, nrm0, pts1, nrm1, fb=None, checkpoint=50):
        """(J, dJ/dfb [3][n_listed], dJ/dtau, dJ/dEs, dJ/dkb) of zf_flux_adjoint."""
        p0, p1 = np.ascontiguousarray(pts0, np.int32), np.ascontiguousarray(pts1, np.int32)
        n0, n1 = np.ascontiguousarray(nrm0, np.float32), np.ascontiguousarray(nrm1, np.float32)
        _fb, pf = self._opt(fb, np.float32)
        g = np.zeros((3, self.n_listed), np.float32)
        J, gt, ge, gk = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        _check(lib().zf_flux_adjoint(self._h, nsteps, t0, t1, p0, p0.size, n0, p1, p1.size, n1, pf, checkpoint,
                                     C.byref(J), g.ctypes.data_as(C.c_void_p), C.byref(gt), C.byref(ge),
                                     C.byref(gk)))
        return J.value, g, gt.value, ge.value, gk.value

    def adjoint_move_cells(self, move=True):
        """zf_adjoint_move_cells: the adjoint calls' forward moves the cells."""
        _check(lib().zf_adjoint_move_cells(self._h, int(bool(move))))

    def adjoint_position_gradient(self):
        """(dJ/dx_0 [3][nc][nn], dJ/dxn_0 [3][nc][nnn]) of the last adjoint with
        moving cells."""
        g = np.empty((3, self.nc, self.nn), np.float32)
        gn = np.empty((3, self.nc, self.nnn), np.float32) if self.nnn else None
        _check(lib().zf_adjoint_position_gradient(self._h, _ptr(g), _ptr(gn)))
        return g, gn

    def repulsion_vjp(self, lam_w):
        """(lam_w^T dwrep/dx, lam_w^T dwrep/dxn) of the repulsion velocities of a
        membrane iteration at the current positions (zf_repulsion_vjp)."""
        lam_w = np.ascontiguousarray(lam_w, np.float32)
        g = np.empty((3, self.nc, self.nn), np.float32)
        gn = np.empty((3, self.nc, self.nnn), np.float32) if self.nnn else None
        _check(lib().zf_repulsion_vjp(self._h, _ptr(lam_w), _ptr(g), _ptr(gn)))
        return g, gn

    def membrane_vjp(self, lam, lam_n=None):
        """(lam^T dF/dx, lam_n^T dF/dxn, lam^T dF/dEs, lam^T dF/dkb) of the
        membrane and nucleus forces at the current positions (zf_membrane_vjp)."""
        lam = np.ascontiguousarray(lam, np.float32)
        ln = None if lam_n is None else np.ascontiguousarray(lam_n, np.float32)
        g = np.empty((3, self.nc, self.nn), np.float32)
        gn = np.empty((3, self.nc, self.nnn), np.float32) if self.nnn else None
        ge, gk = C.c_double(), C.c_double()
        _check(lib().zf_membrane_vjp(self._h, _ptr(lam), _ptr(ln), _ptr(g), _ptr(gn), C.byref(ge),
                                     C.byref(gk)))
        return g, gn, ge.value, gk.value

    def wss(self, node_normals=None, pgauge=120.0):
        """WSS [3][nw] (Pa), wall pressure [nw] (Pa), valid [nw] from the current
        populations (zf_wss); node_normals [3][nw] or None for the mesh's own."""
        nw = self._nw
        wss = np.empty(3 * nw, np.float32)
        press = np.empty(nw, np.float32)
        valid = np.empty(nw, np.int32)
        nrm = None if node_normals is None else np.ascontiguousarray(node_normals, np.float32)
        _check(lib().zf_wss(self._h, None if nrm is None else nrm.ctypes.data_as(C.c_void_p),
                            float(pgauge), wss, press.ctypes.data_as(C.c_void_p),
                            valid.ctypes.data_as(C.c_void_p)))
        return wss.reshape(3, nw), press, valid

    def step_timed(self, n):
        ms = C.c_float()
        _check(lib().zf_step_timed(self._h, n, C.byref(ms)))
        return ms.value

    def iteration(self):
        it = C.c_int64()
        _check(lib().zf_iteration(self._h, C.byref(it)))
        return it.value

    def step_mass(self) -> float:
        m = C.c_double()
        _check(lib().zf_step_mass(self._h, C.byref(m)))
        return m.value

    def set_iteration(self, it):
        """Completed iterations; the next step is iteration it + 1."""
        _check(lib().zf_set_iteration(self._h, int(it)))

    def refresh_moments(self):
        """Recomputes the stored D, U, V, W from the current populations."""
        _check(lib().zf_lbm_moments(self._h))

    def cell_list_counts(self):
        """Triangle centroids per listed point in the last cell list (EulNeigh)."""
        n = np.empty(self.n_listed, np.int32)
        _check(lib().zf_get_cell_list_counts(self._h, n))
        return n

    def save_state(self, path):
        """Exact checkpoint of the time-stepping state (zf_save_state)."""
        _check(lib().zf_save_state(self._h, os.fsencode(path)))

    def load_state(self, path):
        """Restores a checkpoint into this context (same lattice, storage,
        mesh and cell count)."""
        _check(lib().zf_load_state(self._h, os.fsencode(path)))

    def launch_count(self) -> int:
        n = C.c_int64()
        _check(lib().zf_launch_count(self._h, C.byref(n)))
        return n.value

    def profile(self, enable=True, capacity=4096):
        _check(lib().zf_profile(self._h, int(enable), capacity))

    def profile_read(self):
        lm, lc, mm, mc = C.c_float(), C.c_int(), C.c_float(), C.c_int()
        _check(lib().zf_profile_read(self._h, C.byref(lm), C.byref(lc), C.byref(mm), C.byref(mc)))
        return lm.value, lc.value, mm.value, mc.value

    PROFILE_STAGES = ("membrane_forces", "lbm", "ib_interp", "nuc_memb", "cell_list", "rbc_rbc",
                      "ib_spread", "update")

    def profile_stages(self):
        """({stage: summed ms} over the profiled membrane iterations, blocks)."""
        st = (C.c_float * 8)()
        nb = C.c_int()
        _check(lib().zf_profile_stages(self._h, st, C.byref(nb)))
        return dict(zip(self.PROFILE_STAGES, list(st))), nb.value

    def set_stream(self, stream_handle):
        """Queue the context's work on a CUDA stream (a cudaStream_t as int);
        None or 0 selects the context's own stream (so the legacy default
        stream cannot be chosen: pass a created stream)."""
        _check(lib().zf_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def device_bytes(self) -> int:
        b = C.c_int64()
        _check(lib().zf_device_bytes(self._h, C.byref(b)))
        return b.value

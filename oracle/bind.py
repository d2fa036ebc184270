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
            g("orc_lbm_time_steps").restype = C.c_double
            g("orc_lbm_time_steps").argtypes = [C.c_void_p, C.c_int]
        _lib = L
    return _lib


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

    def moments(self):
        outs = [np.empty(self.n) for _ in range(4)]
        self._fn("orc_lbm_get_moments")(self._h, *outs)
        return outs

    def step(self, rbc_flag=False):
        self._fn("orc_lbm_step")(self._h, int(rbc_flag))

    def set_storage_emulation(self, mode, scale=65536.0, rho_ref=1.0):
        """Rounds the stored populations after every step as a storage form
        would: 0 none, 1 raw fp32, 2 fp32 deviation, 3 fp16 deviation,
        4 bf16 deviation (deviation d = f/w - rho_ref, stored as scale*d)."""
        self._fn("orc_lbm_set_storage_emulation")(self._h, int(mode), float(scale), float(rho_ref))

    def mass(self, include_walls=False):
        return float(self._fn("orc_lbm_mass")(self._h, int(include_walls)))

    def time_steps(self, n):
        return float(self._fn("orc_lbm_time_steps")(self._h, int(n)))

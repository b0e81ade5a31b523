"""ctypes front end of the C oracle (test infrastructure only).

Imported by tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of
bench.py; never by the product package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgp_oracle.so")

HD, MHD, RMHD = 0, 1, 2
LIM = {"flat": 0, "minmod": 1, "vl": 2, "vanleer": 2, "mc": 3, "ppm": 4, "mp5": 5,
       "vanalbada": 6, "ospre": 7, "umist": 8, "wenoz": 9, "limo3": 10, "weno3": 11}
SOLVER = {"hll": 0, "hllc": 1, "hlld": 2, "tvdlf": 3}
CT = {"uct_hll": 0, "uct_hlld": 1, "arithmetic": 2, "ct_contact": 3}


class OrcCfg(ctypes.Structure):
    _fields_ = [("physics", ctypes.c_int), ("ndim", ctypes.c_int),
                ("n", ctypes.c_int * 3), ("limiter", ctypes.c_int),
                ("solver", ctypes.c_int), ("ct", ctypes.c_int),
                ("gamma", ctypes.c_double), ("dx", ctypes.c_double * 3),
                ("cfl", ctypes.c_double), ("cfl_max_var", ctypes.c_double),
                ("outflow", ctypes.c_int), ("reflect", ctypes.c_int),
                ("eqtsym", ctypes.c_int), ("rk", ctypes.c_int),
                ("userdef", ctypes.c_int), ("ud_rho", ctypes.c_double),
                ("ud_vn", ctypes.c_double)]

# The inflow of the USERDEF parity cases (oracle/ref/init.cpp UserDefBoundary)
UD_RHO, UD_VN = 1.25, 0.25


def build() -> str:
    subprocess.run(["make", "-s"], cwd=HERE, check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.POINTER(OrcCfg)]
        L.orc_destroy.argtypes = [P]
        L.orc_set_state.argtypes = [P, D, D, D]
        L.orc_get_state.argtypes = [P, D, D, D]
        L.orc_step.restype = ctypes.c_double
        L.orc_step.argtypes = [P, ctypes.c_double, ctypes.POINTER(ctypes.c_uint32)]
        L.orc_next_dt.restype = ctypes.c_double
        L.orc_next_dt.argtypes = [ctypes.c_double] * 4
        L.orc_run.restype = ctypes.c_uint32
        L.orc_run.argtypes = [P, ctypes.c_int, ctypes.c_double, D]
        L.orc_set_ulp_nudge.argtypes = [ctypes.c_int]
        L.orc_set_rmhd_strict.argtypes = [ctypes.c_int]
        L.orc_prim_to_cons.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_long, D, D]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_ulp_nudge(n: int) -> None:
    """Checker knob: perturb the RMHD quartic's acos result by n ulps."""
    lib().orc_set_ulp_nudge(int(n))


def set_cr_trig(on: bool) -> None:
    """Checker knob: correctly rounded acos/cos/sin in the RMHD quartic
    (binary128 evaluation rounded once) instead of the C library's."""
    lib().orc_set_cr_trig(1 if on else 0)


def set_rmhd_strict(on: bool) -> None:
    """Checker knob: fail the RMHD HLLD star state when a Riemann state cannot
    be built (the rule the GPU kernels use); off reproduces the reference."""
    lib().orc_set_rmhd_strict(1 if on else 0)


def prim_to_cons(physics: int, gamma: float, V: np.ndarray) -> np.ndarray:
    V = np.ascontiguousarray(V, dtype=np.float64)
    U = np.empty_like(V)
    ncell = V[0].size
    lib().orc_prim_to_cons(physics, gamma, ncell, _dp(V), _dp(U))
    return U


class Oracle:
    """One grid advanced by the CPU restatement."""

    def __init__(self, state, limiter="mc", solver="hlld", ct="uct_hlld",
                 cfl=0.4, cfl_max_var=1.1, outflow=0, reflect=0, eqtsym=0, rk=2,
                 userdef=0):
        nx, ny, nz = state.shape
        c = OrcCfg()
        c.physics, c.ndim = state.physics, state.ndim
        c.n[0], c.n[1], c.n[2] = nx, ny, nz
        c.limiter, c.solver, c.ct = LIM[limiter], SOLVER[solver], CT[ct]
        c.gamma = state.gamma
        for d in range(3):
            c.dx[d] = (state.xend[d] - state.xbeg[d]) / state.shape[d]
        c.cfl, c.cfl_max_var = cfl, cfl_max_var
        c.outflow, c.reflect, c.eqtsym = outflow, reflect, eqtsym
        c.rk = rk
        c.userdef, c.ud_rho, c.ud_vn = userdef, UD_RHO, UD_VN
        self.cfg = c
        self.shape = (nx, ny, nz)
        self.physics, self.ndim, self.nvar = state.physics, state.ndim, state.nvar
        self.h = lib().orc_create(ctypes.byref(c))
        V = np.ascontiguousarray(state.V)
        U = prim_to_cons(state.physics, state.gamma, V)
        Bs = (np.ascontiguousarray(np.stack(state.Bs)) if state.Bs
              else np.zeros(1))
        lib().orc_set_state(self.h, _dp(V), _dp(U), _dp(Bs))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def step(self, dt: float):
        err = ctypes.c_uint32(0)
        inv = lib().orc_step(self.h, dt, ctypes.byref(err))
        return inv, err.value

    def run(self, nsteps: int, first_dt: float):
        hist = np.zeros(nsteps + 1)
        err = lib().orc_run(self.h, nsteps, first_dt, _dp(hist))
        return hist, err

    def state(self):
        nx, ny, nz = self.shape
        V = np.zeros((self.nvar, nz, ny, nx))
        U = np.zeros_like(V)
        nb = self.ndim if self.physics != HD else 1
        Bs = np.zeros((nb, nz, ny, nx))
        lib().orc_get_state(self.h, _dp(V), _dp(U), _dp(Bs))
        return V, U, (list(Bs) if self.physics != HD else [])

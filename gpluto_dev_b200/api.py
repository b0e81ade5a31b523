"""Python host side of the B200 Godunov step (ctypes over include/gpluto_b200.h).

Mirrors the reference's step interface: :meth:`Solver.AdvanceStep` is
``AdvanceStep(Data*, Grid*, timeStep*)`` (Src/rk_step.cpp:88) for one step
of size dt, :func:`NextTimeStep` is ``NextTimeStep`` (Src/next_time_step.cpp:
20-130), and :meth:`Solver.run` is the main loop of Src/main.cpp:320-485 with
``-maxsteps`` (dt sequence kept on the device).

There is no CPU path.  Constructing a :class:`Solver` without the built
library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import traceback

import numpy as np

from . import ics

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GPLUTO_B200_LIB") or os.path.join(_HERE, "_build",
                                                             "libgpluto_b200.so")

GP_OK, GP_ERR_INVALID, GP_ERR_QUIT, GP_ERR_NO_DEVICE, GP_ERR_IO = 0, -1, -5, -6, -7
GP_ERR_UNSUPPORTED, GP_ERR_CUDA, GP_ERR_TIMEOUT = -2, -3, -8
BC_PERIODIC, BC_OUTFLOW, BC_REFLECTIVE, BC_AXISYMMETRIC, BC_EQTSYMMETRIC = 0, 1, 2, 3, 4
BC_USERDEF = 8
HD, MHD, RMHD = 0, 1, 2
# "ppm", "mp5", "wenoz", "limo3" and "weno3" select those RECONSTRUCTIONs (the limiter then
# plays no part)
LIMITERS = {"flat": 0, "minmod": 1, "vl": 2, "vanleer": 2, "mc": 3, "ppm": 3, "mp5": 3,
            "wenoz": 3, "limo3": 3, "weno3": 3, "vanalbada": 6, "ospre": 7, "umist": 8}
RECONSTRUCTION = {"ppm": 1, "mp5": 2, "wenoz": 3, "limo3": 4, "weno3": 5}
SOLVERS = {"hll": 0, "hllc": 1, "hlld": 2, "tvdlf": 3}
CT_AVG = {"uct_hll": 0, "uct_hlld": 1, "arithmetic": 2, "ct_contact": 3}
FP64, MIXED = 0, 1
LAYOUT_INTERIOR, LAYOUT_REFERENCE = 0, 1
ERR_QUIT = 1 << 15


class GpGridDesc(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("nint", ctypes.c_int * 3), ("nghost", ctypes.c_int),
                ("xbeg", ctypes.c_double * 3), ("xend", ctypes.c_double * 3),
                ("dx", ctypes.POINTER(ctypes.c_double) * 3),
                ("lbound", ctypes.c_int * 3), ("rbound", ctypes.c_int * 3)]


class GpScheme(ctypes.Structure):
    _fields_ = [("physics", ctypes.c_int), ("limiter", ctypes.c_int), ("riemann", ctypes.c_int),
                ("ct_emf", ctypes.c_int), ("rk_stages", ctypes.c_int), ("precision", ctypes.c_int),
                ("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
                ("cfl_max_var", ctypes.c_double), ("small_rho", ctypes.c_double),
                ("small_prs", ctypes.c_double), ("reconstruction", ctypes.c_int)]


class GpStepOut(ctypes.Structure):
    _fields_ = [("err_bits", ctypes.c_uint32), ("invDt_hyp", ctypes.c_double),
                ("dt_next", ctypes.c_double)]


class GPError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gpluto_b200 error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load the in-tree shared library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `python -m gpluto_dev_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, D = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        L.gp_create.argtypes = [ctypes.POINTER(GpGridDesc), ctypes.POINTER(GpScheme), P,
                                ctypes.POINTER(P)]
        L.gp_destroy.argtypes = [P]
        L.gp_upload_state.argtypes = [P, ctypes.c_int, D, D, D, D, D]
        L.gp_download_state.argtypes = [P, ctypes.c_int, D, D, D, D, D]
        L.gp_advance_step.argtypes = [P, ctypes.c_double, ctypes.POINTER(GpStepOut)]
        L.gp_advance_steps.argtypes = [P, ctypes.c_int, D, D, ctypes.POINTER(GpStepOut)]
        L.gp_next_time_step.restype = ctypes.c_double
        L.gp_next_time_step.argtypes = [ctypes.c_double] * 4
        L.gp_device_state.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P * 3)]
        L.gp_launches_per_step.argtypes = [P]
        L.gp_profile_steps.argtypes = [P, ctypes.c_int, D, ctypes.POINTER(ctypes.c_float),
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.gp_kernel_name.restype = ctypes.c_char_p
        L.gp_kernel_name.argtypes = [P, ctypes.c_int]
        L.gp_last_error.restype = ctypes.c_char_p
        L.gp_write_dbl.argtypes = [P, ctypes.c_char_p, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int]
        L.gp_read_dbl.argtypes = [P, ctypes.c_char_p, ctypes.c_int, D, D,
                                  ctypes.POINTER(ctypes.c_int)]
        L.gp_data_minmax.argtypes = [P, D, D, D]
        L.gp_set_userdef_boundary.argtypes = [P, UserdefFn, P]
        _lib = L
    return _lib


def _check(rc):
    if rc != GP_OK:
        raise GPError(rc, lib().gp_last_error().decode())


def _dp(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.dtype == np.float64 and a.flags.c_contiguous
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    # torch tensor (host, possibly pinned)
    return ctypes.cast(a.data_ptr(), ctypes.POINTER(ctypes.c_double))


def NextTimeStep(invDt_hyp: float, cfl: float, cfl_max_var: float, dt: float) -> float:
    """Src/next_time_step.cpp:80,125: min(cfl/invDt_hyp, cfl_max_var*dt)."""
    return lib().gp_next_time_step(invDt_hyp, cfl, cfl_max_var, dt)


@dataclasses.dataclass
class Scheme:
    physics: int = MHD
    limiter: str = "mc"
    riemann: str = "hlld"
    ct_emf: str = "uct_hlld"
    precision: int = FP64
    gamma: float = 5.0 / 3.0
    cfl: float = 0.4
    cfl_max_var: float = 1.1
    small_rho: float = 1e-12
    small_prs: float = 1e-12
    rk: int = 2                # TIME_STEPPING: 2 (RK2) or 3 (RK3)

    def to_c(self) -> GpScheme:
        s = GpScheme()
        s.physics = self.physics
        s.limiter = LIMITERS[self.limiter]
        s.reconstruction = RECONSTRUCTION.get(self.limiter, 0)
        s.riemann = SOLVERS[self.riemann]
        s.ct_emf = CT_AVG[self.ct_emf]
        s.rk_stages = self.rk
        s.precision = self.precision
        s.gamma, s.cfl, s.cfl_max_var = self.gamma, self.cfl, self.cfl_max_var
        s.small_rho, s.small_prs = self.small_rho, self.small_prs
        return s


@dataclasses.dataclass
class StepOut:
    err_bits: int
    invDt_hyp: float
    dt_next: float


class GpUserdefSide(ctypes.Structure):
    _fields_ = [("side", ctypes.c_int), ("stage", ctypes.c_int),
                ("beg", ctypes.c_int * 3), ("end", ctypes.c_int * 3),
                ("dom_beg", ctypes.c_int * 3), ("nint", ctypes.c_int * 3),
                ("dims", ctypes.c_int * 3), ("nvar", ctypes.c_int),
                ("V", ctypes.c_void_p), ("Vs", ctypes.c_void_p * 3)]


UserdefFn = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(GpUserdefSide),
                             ctypes.c_void_p)


class _DeviceArray:
    """A float64 device array described by __cuda_array_interface__."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


class UserdefSide:
    """One USERDEF side as the library hands it to the fill: ``side`` (0..5:
    X1_BEG, X1_END, ... X3_END), ``stage``, the inclusive ghost box
    ``beg``/``end`` (i, j, k array indices), ``dom_beg`` (first domain cell),
    ``nint``, the array extents ``dims``, ``nvar``, the device pointers ``V``
    and ``Vs`` and the ``stream`` the fill's work must go on."""

    def __init__(self, c: GpUserdefSide, stream):
        self.side, self.stage, self.nvar = c.side, c.stage, c.nvar
        self.beg, self.end = tuple(c.beg), tuple(c.end)
        self.dom_beg, self.nint, self.dims = tuple(c.dom_beg), tuple(c.nint), tuple(c.dims)
        self.V, self.Vs = c.V, [c.Vs[e] for e in range(3)]
        self.stream = stream or 0

    def tensors(self):
        """torch views (no copy) of V as [nvar, nz, ny, nx] and of each face
        field as [nz, ny, nx] (None where absent)."""
        import torch
        nx, ny, nz = self.dims
        V = torch.as_tensor(_DeviceArray(self.V, (self.nvar, nz, ny, nx)), device="cuda")
        Vs = [torch.as_tensor(_DeviceArray(p, (nz, ny, nx)), device="cuda") if p else None
              for p in self.Vs]
        return V, Vs

    def torch_stream(self):
        """A torch stream context for ``self.stream``."""
        import torch
        st = (torch.cuda.ExternalStream(self.stream) if self.stream
              else torch.cuda.default_stream())
        return torch.cuda.stream(st)


class Solver:
    """Device-resident state of one grid and its Godunov step."""

    def __init__(self, ndim: int, shape, scheme: Scheme, xbeg=(0.0, 0.0, 0.0),
                 xend=(1.0, 1.0, 1.0), nghost: int = 2, stream=None, outflow: int = 0,
                 reflect: int = 0, eqtsym: int = 0, userdef: int = 0, userdef_fill=None):
        """Side masks: bit 2d (2d+1) of ``outflow`` / ``reflect`` / ``eqtsym``
        / ``userdef`` makes the low (high) side of direction d an OUTFLOW /
        REFLECTIVE / EQTSYMMETRIC / USERDEF boundary; other sides are
        periodic.  USERDEF sides are filled by ``userdef_fill`` (see
        set_userdef_boundary)."""
        g = GpGridDesc()
        g.ndim = ndim
        nx, ny, nz = (tuple(shape) + (1, 1, 1))[:3]
        g.nint[0], g.nint[1], g.nint[2] = nx, ny, (nz if ndim == 3 else 1)
        g.nghost = nghost
        for d in range(3):
            g.xbeg[d], g.xend[d] = xbeg[d], xend[d]
            for e, attr in ((0, "lbound"), (1, "rbound")):
                bit = 2 * d + e
                t = BC_PERIODIC
                if (outflow >> bit) & 1:
                    t = BC_OUTFLOW
                elif (reflect >> bit) & 1:
                    t = BC_REFLECTIVE
                elif (eqtsym >> bit) & 1:
                    t = BC_EQTSYMMETRIC
                elif (userdef >> bit) & 1:
                    t = BC_USERDEF
                getattr(g, attr)[d] = t
        self.outflow, self.reflect, self.eqtsym = outflow, reflect, eqtsym
        self.userdef = userdef
        self._ud_cb = None
        self.ndim, self.shape = ndim, (nx, ny, nz if ndim == 3 else 1)
        self.scheme = scheme
        self.nvar = 5 if scheme.physics == HD else 8
        self.nghost = nghost
        self._gdesc, self._sdesc = g, scheme.to_c()
        h = ctypes.c_void_p()
        sp = ctypes.c_void_p(stream) if stream is not None else None
        _check(lib().gp_create(ctypes.byref(g), ctypes.byref(self._sdesc), sp, ctypes.byref(h)))
        self._h = h
        if userdef_fill is not None:
            self.set_userdef_boundary(userdef_fill)

    def set_userdef_boundary(self, fill):
        """Register the fill of the USERDEF sides: ``fill(side)`` is called
        before every RK stage with a :class:`UserdefSide` and enqueues its
        device work on ``side.stream`` (e.g. torch operations on
        ``side.tensors()`` inside ``with side.torch_stream():``).  It returns
        nothing; an exception aborts the step (GPError GP_ERR_INVALID)."""
        def cb(user, sp, stream):
            try:
                fill(UserdefSide(sp.contents, stream))
                return 0
            except Exception:
                traceback.print_exc()
                return 1
        self._ud_cb = UserdefFn(cb) if fill is not None else None
        _check(lib().gp_set_userdef_boundary(self._h, self._ud_cb or UserdefFn(), None))

    # -- construction helpers -------------------------------------------
    @classmethod
    def from_state(cls, st: "ics.PrimState", scheme: Scheme | None = None, **kw) -> "Solver":
        scheme = scheme or Scheme(physics=st.physics, gamma=st.gamma)
        scheme.gamma = st.gamma
        s = cls(st.ndim, st.shape, scheme, st.xbeg, st.xend, **kw)
        s.upload(st.V, None, st.Bs)
        return s

    def close(self):
        if getattr(self, "_h", None):
            lib().gp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:   # interpreter shutdown: the library may already be gone
            pass

    # -- state transfer ---------------------------------------------------
    def upload(self, V, U=None, Bs=None, layout=LAYOUT_INTERIOR):
        """Host -> device (Uc=None: start-up PrimToCons on the device)."""
        bs = list(Bs or []) + [None] * 3
        _check(lib().gp_upload_state(self._h, layout, _dp(U), _dp(V), _dp(bs[0]), _dp(bs[1]),
                                     _dp(bs[2])))

    def download(self, layout=LAYOUT_INTERIOR):
        """Device -> host: (V, U, Bs) in the interior layout."""
        nx, ny, nz = self.shape
        if layout != LAYOUT_INTERIOR:
            raise ValueError("use download_reference for the ghosted layout")
        V = np.empty((self.nvar, nz, ny, nx))
        U = np.empty_like(V)
        Bs = [np.empty((nz, ny, nx)) for _ in range(self.ndim)] if self.scheme.physics != HD else []
        bs = Bs + [None] * 3
        _check(lib().gp_download_state(self._h, layout, _dp(U), _dp(V), _dp(bs[0]), _dp(bs[1]),
                                       _dp(bs[2])))
        return V, U, Bs

    def reference_shapes(self):
        """Shapes of Data::Uc/Vc and Data::Vs[d] including ghost zones."""
        g = self.nghost
        n = list(self.shape)
        tot = [n[d] + (2 * g if d < self.ndim else 0) for d in range(3)]
        cell = (self.nvar, tot[2], tot[1], tot[0])
        faces = []
        for d in range(self.ndim):
            t = list(tot)
            t[d] += 1
            faces.append((t[2], t[1], t[0]))
        return cell, faces

    # -- stepping ----------------------------------------------------------
    def AdvanceStep(self, dt: float) -> StepOut:
        """One RK2 step (Src/rk_step.cpp:88-593); raises on ERR_QUIT."""
        out = GpStepOut()
        _check(lib().gp_advance_step(self._h, dt, ctypes.byref(out)))
        return StepOut(out.err_bits, out.invDt_hyp, out.dt_next)

    def run(self, nsteps: int, dt: float, history: bool = True):
        """``nsteps`` steps with the device-side dt sequence.

        Returns (dt_after, dt_hist, StepOut)."""
        d = ctypes.c_double(dt)
        hist = np.zeros(max(nsteps, 1)) if history else None
        out = GpStepOut()
        _check(lib().gp_advance_steps(self._h, nsteps, ctypes.byref(d), _dp(hist),
                                      ctypes.byref(out)))
        return d.value, (hist[:nsteps] if history else None), StepOut(out.err_bits,
                                                                       out.invDt_hyp,
                                                                       out.dt_next)

    def profile(self, nsteps: int, dt: float):
        """Mean per-launch kernel times (ms) over ``nsteps`` instrumented steps.

        Returns (list of (name, stage, ms), dt_after)."""
        buf = (ctypes.c_float * 64)()
        nk = ctypes.c_int(0)
        d = ctypes.c_double(dt)
        _check(lib().gp_profile_steps(self._h, nsteps, ctypes.byref(d), buf, 64, ctypes.byref(nk)))
        per = nk.value // self.scheme.rk
        res = [(lib().gp_kernel_name(self._h, q).decode(), 1 + q // per, float(buf[q]))
               for q in range(nk.value)]
        return res, d.value

    # -- output, restart, diagnostics (reference formats) ------------------
    def write_dbl(self, dir: str, nfile: int, t: float, dt: float, nstep: int):
        """WriteData (DBL, single_file) + RestartDump: data.NNNN.dbl, dbl.out,
        restart.out in ``dir`` (Src/write_data.cpp:35-503,
        Src/restart.cpp:423-458)."""
        _check(lib().gp_write_dbl(self._h, os.fsencode(dir), nfile, t, dt, nstep))

    def read_dbl(self, dir: str, nrestart: int):
        """RestartFromFile for a .dbl output (Src/restart.cpp:34-411): loads
        output #nrestart and returns (t, dt, nstep) of its restart record."""
        t, dt, ns = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib().gp_read_dbl(self._h, os.fsencode(dir), nrestart, ctypes.byref(t),
                                 ctypes.byref(dt), ctypes.byref(ns)))
        return t.value, dt.value, ns.value

    def minmax(self):
        """DataMinMax (Src/main.cpp:752-900): (vmin, vmax, mach_max)."""
        vmin, vmax = np.zeros(self.nvar), np.zeros(self.nvar)
        mach = ctypes.c_double()
        _check(lib().gp_data_minmax(self._h, _dp(vmin), _dp(vmax), ctypes.byref(mach)))
        return vmin, vmax, mach.value

    def device_pointers(self):
        u, v = ctypes.c_void_p(), ctypes.c_void_p()
        bs = (ctypes.c_void_p * 3)()
        _check(lib().gp_device_state(self._h, ctypes.byref(u), ctypes.byref(v), ctypes.byref(bs)))
        return u.value, v.value, [bs[i] for i in range(3)]

    @property
    def launches_per_step(self) -> int:
        return lib().gp_launches_per_step(self._h)

"""Batched step: many independent grids advanced together on one GPU.

ctypes front end of the ``gp_batch_*`` entry points of
include/gpluto_b200.h.  A :class:`Batch` owns one device pool; every
admitted grid ("slot") keeps its state there, its own dt sequence (the
reference's NextTimeStep, Src/next_time_step.cpp:80,125, evaluated on the
device) and its own step budget.  :meth:`Batch.advance` runs, per RK stage,
one persistent sweep launch and one persistent EMF/finish launch over all
slots, the launches of a run of steps replayed from a captured CUDA graph.

Each slot advances exactly like :class:`gpluto_dev_b200.api.Solver.run` on
its own (same kernels, same operation order): the FP64 form is
bit-identical to the single-grid FP64 step.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import api, ics


class GpTileShape(ctypes.Structure):
    _fields_ = [("seg", ctypes.c_int), ("cells_per_thread", ctypes.c_int)]


class GpSlotStatus(ctypes.Structure):
    _fields_ = [("steps_done", ctypes.c_int), ("steps_left", ctypes.c_int),
                ("err_bits", ctypes.c_uint32), ("dt", ctypes.c_double),
                ("invDt_hyp", ctypes.c_double)]


_bound = False


def _lib():
    global _bound
    L = api.lib()
    if not _bound:
        P, D = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        G, S = ctypes.POINTER(api.GpGridDesc), ctypes.POINTER(api.GpScheme)
        L.gp_batch_create.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_int, P,
                                      ctypes.POINTER(P)]
        L.gp_batch_destroy.argtypes = [P]
        L.gp_batch_slot_bytes.restype = ctypes.c_size_t
        L.gp_batch_slot_bytes.argtypes = [G, S]
        L.gp_batch_add.argtypes = [P, G, S, ctypes.POINTER(GpTileShape), D, D, D, D,
                                   ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.gp_batch_remove.argtypes = [P, ctypes.c_int]
        L.gp_batch_set_shape.argtypes = [P, ctypes.c_int, ctypes.POINTER(GpTileShape)]
        L.gp_batch_set_ctas.argtypes = [P, ctypes.c_int]
        L.gp_batch_advance.argtypes = [P, ctypes.c_int]
        L.gp_batch_wait.argtypes = [P]
        L.gp_batch_inject_wait_fault.argtypes = [P, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_longlong]
        L.gp_batch_slot_status.argtypes = [P, ctypes.c_int, ctypes.POINTER(GpSlotStatus)]
        L.gp_batch_download.argtypes = [P, ctypes.c_int, D, D, D, D, D]
        L.gp_batch_info.argtypes = [P, ctypes.POINTER(ctypes.c_size_t),
                                    ctypes.POINTER(ctypes.c_size_t),
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        _bound = True
    return L


def grid_desc(st: "ics.PrimState") -> api.GpGridDesc:
    g = api.GpGridDesc()
    g.ndim = st.ndim
    nx, ny, nz = st.shape
    g.nint[0], g.nint[1], g.nint[2] = nx, ny, (nz if st.ndim == 3 else 1)
    g.nghost = 2
    for d in range(3):
        g.xbeg[d], g.xend[d] = st.xbeg[d], st.xend[d]
        g.lbound[d] = g.rbound[d] = 0
    return g


@dataclasses.dataclass
class TileShape:
    seg: int = 0                # pencil segment of the y/z sweeps (0: default)
    cells_per_thread: int = 0   # cells per thread of EMF/finish tiles (0: default)

    def to_c(self) -> GpTileShape:
        return GpTileShape(self.seg, self.cells_per_thread)


@dataclasses.dataclass
class SlotStatus:
    steps_done: int
    steps_left: int
    err_bits: int
    dt: float
    invDt_hyp: float


def slot_bytes(st: "ics.PrimState", scheme: api.Scheme) -> int:
    """Device bytes one slot of this grid and scheme takes from the pool."""
    return int(_lib().gp_batch_slot_bytes(ctypes.byref(grid_desc(st)),
                                          ctypes.byref(scheme.to_c())))


class Batch:
    """A device pool of independent grids advanced together."""

    def __init__(self, pool_bytes: int, max_slots: int, ctas: int = 0, stream=None):
        h = ctypes.c_void_p()
        sp = ctypes.c_void_p(stream) if stream is not None else None
        api._check(_lib().gp_batch_create(pool_bytes, max_slots, ctas, sp, ctypes.byref(h)))
        self._h = h
        self._meta = {}

    def close(self):
        if getattr(self, "_h", None):
            _lib().gp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:   # interpreter shutdown: the library may already be gone
            pass

    def add(self, st: "ics.PrimState", scheme: api.Scheme, dt0: float, nsteps: int,
            shape: TileShape | None = None) -> int:
        """Admit a grid (start-up PrimToCons on the device); returns its slot."""
        scheme = dataclasses.replace(scheme, gamma=st.gamma)
        g, s = grid_desc(st), scheme.to_c()
        V = np.ascontiguousarray(st.V, dtype=np.float64)
        bs = [np.ascontiguousarray(b, dtype=np.float64) for b in st.Bs] + [None] * 3
        slot = ctypes.c_int(-1)
        ts = (shape or TileShape()).to_c()
        api._check(_lib().gp_batch_add(self._h, ctypes.byref(g), ctypes.byref(s), ctypes.byref(ts),
                                       api._dp(V), api._dp(bs[0]), api._dp(bs[1]),
                                       api._dp(bs[2]), dt0, nsteps, ctypes.byref(slot)))
        self._meta[slot.value] = (st.ndim, st.shape, 5 if st.physics == api.HD else 8,
                                  st.physics)
        return slot.value

    def set_shape(self, slot: int, shape: TileShape):
        api._check(_lib().gp_batch_set_shape(self._h, slot, ctypes.byref(shape.to_c())))

    def set_ctas(self, ctas: int):
        """Blocks of the sweep launch (0: all that fit on the device)."""
        api._check(_lib().gp_batch_set_ctas(self._h, ctas))

    def remove(self, slot: int):
        api._check(_lib().gp_batch_remove(self._h, slot))
        self._meta.pop(slot, None)

    def advance(self, nsteps: int):
        """Enqueue nsteps steps of every slot with budget left (asynchronous)."""
        api._check(_lib().gp_batch_advance(self._h, nsteps))

    def wait(self):
        api._check(_lib().gp_batch_wait(self._h))

    def inject_wait_fault(self, slot: int, extra_need: int, spin_limit: int = 0):
        """Test hook: from the next advance, ``slot``'s finish tiles wait for
        ``extra_need`` EMF tiles that do not exist and a wait gives up after
        ``spin_limit`` polls (0: the default limit); wait() then raises
        GPError(GP_ERR_TIMEOUT).  extra_need 0 removes the fault."""
        api._check(_lib().gp_batch_inject_wait_fault(self._h, slot, extra_need, spin_limit))

    def status(self, slot: int) -> SlotStatus:
        st = GpSlotStatus()
        api._check(_lib().gp_batch_slot_status(self._h, slot, ctypes.byref(st)))
        return SlotStatus(st.steps_done, st.steps_left, st.err_bits, st.dt, st.invDt_hyp)

    def download(self, slot: int):
        """(V, U, Bs) of a slot, interior layout."""
        ndim, (nx, ny, nz), nvar, phys = self._meta[slot]
        V = np.empty((nvar, nz, ny, nx))
        U = np.empty_like(V)
        Bs = [np.empty((nz, ny, nx)) for _ in range(ndim)] if phys != api.HD else []
        bs = Bs + [None] * 3
        api._check(_lib().gp_batch_download(self._h, slot, api._dp(U), api._dp(V),
                                            api._dp(bs[0]), api._dp(bs[1]), api._dp(bs[2])))
        return V, U, Bs

    def info(self):
        used, total = ctypes.c_size_t(), ctypes.c_size_t()
        n, ctas = ctypes.c_int(), ctypes.c_int()
        api._check(_lib().gp_batch_info(self._h, ctypes.byref(used), ctypes.byref(total),
                                        ctypes.byref(n), ctypes.byref(ctas)))
        return {"pool_used": used.value, "pool_bytes": total.value, "slots": n.value,
                "ctas": ctas.value}

    @property
    def slots(self):
        return list(self._meta)

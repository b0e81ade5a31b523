"""Seeded synthetic workloads of the batched and serving forms.

* :func:`ensemble` -- independent 2-D ideal-MHD grids, each built like the
  2-D turbulence case (:func:`ics.mhd2d_turbulence`) from its own seed; side
  lengths log-uniform between ``lo`` and ``hi``, alternately square and 2:1;
  half of them FP64 and half mixed precision (alternating in pairs, so both
  shapes occur in both forms).
* :func:`requests` -- a serving stream: Poisson arrivals at rate ``lam``
  (per second) of 2-D/3-D ideal-MHD or HD problems from per-request seeds,
  total cells log-uniform between 32^2 and 128^3, step counts log-uniform
  in [50, 2000], precision FP64 or mixed.

No public dataset exists for these; the generators are the workload.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import api, ics


MHD_SCHEME = dict(physics=api.MHD, limiter="mc", riemann="hlld", ct_emf="uct_hlld",
                  cfl=0.4, cfl_max_var=1.1)
HD_SCHEME = dict(physics=api.HD, limiter="mc", riemann="hllc", ct_emf="uct_hll",
                 cfl=0.4, cfl_max_var=1.1)


def scheme_for(physics: int, precision: int, gamma: float) -> api.Scheme:
    base = MHD_SCHEME if physics == api.MHD else HD_SCHEME
    return api.Scheme(precision=precision, gamma=gamma, **base)


@dataclasses.dataclass
class Member:
    seed: int
    shape: tuple
    precision: int
    state: "ics.PrimState"

    @property
    def scheme(self) -> api.Scheme:
        return scheme_for(self.state.physics, self.precision, self.state.gamma)


def ensemble_shapes(ngrids: int = 512, lo: int = 64, hi: int = 512, seed: int = 2024):
    rng = np.random.default_rng(seed)
    out = []
    for g in range(ngrids):
        side = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        shape = (side, side) if g % 2 == 0 else (side, max(2, side // 2))
        precision = api.FP64 if (g // 2) % 2 == 0 else api.MIXED
        out.append((shape, precision))
    return out


def ensemble(ngrids: int = 512, lo: int = 64, hi: int = 512, seed: int = 2024,
             seed0: int = 0, members=None) -> list:
    """The ensemble's members (or only those whose index is in ``members``)."""
    out = []
    for g, (shape, precision) in enumerate(ensemble_shapes(ngrids, lo, hi, seed)):
        if members is not None and g not in members:
            continue
        st = ics.mhd2d_turbulence(n=shape, seed=seed0 + g)
        out.append(Member(seed0 + g, shape, precision, st))
    return out


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float            # seconds after the stream starts
    physics: int
    ndim: int
    shape: tuple
    nsteps: int
    precision: int
    seed: int

    @property
    def cells(self) -> int:
        return int(np.prod(self.shape))

    def state(self) -> "ics.PrimState":
        if self.physics == api.MHD:
            if self.ndim == 2:
                return ics.mhd2d_turbulence(n=self.shape, seed=self.seed)
            return ics.mhd3d_turbulence(n=self.shape, seed=self.seed)
        return ics.hd_turbulence(n=self.shape, seed=self.seed)

    def scheme(self) -> api.Scheme:
        return scheme_for(self.physics, self.precision, 5.0 / 3.0)


def request_shape(rng, ndim: int, cells_lo: float = 32 ** 2, cells_hi: float = 128 ** 3):
    cells = math.exp(rng.uniform(math.log(cells_lo), math.log(cells_hi)))
    side = max(8, int(round(cells ** (1.0 / ndim))))
    if ndim == 2:
        return (min(side, 2048), min(side, 2048))
    side = min(side, 128)
    return (side, side, side)


def requests(n: int, lam: float, seed: int = 7, steps_lo: int = 50,
             steps_hi: int = 2000) -> list:
    """n requests of a Poisson stream at rate lam per second."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in range(n):
        t += rng.exponential(1.0 / lam)
        physics = api.MHD if rng.uniform() < 0.5 else api.HD
        ndim = 2 if rng.uniform() < 0.5 else 3
        shape = request_shape(rng, ndim)
        nsteps = int(round(math.exp(rng.uniform(math.log(steps_lo), math.log(steps_hi)))))
        precision = api.FP64 if rng.uniform() < 0.5 else api.MIXED
        out.append(Request(r, t, physics, ndim, shape, nsteps, precision, 100000 + r))
    return out

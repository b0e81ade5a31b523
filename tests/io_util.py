"""Loader and parsers for the output/restart fixtures (tests/golden/io): files
written by the reference itself (data.0000.dbl, data.0001.dbl, dbl.out,
restart.out) and the state of the reference restarted from output #1."""
from __future__ import annotations

import os
import struct

import numpy as np

import golden_util as gu
from gpluto_dev_b200 import ics

IO_DIR = os.path.join(gu.GOLDEN_DIR, "io")


def names():
    return sorted(f[:-4] for f in os.listdir(IO_DIR) if f.endswith(".npz"))


class IOCase:
    def __init__(self, name: str):
        z = np.load(os.path.join(IO_DIR, name + ".npz"))
        self.name = name
        self.physics = int(z["physics"])
        self.ndim = int(z["ndim"])
        self.shape = tuple(int(x) for x in z["shape"])
        self.gamma = float(z["gamma"])
        Bs0 = list(z["Bs0"]) if self.physics != ics.PHYS_HD else []
        self.ic = ics.PrimState(self.physics, self.ndim, self.shape, self.gamma,
                                z["V0"].copy(), [b.copy() for b in Bs0])
        self.files = {"data.0000.dbl": z["dbl0"].tobytes(), "data.0001.dbl": z["dbl1"].tobytes(),
                      "dbl.out": z["dbl_out"].tobytes(), "restart.out": z["restart_out"].tobytes()}
        self.rst_V, self.rst_U = z["rst_V"], z["rst_U"]
        self.rst_Bs = list(z["rst_Bs"]) if self.physics != ics.PHYS_HD else []
        self.rst_dt = z["rst_dt"]
        self.every, self.nsteps = int(z["every"]), int(z["nsteps"])
        self.limiter = gu.LIMITER[str(z["limiter"])]
        self.solver = str(z["solver"])
        self.ct = gu.CT[str(z["ct"])]
        self.cfl, self.cfl_max_var = float(z["cfl"]), float(z["cfl_max_var"])
        self.first_dt = float(z["first_dt"])
        self.outflow = int(z["outflow"])
        self.nvar = 5 if self.physics == ics.PHYS_HD else 8

    def write_files(self, d: str, which=("data.0001.dbl", "dbl.out", "restart.out")):
        for f in which:
            with open(os.path.join(d, f), "wb") as fh:
                fh.write(self.files[f])


def restart_records(b: bytes):
    """(t, dt, nstep, nfile[16]) of each 256-byte Restart record."""
    out = []
    for r in range(len(b) // 256):
        rec = b[256 * r:256 * (r + 1)]
        t, dt = struct.unpack_from("<2d", rec, 0)
        nstep, = struct.unpack_from("<i", rec, 112)
        nfile = struct.unpack_from("<16i", rec, 116)
        out.append((t, dt, nstep, nfile))
    return out


def read_dbl(b: bytes, c: IOCase):
    """Split a data.NNNN.dbl of case c into V [nvar][nz][ny][nx] and the
    staggered fields (one extra face along their own direction)."""
    a = np.frombuffer(b, "<f8")
    nx, ny, nz = c.shape
    n = nx * ny * nz
    V = a[:c.nvar * n].reshape(c.nvar, nz, ny, nx)
    off = c.nvar * n
    Bs = []
    if c.physics != ics.PHYS_HD:
        for d in range(c.ndim):
            m = [nx, ny, nz]
            m[d] += 1
            k = m[0] * m[1] * m[2]
            Bs.append(a[off:off + k].reshape(m[2], m[1], m[0]))
            off += k
    assert off == a.size
    return V, Bs

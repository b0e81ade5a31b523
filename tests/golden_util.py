"""Helpers to load the committed golden fixtures (reference outputs)."""
from __future__ import annotations

import glob
import os

import numpy as np

from gpluto_dev_b200 import ics

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

LIMITER = {"MC_LIM": "mc", "VANLEER_LIM": "vl", "MINMOD_LIM": "minmod", "FLAT_LIM": "flat",
           "VANALBADA_LIM": "vanalbada", "OSPRE_LIM": "ospre", "UMIST_LIM": "umist"}
CT = {"UCT_HLLD": "uct_hlld", "UCT_HLL": "uct_hll", "ARITHMETIC": "arithmetic",
      "CT_CONTACT": "ct_contact",
      "none": "uct_hll"}


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


class Golden:
    def __init__(self, name: str):
        z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
        self.name = name
        self.physics = int(z["physics"])
        self.ndim = int(z["ndim"])
        self.shape = tuple(int(x) for x in z["shape"])
        self.gamma = float(z["gamma"])
        Bs0 = list(z["Bs0"]) if self.physics != ics.PHYS_HD else []
        self.ic = ics.PrimState(self.physics, self.ndim, self.shape, self.gamma,
                                z["V0"].copy(), [b.copy() for b in Bs0])
        self.V, self.U = z["V"], z["U"]
        self.Bs = list(z["Bs"]) if self.physics != ics.PHYS_HD else []
        self.dt = z["dt"]
        self.nsteps = int(z["nsteps"])
        self.limiter = LIMITER[str(z["limiter"])]
        self.solver = str(z["solver"])
        self.ct = CT[str(z["ct"])]
        self.cfl = float(z["cfl"])
        self.cfl_max_var = float(z["cfl_max_var"])
        self.first_dt = float(z["first_dt"])
        self.reconstruction = str(z["reconstruction"]) if "reconstruction" in z else "LINEAR"
        self.outflow = int(z["outflow"]) if "outflow" in z else 0
        self.reflect = int(z["reflect"]) if "reflect" in z else 0
        self.eqtsym = int(z["eqtsym"]) if "eqtsym" in z else 0
        self.userdef = int(z["userdef"]) if "userdef" in z else 0
        # side types as keyword arguments of the oracle and of api.Solver
        self.bc = dict(outflow=self.outflow, reflect=self.reflect, eqtsym=self.eqtsym)
        if self.userdef:
            self.bc["userdef"] = self.userdef
        self.rk = int(z["rk"]) if "rk" in z else 2
        if self.reconstruction == "PARABOLIC":
            self.limiter = "ppm"
        elif self.reconstruction == "MP5":
            self.limiter = "mp5"
        elif self.reconstruction == "WENOZ":
            self.limiter = "wenoz"
        elif self.reconstruction == "LimO3":
            self.limiter = "limo3"
        elif self.reconstruction == "WENO3":
            self.limiter = "weno3"

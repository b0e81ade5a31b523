"""Build the sm_100a shared library of the Godunov step (in-tree).

    python -m gpluto_dev_b200.build

Produces gpluto_dev_b200/_build/libgpluto_b200.so from csrc/ with nvcc:
gp_launch.cu twice (FP64 form with -fmad=false so the plain form keeps the
reference's rounding sequence; mixed form with contraction), gp_api.cu for
the C ABI, and the batched step (gp_batch_tiles.cu four times + gp_batch.cu) as
relocatable device code with its device-link object.  Objects are rebuilt
only when a source is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libgpluto_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]

# The mixed form's FP32 arithmetic (reconstruction, Riemann fluxes, UCT
# EMFs) uses the approximate FP32 divide and square root and flushes FP32
# denormals: its sweeps are issue-bound, and these cut their instruction
# count by about a fifth.  These flags touch single precision only, so the FP64
# accumulation, CT update and con2prim of that form stay IEEE.
MIXED_FP32 = ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
# The stage kernels are instantiated per form and per scheme group (GP_PART:
# 0 HD, 1 MHD with HLLD/HLL, 2 RMHD, 3 MHD with Lax-Friedrichs/HLLC) in eight
# units that compile in parallel.
UNITS = [
    *[(f"gp_launch_fp64_p{p}.o", "gp_launch.cu", ["-DGP_MIXED=0", f"-DGP_PART={p}", "-fmad=false"])
      for p in (1, 2, 3, 0)],
    *[(f"gp_launch_mixed_p{p}.o", "gp_launch.cu", ["-DGP_MIXED=1", f"-DGP_PART={p}", *MIXED_FP32])
      for p in (1, 2, 3, 0)],
    ("gp_launch_dispatch.o", "gp_launch_dispatch.cu", []),
    ("gp_api.o", "gp_api.cu", ["-fmad=false"]),
    ("gp_noalloc.o", "gp_noalloc.cu", ["-fmad=false"]),
]
# Batched step: relocatable device code, so that one persistent kernel can
# call the tile bodies of both forms (each compiled with its own contraction
# rule).  Sweep tiles: 168 registers = 3 blocks of 128 threads per SM, as the
# single-grid sweeps; EMF/finish tiles: 64 registers = 8 blocks per SM.
SWEEP_RDC = ["-rdc=true", "-maxrregcount=168", "-DGP_BATCH_PART=0"]
CELL_RDC = ["-rdc=true", "-maxrregcount=64", "-DGP_BATCH_PART=1"]
RDC_UNITS = [
    ("gp_batch_sweeps_fp64.o", "gp_batch_tiles.cu", ["-DGP_MIXED=0", "-fmad=false", *SWEEP_RDC]),
    ("gp_batch_sweeps_mixed.o", "gp_batch_tiles.cu", ["-DGP_MIXED=1", *MIXED_FP32, *SWEEP_RDC]),
    ("gp_batch_cells_fp64.o", "gp_batch_tiles.cu", ["-DGP_MIXED=0", "-fmad=false", *CELL_RDC]),
    ("gp_batch_cells_mixed.o", "gp_batch_tiles.cu", ["-DGP_MIXED=1", *MIXED_FP32, *CELL_RDC]),
    ("gp_batch.o", "gp_batch.cu", ["-fmad=false", "-rdc=true"]),
]
DLINK = "gp_batch_dlink.o"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _deps() -> list:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(os.path.dirname(HERE), "include", "gpluto_b200.h"),
        os.path.abspath(__file__)]  # the flags live here


def build(verbose: bool = False, jobs: int = 0) -> str:
    os.makedirs(OUT, exist_ok=True)
    newest = max(os.path.getmtime(p) for p in _deps())
    procs = []
    objs = []
    rdc_objs = []
    for obj, src, flags in UNITS + RDC_UNITS:
        o = os.path.join(OUT, obj)
        objs.append(o)
        if (obj, src, flags) in RDC_UNITS:
            rdc_objs.append(o)
        if os.path.exists(o) and os.path.getmtime(o) >= newest:
            continue
        cmd = [nvcc(), *ARCH, *BASE, *flags, "-c", os.path.join(CSRC, src), "-o", o]
        if verbose:
            print(" ".join(cmd))
        procs.append(cmd)
    # at most `jobs` (default: the core count) compilers at a time, largest
    # units first as listed
    jobs = jobs or os.cpu_count() or 4
    running = []
    for cmd in procs + [None] * jobs:
        while len(running) >= jobs or (cmd is None and running):
            c, p = running.pop(0)
            out, _ = p.communicate()
            if p.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + " ".join(c) + "\n" + out.decode()[-6000:])
            if cmd is not None:
                break
        if cmd is not None:
            running.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                  stderr=subprocess.STDOUT)))
    dl = os.path.join(OUT, DLINK)
    if (not os.path.exists(dl)) or os.path.getmtime(dl) < max(os.path.getmtime(o) for o in rdc_objs):
        subprocess.run([nvcc(), *ARCH, "-Xcompiler", "-fPIC", "-dlink", *rdc_objs, "-o", dl],
                       check=True)
    objs.append(dl)
    if (not os.path.exists(LIB)) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

"""Reference runs at the full sizes of the three single-grid workloads.

Run in a container that has the reference tree (``GP_REFERENCE_ROOT``, by
default ``../reference`` beside the repository):

    python tests/golden/make_atsize.py [mhd2d_256 | mhd3d_blast_256 | rmhd3d_192] ...

Each case builds the reference serial binary into its own directory under
``oracle/_ref/`` (oracle/ref/build_ref.py: reference sources compiled in
place, ``g++ -O3``), writes the seeded initial condition that ``bench.py``
and the GPU tests use (gpluto_dev_b200/ics.py), runs 100 steps with FTZ/DAZ
off and stores a compact summary of the final state (``tests/atsize_util``:
per-plane digests, sums and maxima, a strided cell sample, the centre
x-line) with the reference's dt history as ``atsize/<name>.npz``.  The full
dump stays in ``oracle/_ref/`` (not committed).

Cost on one core of an 8-vCPU Xeon: 2-D 256^2 about 10 s, 3-D MHD 256^3
about 1.5-2 h (11 GB of memory), 3-D RMHD 192^3 a few hours.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from gpluto_dev_b200 import ics  # noqa: E402
import atsize_util  # noqa: E402
import build_ref as br  # noqa: E402

NSTEPS = 100
# name: (generator, kwargs, RefConfig kwargs) -- the workloads of bench.py
CASES = {
    "mhd2d_256": (ics.mhd2d_turbulence, dict(n=(256, 256), seed=0),
                  dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                       ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4)),
    "mhd3d_blast_256": (ics.mhd3d_blast, dict(n=(256, 256, 256), seed=1),
                        dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                             ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4)),
    "rmhd3d_192": (ics.rmhd3d_turbulence, dict(n=(192, 192, 192), seed=1),
                   dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                        ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4)),
}


def make(name: str) -> str:
    gen, kw, rc = CASES[name]
    st = gen(**kw)
    cfg = br.RefConfig(name=f"atsize_{name}", n=st.shape, **rc)
    binary = br.build(cfg)
    d = os.path.dirname(binary)
    icp = os.path.join(d, "ic.bin")
    dmp = os.path.join(d, "out.dump")
    ics.write_ic(icp, st)
    del st
    t0 = time.time()
    dump = br.run_ref(binary, icp, NSTEPS, dmp)
    wall = time.time() - t0
    summ = atsize_util.summarize(dump.V, dump.U, dump.Bs, dump.ndim)
    os.makedirs(os.path.join(HERE, "atsize"), exist_ok=True)
    out = os.path.join(HERE, "atsize", f"{name}.npz")
    np.savez_compressed(out, physics=dump.physics, ndim=dump.ndim,
                        shape=np.array(dump.shape), dt=dump.dt, nsteps=NSTEPS,
                        step_wall=np.diff(dump.wall), run_wall=wall, **summ)
    return out


if __name__ == "__main__":
    for nm in sys.argv[1:] or list(CASES):
        p = make(nm)
        print(f"{nm}: {os.path.getsize(p) / 1024:.0f} KiB", flush=True)

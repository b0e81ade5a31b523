"""Reference output files for the drop-in driver test.

Run in a container that has the reference tree (``GP_REFERENCE_ROOT``, by
default ``../reference`` beside the repository) after building the library:

    python tests/golden/make_dropin.py

Builds the reference serial binary for the 2-D ideal-MHD 256^2 workload
(PLM-MC, HLLD, UCT_HLLD, RK2, CFL 0.4; oracle/ref/build_ref.py), runs it
from the seeded initial condition with .dbl output every 100 steps, and
stores the SHA-256 and size of data.0000.dbl, data.0001.dbl (the state after
100 steps), dbl.out and the defined fields of restart.out's records as
``dropin/mhd2d_256.json``.  It also
builds the drop-in driver (oracle/ref/build_dropin.py: the same reference
sources with AdvanceStep replaced by the B200 library), which the GPU test
runs and whose files must have these digests.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))

from gpluto_dev_b200 import ics  # noqa: E402
import build_dropin as bd  # noqa: E402
import build_ref as br  # noqa: E402

EVERY, NSTEPS = 100, 101


def config():
    return br.RefConfig(name="mhd2d_mc_lim_hlld_uct_hlld", physics="MHD", ndim=2,
                        n=(256, 256, 1), limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLLD",
                        cfl=0.4, first_dt=1e-4)


def initial_condition():
    return ics.mhd2d_turbulence(n=(256, 256), seed=0)


# Restart records (Src/structs.hpp:382-390) are 256 bytes: t, dt, param[12],
# nstep, nfile[16] fill bytes 0-180; nfileParticles[16], fill[10] and the
# padding are not all set by the reference (two identical reference runs
# differ there), so only the first 180 bytes of each record are compared.
RESTART_RECORD, RESTART_DEFINED = 256, 180


def restart_defined(b: bytes) -> bytes:
    return b"".join(b[r:r + RESTART_DEFINED] for r in range(0, len(b), RESTART_RECORD))


def digests(files: dict) -> dict:
    out = {}
    for f, b in files.items():
        if f == "restart.out":
            b = restart_defined(b)
        out[f] = {"sha256": hashlib.sha256(b).hexdigest(), "bytes": len(b)}
    return out


if __name__ == "__main__":
    cfg = config()
    ref = br.build(cfg)
    with tempfile.TemporaryDirectory() as tmp:
        icp = os.path.join(tmp, "ic.bin")
        ics.write_ic(icp, initial_condition())
        wd = os.path.join(tmp, "run")
        os.makedirs(wd)
        files = bd.run_dbl(ref, icp, EVERY, NSTEPS, wd)
    out = {"every": EVERY, "nsteps": NSTEPS, "files": digests(files)}
    os.makedirs(os.path.join(HERE, "dropin"), exist_ok=True)
    with open(os.path.join(HERE, "dropin", "mhd2d_256.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))
    print("drop-in driver:", bd.build(cfg))

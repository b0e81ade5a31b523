"""The reference's own C++ driver calling the B200 library (the C ABI as
INTEGRATION.md describes it), compiled from the reference sources by
oracle/ref/build_dropin.py: AdvanceStep (Src/main.cpp:446) replaced by
gp_advance_step, everything else -- NextTimeStep, output, restart dump --
the reference's code.  On the 2-D ideal-MHD 256^2 workload with .dbl output
every 100 steps, its data.0000.dbl, data.0001.dbl (the state after 100
steps) and dbl.out must be byte-identical to the files the reference's
serial CPU build writes, and so must restart.out's records apart from the
bytes the reference leaves unset (SHA-256 digests in tests/golden/dropin/,
made by tests/golden/make_dropin.py)."""
import hashlib
import json
import os
import sys
import tempfile

import pytest

from gpluto_dev_b200 import ics

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "oracle", "_ref", "dropin_mhd2d_mc_lim_hlld_uct_hlld", "pluto")
FIX = os.path.join(ROOT, "tests", "golden", "dropin", "mhd2d_256.json")


def test_dropin_driver_writes_the_reference_files():
    if not os.path.exists(BINARY):
        pytest.skip("the drop-in driver is built from the reference tree (build())")
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
    import build_dropin as bd
    ref = json.load(open(FIX))
    with tempfile.TemporaryDirectory() as tmp:
        icp = os.path.join(tmp, "ic.bin")
        ics.write_ic(icp, ics.mhd2d_turbulence(n=(256, 256), seed=0))
        wd = os.path.join(tmp, "run")
        os.makedirs(wd)
        files = bd.run_dbl(BINARY, icp, ref["every"], ref["nsteps"], wd, timeout=600)
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_dropin as md
    assert sorted(files) == sorted(ref["files"])
    for name, want in ref["files"].items():
        got = files[name] if name != "restart.out" else md.restart_defined(files[name])
        assert len(got) == want["bytes"], name
        assert hashlib.sha256(got).hexdigest() == want["sha256"], name

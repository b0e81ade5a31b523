"""The output/restart fixtures against the oracle (CPU): restarting the oracle
from the reference's own data.0001.dbl (Uc = PrimToCons(Vc), the record's dt)
reproduces the reference's restarted run bit for bit, which pins what a
restart means (Src/restart.cpp:34-283) before the device is asked to do it."""
import os
import sys

import numpy as np
import pytest

import io_util as iu
from gpluto_dev_b200 import ics

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import oracle as orc  # noqa: E402  (checker only)

PERIODIC = [n for n in iu.names() if iu.IOCase(n).outflow == 0]


@pytest.mark.parametrize("name", iu.names())
def test_fixture_files_are_consistent(name):
    c = iu.IOCase(name)
    lines = c.files["dbl.out"].decode().splitlines()
    assert len(lines) == 2 and lines[1].split()[:1] == ["1"]
    recs = iu.restart_records(c.files["restart.out"])
    assert [r[3][1] for r in recs] == [0, 1] and recs[1][2] == c.every
    V0, _ = iu.read_dbl(c.files["data.0000.dbl"], c)
    np.testing.assert_array_equal(V0, c.ic.V)          # output #0 is the initial state


@pytest.mark.parametrize("name", PERIODIC)
def test_oracle_restart_from_reference_output_matches_reference_restart(name):
    c = iu.IOCase(name)
    V, Bs = iu.read_dbl(c.files["data.0001.dbl"], c)
    # periodic: the last face of each staggered field is the first one
    for d, b in enumerate(Bs):
        first = np.take(b, [0], axis=2 - d)
        last = np.take(b, [b.shape[2 - d] - 1], axis=2 - d)
        np.testing.assert_array_equal(first, last)
    Bl = [np.ascontiguousarray(np.take(b, range(b.shape[2 - d] - 1), axis=2 - d))
          for d, b in enumerate(Bs)]
    st = ics.PrimState(c.physics, c.ndim, c.shape, c.gamma, V.copy(), Bl)
    kw = dict(limiter=c.limiter, solver=c.solver)
    if c.physics != ics.PHYS_HD:
        kw["ct"] = c.ct
    o = orc.Oracle(st, cfl=c.cfl, **kw)
    t, dt, nstep, _ = iu.restart_records(c.files["restart.out"])[1]
    hist, err = o.run(c.nsteps - c.every, dt)
    np.testing.assert_array_equal(hist, c.rst_dt)
    Vo, Uo, Bo = o.state()
    np.testing.assert_array_equal(Vo, c.rst_V)
    np.testing.assert_array_equal(Uo, c.rst_U)
    for a, b in zip(Bo, c.rst_Bs):
        np.testing.assert_array_equal(a, b)

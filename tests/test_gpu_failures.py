"""Failure detection on the GPU, with every failure made on the host.

* A poisoned state (negative density, a NaN face field) uploaded to a handle
  makes the step return GP_ERR_QUIT with the error bits the reference raises
  (Src/mappers3D.cpp:113-176, Src/MHD/hlld.cpp:477-511; the oracle, pinned
  to the reference, gives the expected bits); the handle then steps a clean
  state exactly as a fresh one does.
* In a batch, a poisoned slot stops while its neighbour advances exactly as
  it does alone.
* The batch's bounded dependency wait: a slot's finish tiles are told to wait
  for EMF tiles that never come (host-side injection) with a short poll
  limit; the wait runs out, the launch ends, gp_batch_wait reports
  GP_ERR_TIMEOUT, and the same batch then advances a clean slot correctly.
No kernel is made to fault, trap or hang.
"""
import ctypes

import numpy as np
import pytest

import oracle as orc
from gpluto_dev_b200 import api, ics
from gpluto_dev_b200 import batch as gb

pytestmark = pytest.mark.gpu



def _poison(kind):
    st = ics.mhd3d_turbulence(n=(12, 10, 8), seed=5)
    bad = st.copy()
    if kind == "negative_density":
        bad.V[0][3, 4, 5] = -0.5
    elif kind == "nan_face":
        bad.Bs[1][2, 3, 4] = np.nan
    else:                       # negative pressure: flagged, not fatal
        bad.V[7][3, 4, 5] = -0.5
    return st, bad


def _step_raw(s, dt):
    out = api.GpStepOut()
    rc = api.lib().gp_advance_step(s._h, dt, ctypes.byref(out))
    return rc, out.err_bits


@pytest.mark.parametrize("kind", ["negative_density", "nan_face", "negative_pressure"])
def test_poisoned_state_reports_reference_bits_and_handle_recovers(kind):
    st, bad = _poison(kind)
    o = orc.Oracle(bad, limiter="mc", solver="hlld", ct="uct_hlld")
    _, oerr = o.run(1, 1e-4)
    sch = api.Scheme(physics=api.MHD, gamma=st.gamma)
    s = api.Solver.from_state(bad, sch)
    rc, err = _step_raw(s, 1e-4)
    assert err == oerr, (hex(err), hex(oerr))
    assert rc == (api.GP_ERR_QUIT if oerr & api.ERR_QUIT else api.GP_OK)
    # the same handle, given a clean state, steps exactly as a fresh one
    s.upload(st.V, None, st.Bs)
    rc, err = _step_raw(s, 1e-4)
    assert rc == api.GP_OK and err == 0
    fresh = api.Solver.from_state(st, sch)
    fresh.AdvanceStep(1e-4)
    for a, b in zip(s.download(), fresh.download()):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_batch_poisoned_slot_stops_while_its_neighbour_advances():
    st, bad = _poison("nan_face")
    good = ics.mhd3d_turbulence(n=(16, 12, 10), seed=6)
    sch = api.Scheme(physics=api.MHD)
    b = gb.Batch(1 << 28, 4)
    sg = b.add(good, sch, 1e-4, 5)
    sb = b.add(bad, sch, 1e-4, 5)
    b.advance(5)
    b.wait()
    stb = b.status(sb)
    assert stb.err_bits & api.ERR_QUIT and stb.steps_left == 0 and stb.steps_done == 1
    stg = b.status(sg)
    assert stg.err_bits & api.ERR_QUIT == 0 and stg.steps_done == 5
    s = api.Solver.from_state(good, dataclass_gamma(sch, good))
    s.run(5, 1e-4)
    for x, y in zip(b.download(sg), s.download()):
        for p, q in zip(x, y):
            np.testing.assert_array_equal(p, q)
    b.close()


def dataclass_gamma(sch, st):
    import dataclasses
    return dataclasses.replace(sch, gamma=st.gamma)


def test_batch_dependency_wait_runs_out_and_reports_timeout():
    st = ics.mhd2d_turbulence(n=(48, 40), seed=8)
    sch = api.Scheme(physics=api.MHD)
    b = gb.Batch(1 << 28, 4)
    s0 = b.add(st, sch, 1e-4, 3)
    # slot s0's finish tiles wait for 1000 EMF tiles that do not exist; a
    # wait gives up after 2000 polls (about a millisecond)
    b.inject_wait_fault(s0, 1000, 2000)
    b.advance(1)
    with pytest.raises(api.GPError) as ei:
        b.wait()
    assert ei.value.code == api.GP_ERR_TIMEOUT
    # the context and the batch stay usable: remove the fault and the slot,
    # admit the grid again and compare with the single-grid step
    b.inject_wait_fault(s0, 0, 0)
    b.remove(s0)
    s1 = b.add(st, sch, 1e-4, 3)
    b.advance(3)
    b.wait()
    assert b.status(s1).steps_done == 3
    s = api.Solver.from_state(st, dataclass_gamma(sch, st))
    s.run(3, 1e-4)
    for x, y in zip(b.download(s1), s.download()):
        for p, q in zip(x, y):
            np.testing.assert_array_equal(p, q)
    b.close()

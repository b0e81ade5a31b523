"""Output, restart and the min/max diagnostic on the device, against files
written by the reference itself (tests/golden/io):

* gp_write_dbl after 0 and `every` steps gives the reference's data.0000.dbl
  and data.0001.dbl byte for byte, its dbl.out text, and restart.out records
  with the same t, dt, step and file numbers;
* gp_read_dbl of the reference's output #1, then the remaining steps, gives
  the reference's own restarted run bit for bit (state and dt sequence);
* gp_data_minmax equals the same reductions taken on the downloaded state.
"""
import numpy as np
import pytest

import io_util as iu
from gpluto_dev_b200 import api

pytestmark = pytest.mark.gpu


def solver(c):
    sch = api.Scheme(physics=c.physics, limiter=c.limiter, riemann=c.solver, ct_emf=c.ct,
                     gamma=c.gamma, cfl=c.cfl, cfl_max_var=c.cfl_max_var)
    return api.Solver.from_state(c.ic, sch, outflow=c.outflow)


@pytest.mark.parametrize("name", iu.names())
def test_write_dbl_reproduces_reference_files(name, tmp_path):
    c = iu.IOCase(name)
    s = solver(c)
    s.write_dbl(str(tmp_path), 0, 0.0, c.first_dt, 0)
    dt_next, hist, out = s.run(c.every, c.first_dt)
    t = 0.0
    for d in hist:               # Dts->time += dt, step by step
        t += float(d)
    s.write_dbl(str(tmp_path), 1, t, dt_next, c.every)
    s.close()
    for f in ("data.0000.dbl", "data.0001.dbl", "dbl.out"):
        assert (tmp_path / f).read_bytes() == c.files[f], f
    ours = iu.restart_records((tmp_path / "restart.out").read_bytes())
    ref = iu.restart_records(c.files["restart.out"])
    assert ours == ref


@pytest.mark.parametrize("name", iu.names())
def test_restart_from_reference_output_continues_bit_exact(name, tmp_path):
    c = iu.IOCase(name)
    c.write_files(str(tmp_path))
    s = solver(c)
    t, dt, nstep = s.read_dbl(str(tmp_path), 1)
    rt, rdt, rstep, _ = iu.restart_records(c.files["restart.out"])[1]
    assert (t, dt, nstep) == (rt, rdt, rstep)
    dt_next, hist, out = s.run(c.nsteps - c.every, dt)
    np.testing.assert_array_equal(hist, c.rst_dt[:-1])
    assert dt_next == c.rst_dt[-1]
    V, U, Bs = s.download()
    s.close()
    np.testing.assert_array_equal(V, c.rst_V)
    np.testing.assert_array_equal(U, c.rst_U)
    for a, b in zip(Bs, c.rst_Bs):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", iu.names())
def test_data_minmax_matches_host_reduction(name):
    c = iu.IOCase(name)
    s = solver(c)
    s.run(c.every, c.first_dt)
    vmin, vmax, mach = s.minmax()
    V, _, _ = s.download()
    s.close()
    np.testing.assert_array_equal(vmin, V.reshape(c.nvar, -1).min(axis=1))
    np.testing.assert_array_equal(vmax, V.reshape(c.nvar, -1).max(axis=1))
    cs = np.sqrt(V[c.nvar - 1] / V[0])
    m = np.maximum(np.maximum(np.abs(V[1]) / cs, np.abs(V[2]) / cs), np.abs(V[3]) / cs)
    assert mach == m.max()


def test_read_dbl_reports_missing_files(tmp_path):
    c = iu.IOCase(iu.names()[0])
    s = solver(c)
    with pytest.raises(api.GPError) as ei:
        s.read_dbl(str(tmp_path), 1)
    assert ei.value.code == api.GP_ERR_IO
    c.write_files(str(tmp_path), which=("dbl.out", "restart.out"))
    with pytest.raises(api.GPError) as ei:          # no data file
        s.read_dbl(str(tmp_path), 1)
    assert ei.value.code == api.GP_ERR_IO
    with pytest.raises(api.GPError) as ei:          # no such output number
        s.read_dbl(str(tmp_path), 5)
    assert ei.value.code == api.GP_ERR_IO
    s.close()

"""Special-relativistic MHD on the GPU against the reference and the oracle.

The RMHD fast speeds come from a quartic solved with acos/cos/sin
(Src/RMHD/rmhd.hpp:390-452).  The GPU evaluates those three correctly
rounded (gpluto_dev_b200/csrc/gp_crmath.cuh); the reference calls glibc,
whose results differ from the correctly rounded ones in about 0.04-0.13% of
the calls.  So the GPU's FP64 form is checked

* bit for bit against the oracle run with correctly rounded trigonometry
  (``orc.set_cr_trig``) and the strict Riemann-state rule that the kernels
  use (``orc.set_rmhd_strict``), on every RMHD reference fixture's initial
  condition;
* against the reference's own outputs to 1e-11 relative L-infinity per
  variable, or, where glibc's rounding alone moves the reference further
  (the 2-D HLLD fixture: the oracle with correctly rounded trigonometry is
  2.5e-10 away), to that oracle's own distance from the reference.
"""
import numpy as np
import pytest

import golden_util as gu
import oracle as orc
from gpluto_dev_b200 import api, ics

pytestmark = pytest.mark.gpu

RMHD_FIXTURES = [n for n in gu.names() if n.startswith("rmhd")]
RTOL_REF = 1e-11


def rel_linf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def solver(st, lim, rs, cfl=0.3, precision=api.FP64, outflow=0, reflect=0, eqtsym=0, rk=2):
    sch = api.Scheme(physics=api.RMHD, limiter=lim, riemann=rs, ct_emf="uct_hll",
                     precision=precision, gamma=st.gamma, cfl=cfl, rk=rk)
    return api.Solver.from_state(st, sch, outflow=outflow, reflect=reflect, eqtsym=eqtsym)


def cr_oracle(st, nsteps, first_dt, **kw):
    """The oracle with correctly rounded acos/cos/sin and the strict rule."""
    orc.set_cr_trig(True)
    orc.set_rmhd_strict(True)
    try:
        o = orc.Oracle(st, **kw)
        hist, err = o.run(nsteps, first_dt)
        return hist, err, o.state()
    finally:
        orc.set_cr_trig(False)
        orc.set_rmhd_strict(False)


def worst_rel_linf(V, U, Bs, G):
    return max([rel_linf(U[nv], G.U[nv]) for nv in range(8)]
               + [rel_linf(V[nv], G.V[nv]) for nv in range(8)]
               + [rel_linf(a, b) for a, b in zip(Bs, G.Bs)])


@pytest.mark.parametrize("name", RMHD_FIXTURES)
def test_rmhd_fp64_bitwise_vs_correctly_rounded_oracle(name):
    g = gu.Golden(name)
    oh, oerr, (Vo, Uo, Bo) = cr_oracle(g.ic, g.nsteps, g.first_dt, limiter=g.limiter,
                                       solver=g.solver, ct=g.ct, cfl=g.cfl, **g.bc, rk=g.rk)
    s = solver(g.ic, g.limiter, g.solver, g.cfl, **g.bc, rk=g.rk)
    _, hist, out = s.run(g.nsteps, g.first_dt)
    V, U, Bs = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, oh[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)
    for a, b in zip(Bs, Bo):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", RMHD_FIXTURES)
def test_rmhd_fp64_matches_reference_fixture(name):
    g = gu.Golden(name)
    _, _, (Vo, Uo, Bo) = cr_oracle(g.ic, g.nsteps, g.first_dt, limiter=g.limiter,
                                   solver=g.solver, ct=g.ct, cfl=g.cfl, **g.bc, rk=g.rk)
    glibc_part = worst_rel_linf(Vo, Uo, Bo, g)      # glibc's rounding alone
    s = solver(g.ic, g.limiter, g.solver, g.cfl, **g.bc, rk=g.rk)
    _, hist, out = s.run(g.nsteps, g.first_dt)
    V, U, Bs = s.download()
    assert out.err_bits & api.ERR_QUIT == 0
    np.testing.assert_allclose(hist, g.dt[:-1], rtol=RTOL_REF)
    assert worst_rel_linf(V, U, Bs, g) <= max(RTOL_REF, glibc_part), glibc_part


def test_rmhd_fp64_smooth_case_matches_oracle():
    # smooth 3-D RMHD (no error bits raised), 20 steps: bit for bit
    st = ics.rmhd3d_turbulence(n=(24, 24, 24), seed=5, lorentz_max=3.0, sigma=0.3, p0=1.0)
    oh, oerr, (Vo, Uo, Bo) = cr_oracle(st, 20, 1e-4, limiter="mc", solver="hlld",
                                       ct="uct_hll", cfl=0.3)
    s = solver(st, "mc", "hlld")
    _, hist, out = s.run(20, 1e-4)
    V, U, Bs = s.download()
    assert oerr == 0 and out.err_bits == 0
    np.testing.assert_array_equal(U, Uo)
    np.testing.assert_array_equal(V, Vo)


def test_rmhd_mixed_error_bounded():
    st = ics.rmhd3d_turbulence(n=(24, 24, 24), seed=5, lorentz_max=3.0, sigma=0.3, p0=1.0)
    a = solver(st, "mc", "hlld")
    b = solver(st, "mc", "hlld", precision=api.MIXED)
    a.run(20, 1e-4)
    b.run(20, 1e-4)
    _, Ua, _ = a.download()
    _, Ub, _ = b.download()
    for nv in range(8):
        l1 = np.abs(Ub[nv] - Ua[nv]).mean() / np.abs(Ua[nv]).mean()
        assert l1 <= 1e-4, (nv, l1)


def test_rmhd_192_config_runs_100_steps_without_errors():
    st = ics.rmhd3d_turbulence(n=(192, 192, 192), seed=1)
    s = solver(st, "mc", "hlld")
    _, _, out = s.run(100, 1e-4, history=False)
    assert out.err_bits == 0
    _, _, Bs = s.download()
    div = ((np.roll(Bs[0], -1, 2) - Bs[0]) + (np.roll(Bs[1], -1, 1) - Bs[1])
           + (np.roll(Bs[2], -1, 0) - Bs[2]))
    assert np.abs(div).max() / max(np.abs(b).max() for b in Bs) <= 1e-12

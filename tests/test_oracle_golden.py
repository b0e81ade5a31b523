"""Pin the C oracle against the reference gPLUTO serial build.

The fixtures in tests/golden/ were produced by tests/golden/make_golden.py,
which compiles the reference sources (Config/linux.g++.defs flags) and runs
them on seeded initial conditions.  The oracle must reproduce every final
Vc/Uc/Vs array and the dt sequence bit for bit.
"""
import numpy as np
import pytest

import golden_util as gu
import oracle as orc


@pytest.mark.parametrize("name", gu.names())
def test_oracle_matches_reference_bitwise(name):
    g = gu.Golden(name)
    o = orc.Oracle(g.ic, limiter=g.limiter, solver=g.solver, ct=g.ct,
                   cfl=g.cfl, cfl_max_var=g.cfl_max_var)
    hist, err = o.run(g.nsteps, g.first_dt)
    V, U, Bs = o.state()
    assert err & (1 << 15) == 0, f"oracle raised ERR_QUIT ({err:#x})"
    np.testing.assert_array_equal(hist, g.dt)
    np.testing.assert_array_equal(V, g.V)
    np.testing.assert_array_equal(U, g.U)
    for a, b in zip(Bs, g.Bs):
        np.testing.assert_array_equal(a, b)


def test_oracle_divb_roundoff():
    g = gu.Golden("mhd3d_mc_hlld_ucthlld")
    o = orc.Oracle(g.ic, limiter=g.limiter, solver=g.solver, ct=g.ct)
    o.run(g.nsteps, g.first_dt)
    _, _, Bs = o.state()
    nx, ny, nz = g.shape
    div = ((np.roll(Bs[0], -1, 2) - Bs[0]) * nx + (np.roll(Bs[1], -1, 1) - Bs[1]) * ny
           + (np.roll(Bs[2], -1, 0) - Bs[2]) * nz)
    bmax = max(np.abs(b).max() for b in Bs)
    assert np.abs(div).max() / (bmax * max(nx, ny, nz)) < 1e-12

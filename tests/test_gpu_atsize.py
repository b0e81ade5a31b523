"""Parity at the full sizes of the single-grid workloads, 100 steps each,
against the reference's own serial build (fixtures written by
tests/golden/make_atsize.py; see tests/atsize_util.py for the summary).

* 2-D ideal MHD 256^2 (PLM-MC, HLLD, UCT_HLLD, RK2, CFL 0.4) and the
  3-D MHD blast at 256^3 (the bench workload): every plane of every
  primitive, conserved and face array bit-identical, and the dt sequence too.
* 3-D relativistic MHD at 192^3 (PLM-MC, HLLD, UCT_HLL, CFL 0.3): relative
  L-infinity per variable on the sampled cells and the centre line within
  1e-11, the per-plane sums within 1e-11 of the plane's absolute sum, the dt
  sequence within 1e-11 (the GPU's acos/cos/sin are correctly rounded where
  glibc's occasionally are not, so bit identity is not expected there).
"""
import os

import numpy as np
import pytest

import atsize_util as au
from gpluto_dev_b200 import api, ics

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "atsize")
RTOL = 1e-11

CASES = {
    "mhd2d_256": (ics.mhd2d_turbulence, dict(n=(256, 256), seed=0),
                  dict(physics=api.MHD, limiter="mc", riemann="hlld", ct_emf="uct_hlld",
                       cfl=0.4)),
    "mhd3d_blast_256": (ics.mhd3d_blast, dict(n=(256, 256, 256), seed=1),
                        dict(physics=api.MHD, limiter="mc", riemann="hlld", ct_emf="uct_hlld",
                             cfl=0.4)),
    "rmhd3d_192": (ics.rmhd3d_turbulence, dict(n=(192, 192, 192), seed=1),
                   dict(physics=api.RMHD, limiter="mc", riemann="hlld", ct_emf="uct_hll",
                        cfl=0.3)),
}


def _run(name):
    path = os.path.join(FIX, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"no reference fixture {name}")
    ref = dict(np.load(path))
    gen, kw, sch = CASES[name]
    st = gen(**kw)
    s = api.Solver.from_state(st, api.Scheme(gamma=st.gamma, cfl_max_var=1.1, **sch))
    dt_after, hist, out = s.run(int(ref["nsteps"]), 1e-4)
    V, U, Bs = s.download()
    s.close()
    got = au.summarize(V, U, Bs, st.ndim)
    return ref, got, np.append(hist, dt_after), out, V.shape[0]


@pytest.mark.parametrize("name", ["mhd2d_256", "mhd3d_blast_256"])
def test_mhd_100_steps_at_size_bitwise(name):
    ref, got, hist, out, nvar = _run(name)
    assert out.err_bits & api.ERR_QUIT == 0
    np.testing.assert_array_equal(hist, ref["dt"])
    cmp = au.compare(got, ref, nvar)
    bad = [n for n, same in zip(cmp["names"], cmp["bitwise"]) if not same]
    assert not bad, (bad, max(cmp["rel_linf"]))


def test_rmhd_100_steps_at_size():
    ref, got, hist, out, nvar = _run("rmhd3d_192")
    assert out.err_bits & api.ERR_QUIT == 0
    np.testing.assert_allclose(hist, ref["dt"], rtol=RTOL, atol=0)
    cmp = au.compare(got, ref, nvar)
    worst = max(cmp["rel_linf"])
    assert worst <= RTOL, dict(zip(cmp["names"], cmp["rel_linf"]))
    assert max(cmp["plane_sum_rel"]) <= RTOL

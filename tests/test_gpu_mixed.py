"""Mixed form (FP32 reconstruction, limiter, Riemann fluxes and UCT EMFs;
FP64 accumulation, CT update and con2prim) against the FP64 form.

The FP64 form is bit-identical to the oracle and the reference, so it is
the FP64 oracle here.  Both forms take the FP64 run's dt sequence, so the
difference is the arithmetic alone.  Bounds: relative L1 error
sum|mixed - fp64| / sum|fp64| <= 1e-5 per conserved variable, and the
mixed form's div(B) <= 1e-12 relative to max|B|/dx (constrained transport
keeps it at round-off in either form).
"""
import numpy as np
import pytest

from gpluto_dev_b200 import api, ics

pytestmark = pytest.mark.gpu


def divb_rel(Bs, shape, ndim):
    nx, ny, nz = shape
    dx = [1.0 / nx, 1.0 / ny, 1.0 / max(nz, 1)]
    axes = {0: 2, 1: 1, 2: 0}
    div = sum((np.roll(Bs[d], -1, axis=axes[d]) - Bs[d]) / dx[d] for d in range(ndim))
    bmax = max(np.abs(b).max() for b in Bs)
    return np.abs(div).max() / (bmax / min(dx[:ndim]))


def run_pair(st, nsteps, dt0):
    sch = api.Scheme(physics=api.MHD, gamma=st.gamma)
    a = api.Solver.from_state(st, sch)
    _, hist, oa = a.run(nsteps, dt0)
    b = api.Solver.from_state(st, api.Scheme(physics=api.MHD, gamma=st.gamma,
                                             precision=api.MIXED))
    for dt in hist:
        ob = b.AdvanceStep(float(dt))
    Va, Ua, Ba = a.download()
    Vb, Ub, Bb = b.download()
    a.close()
    b.close()
    return (Ua, Ba), (Ub, Bb), oa, ob


@pytest.mark.parametrize("case", ["mhd2d_256_100steps", "mhd3d_blast_64_50steps"])
def test_mixed_l1_error_and_divb(case):
    if case.startswith("mhd2d"):
        st, n = ics.mhd2d_turbulence(n=(256, 256), seed=0), 100
    else:
        st, n = ics.mhd3d_blast(n=(64, 64, 64), seed=1), 50
    (Ua, Ba), (Ub, Bb), oa, ob = run_pair(st, n, 1e-4)
    assert ob.err_bits & api.ERR_QUIT == 0
    for nv in range(8):
        den = np.abs(Ua[nv]).sum()
        if den == 0.0:            # a component that stays zero (2-D: v_z, B_z)
            assert np.abs(Ub[nv]).sum() == 0.0, (case, nv)
            continue
        l1 = np.abs(Ub[nv] - Ua[nv]).sum() / den
        assert l1 <= 1e-5, (case, nv, l1)
    assert divb_rel(Bb, st.shape, st.ndim) <= 1e-12
    assert divb_rel(Ba, st.shape, st.ndim) <= 1e-12


MIXED_SCHEMES = [
    # (generator, kwargs, limiter, solver, ct, Solver keyword arguments, rk, nsteps)
    (ics.hd_turbulence, dict(n=(96, 80), seed=121), "mc", "hllc", "uct_hll", dict(), 2, 40),
    (ics.mhd2d_turbulence, dict(n=(96, 96), seed=122), "ppm", "hlld", "uct_hlld", dict(), 2, 40),
    (ics.mhd2d_turbulence, dict(n=(80, 64), seed=123), "mc", "hlld", "uct_hlld",
     dict(outflow=0b0011, reflect=0b1100), 3, 30),
    (ics.mhd3d_turbulence, dict(n=(40, 36, 32), seed=124), "vl", "hll", "uct_hll",
     dict(eqtsym=0b110000), 3, 15),
    (ics.mhd2d_turbulence, dict(n=(80, 72), seed=125), "vanalbada", "hlld", "uct_hlld",
     dict(), 2, 30),
    (ics.mhd3d_turbulence, dict(n=(36, 32, 28), seed=126), "ospre", "hlld", "uct_hlld",
     dict(), 2, 12),
    (ics.mhd3d_turbulence, dict(n=(36, 32, 28), seed=127), "mc", "hllc", "uct_hll",
     dict(), 2, 12),
    (ics.mhd3d_turbulence, dict(n=(36, 32, 28), seed=128), "mc", "hlld", "ct_contact",
     dict(), 2, 12),
]


@pytest.mark.parametrize("case", range(len(MIXED_SCHEMES)))
def test_mixed_l1_error_other_schemes(case):
    """The ≤ 1e-5 relative L1 bound of the mixed form for HD, PPM, RK3,
    non-periodic sides and the van Albada and OSPRE limiters, on the FP64
    run's dt sequence."""
    gen, kw, lim, rs, ct, bc, rk, n = MIXED_SCHEMES[case]
    st = gen(**kw)

    def scheme(prec):
        return api.Scheme(physics=st.physics, limiter=lim, riemann=rs, ct_emf=ct,
                          gamma=st.gamma, precision=prec, rk=rk)
    a = api.Solver.from_state(st, scheme(api.FP64), **bc)
    _, hist, oa = a.run(n, 1e-4)
    b = api.Solver.from_state(st, scheme(api.MIXED), **bc)
    for dt in hist:
        ob = b.AdvanceStep(float(dt))
    Ua, Ub = a.download()[1], b.download()[1]
    a.close()
    b.close()
    assert oa.err_bits & api.ERR_QUIT == 0 and ob.err_bits & api.ERR_QUIT == 0
    for nv in range(Ua.shape[0]):
        den = np.abs(Ua[nv]).sum()
        if den == 0.0:
            continue
        assert np.abs(Ub[nv] - Ua[nv]).sum() / den <= 1e-5, (case, nv)

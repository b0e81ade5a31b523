"""gp_advance_step_noalloc: the RK2 step for callers that cannot allocate.

Callers whose device memory belongs to another allocator, or whose step loop
must not allocate, cannot call cudaMalloc.  The entry point keeps every
intermediate in a static device array and updates the caller's own device
arrays in place.  Checked here against gp_advance_step on two consecutive
steps, with the exact equality the FP64 parity tests use, and for the size
limit.  This file is collected last so that a failure here cannot hide the
other tests.
"""
import ctypes

import numpy as np
import pytest

from gpluto_dev_b200 import api, ics

pytestmark = pytest.mark.gpu


def _entry():
    L = api.lib()
    f = L.gp_advance_step_noalloc
    P, D = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.POINTER(api.GpGridDesc), ctypes.POINTER(api.GpScheme),
                  P, P, P, P, P, ctypes.c_double, P, ctypes.POINTER(api.GpStepOut)]
    f.restype = ctypes.c_int
    return f


def _noalloc_run(st, scheme, dts, solver=None):
    import torch
    ref = solver or api.Solver.from_state(st, scheme)   # initial U from the start-up map
    V0, U0, B0 = ref.download()
    dev = torch.device("cuda")
    U = torch.from_numpy(U0).to(dev).contiguous()
    V = torch.from_numpy(V0).to(dev).contiguous()
    B = [torch.from_numpy(b).to(dev).contiguous() for b in B0]
    ptr = [b.data_ptr() for b in B] + [None] * (3 - len(B))
    f = _entry()
    outs = []
    for dt in dts:
        o = api.GpStepOut()
        rc = f(ctypes.byref(ref._gdesc), ctypes.byref(ref._sdesc), U.data_ptr(), V.data_ptr(),
               ptr[0], ptr[1], ptr[2], dt, None, ctypes.byref(o))
        assert rc == api.GP_OK, rc
        outs.append((o.err_bits, o.invDt_hyp, o.dt_next))
    torch.cuda.synchronize()
    return U.cpu().numpy(), V.cpu().numpy(), [b.cpu().numpy() for b in B], outs


def _case(case):
    if case == "mhd3d":
        st = ics.mhd3d_turbulence(n=(20, 18, 16), seed=61)
        return st, api.Scheme(physics=api.MHD, gamma=st.gamma)
    if case == "mhd2d":
        st = ics.mhd2d_turbulence(n=(128, 96), seed=62)
        return st, api.Scheme(physics=api.MHD, gamma=st.gamma)
    if case == "hd3d":
        st = ics.hd_turbulence(n=(24, 20, 16), seed=63)
        return st, api.Scheme(physics=api.HD, riemann="hllc", gamma=st.gamma)
    if case == "mhd3d_mixed":
        # the mixed form carves float face data and EMFs out of the same array
        st = ics.mhd3d_turbulence(n=(24, 20, 16), seed=65)
        return st, api.Scheme(physics=api.MHD, precision=api.MIXED, gamma=st.gamma)
    if case == "rmhd3d":
        st = ics.rmhd3d_turbulence(n=(16, 16, 16), seed=66, lorentz_max=3.0)
        return st, api.Scheme(physics=api.RMHD, limiter="mc", riemann="hlld", ct_emf="uct_hll",
                              gamma=st.gamma, cfl=0.3)
    # PPM with HLL and UCT_HLL at the size limit (128 x 128 = 16384 cells)
    st = ics.mhd2d_turbulence(n=(128, 128), seed=67)
    return st, api.Scheme(physics=api.MHD, limiter="ppm", riemann="hll", ct_emf="uct_hll",
                          gamma=st.gamma)


@pytest.mark.parametrize("case", ["mhd3d", "mhd2d", "hd3d", "mhd3d_mixed", "rmhd3d",
                                  "mhd2d_ppm_limit"])
def test_noalloc_matches_advance_step_twice(case):
    st, scheme = _case(case)
    # two consecutive steps through the regular entry point
    ref = api.Solver.from_state(st, scheme)
    dts, outs = [1e-3 if case != "rmhd3d" else 1e-4], []
    for _ in range(2):
        o = ref.AdvanceStep(dts[-1])
        outs.append((o.err_bits, o.invDt_hyp, o.dt_next))
        dts.append(o.dt_next)
    Vr, Ur, Br = ref.download()
    # the same two steps through the no-allocation entry point: the same
    # kernels on the same inputs, so the same bits in either form
    U, V, B, outs2 = _noalloc_run(st, scheme, dts[:2])
    np.testing.assert_array_equal(U, Ur)
    np.testing.assert_array_equal(V, Vr)
    for a, b in zip(B, Br):
        np.testing.assert_array_equal(a, b)
    assert outs2 == outs


def test_noalloc_takes_the_callers_cell_widths():
    """A caller that passes the grid's cell widths (Grid::dx) and no extent
    gets the same step as one that passes the extent."""
    st, scheme = _case("mhd2d")
    U, V, B, outs = _noalloc_run(st, scheme, [1e-3])
    ref = api.Solver.from_state(st, scheme)
    g = api.GpGridDesc()
    ctypes.memmove(ctypes.byref(g), ctypes.byref(ref._gdesc), ctypes.sizeof(g))
    widths = []
    for d in range(2):
        n = g.nint[d]
        w = np.full(n + 2 * max(g.nghost, 0), (g.xend[d] - g.xbeg[d]) / n)
        widths.append(w)
        g.dx[d] = w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        g.xbeg[d], g.xend[d] = 0.0, 0.0
    ref._gdesc = g
    U2, V2, B2, outs2 = _noalloc_run(st, scheme, [1e-3], solver=ref)
    np.testing.assert_array_equal(U2, U)
    assert outs2 == outs


def test_noalloc_refuses_what_gp_create_refuses():
    """MHD HLL with UCT_HLLD face data is refused (the reference refuses it,
    Src/MHD/hll.cpp:73-77), as are non-periodic sides and RK3."""
    st, _ = _case("mhd2d")
    for kw, side in ((dict(riemann="hll", ct_emf="uct_hlld"), None),
                     (dict(), "outflow"), (dict(rk=3), None)):
        scheme = api.Scheme(physics=api.MHD, gamma=st.gamma, **kw)
        g = api.GpGridDesc()
        g.ndim = 2
        g.nint[0], g.nint[1], g.nint[2] = 128, 96, 1
        for d in range(3):
            g.xbeg[d], g.xend[d] = 0.0, 1.0
        if side:
            g.lbound[0] = g.rbound[0] = api.BC_OUTFLOW
        sc = scheme.to_c()
        o = api.GpStepOut()
        rc = _entry()(ctypes.byref(g), ctypes.byref(sc), 1, 1, 1, 1, None, 1e-3, None,
                      ctypes.byref(o))
        assert rc == api.GP_ERR_UNSUPPORTED, (kw, side, rc)


def test_noalloc_rejects_grids_above_the_limit():
    st = ics.mhd2d_turbulence(n=(256, 128), seed=64)    # 32768 > 16384 cells
    scheme = api.Scheme(physics=api.MHD, gamma=st.gamma)
    g = api.GpGridDesc()
    g.ndim = 2
    g.nint[0], g.nint[1], g.nint[2] = 256, 128, 1
    for d in range(3):
        g.xbeg[d], g.xend[d] = 0.0, 1.0
    s = scheme.to_c()
    o = api.GpStepOut()
    rc = _entry()(ctypes.byref(g), ctypes.byref(s), 1, 1, 1, 1, None, 1e-3, None,
                  ctypes.byref(o))
    assert rc == api.GP_ERR_INVALID

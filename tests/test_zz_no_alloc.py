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


def _noalloc_run(st, scheme, dts):
    import torch
    ref = api.Solver.from_state(st, scheme)        # initial U from the start-up map
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


@pytest.mark.parametrize("case", ["mhd3d", "mhd2d", "hd3d"])
def test_noalloc_matches_advance_step_twice(case):
    if case == "mhd3d":
        st = ics.mhd3d_turbulence(n=(20, 18, 16), seed=61)
        scheme = api.Scheme(physics=api.MHD, gamma=st.gamma)
    elif case == "mhd2d":
        st = ics.mhd2d_turbulence(n=(128, 96), seed=62)
        scheme = api.Scheme(physics=api.MHD, gamma=st.gamma)
    else:
        st = ics.hd_turbulence(n=(24, 20, 16), seed=63)
        scheme = api.Scheme(physics=api.HD, riemann="hllc", gamma=st.gamma)
    # two consecutive steps through the regular entry point
    ref = api.Solver.from_state(st, scheme)
    dts, outs = [1e-3], []
    for _ in range(2):
        o = ref.AdvanceStep(dts[-1])
        outs.append((o.err_bits, o.invDt_hyp, o.dt_next))
        dts.append(o.dt_next)
    Vr, Ur, Br = ref.download()
    # the same two steps through the no-allocation entry point
    U, V, B, outs2 = _noalloc_run(st, scheme, dts[:2])
    np.testing.assert_array_equal(U, Ur)
    np.testing.assert_array_equal(V, Vr)
    for a, b in zip(B, Br):
        np.testing.assert_array_equal(a, b)
    assert outs2 == outs


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

"""Parity of the sm_100a Godunov step with the reference and the oracle.

The FP64 form must reproduce the reference serial build bit for bit (the
kernels keep the reference's operation order and are compiled with
-fmad=false); where a bound is written below it is the acceptance bound of
the plain form (relative L-infinity <= 1e-11 per variable).
"""
import numpy as np
import pytest

import golden_util as gu
import oracle as orc
import userdef_util as ud
from gpluto_dev_b200 import api, ics

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-11


def rel_linf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make_solver(st, limiter, solver, ct, cfl=0.4, cfl_max_var=1.1, precision=api.FP64,
                outflow=0, reflect=0, eqtsym=0, rk=2, userdef=0):
    """USERDEF sides get the inflow fill of the parity cases."""
    sch = api.Scheme(physics=st.physics, limiter=limiter, riemann=solver, ct_emf=ct,
                     precision=precision, gamma=st.gamma, cfl=cfl, cfl_max_var=cfl_max_var,
                     rk=rk)
    return api.Solver.from_state(st, sch, outflow=outflow, reflect=reflect, eqtsym=eqtsym,
                                 userdef=userdef,
                                 userdef_fill=ud.inflow_fill if userdef else None)


@pytest.mark.parametrize("name", [n for n in gu.names() if not n.startswith("rmhd")])
def test_gpu_matches_reference_fixture_bitwise(name):
    g = gu.Golden(name)
    s = make_solver(g.ic, g.limiter, g.solver, g.ct, g.cfl, g.cfl_max_var, **g.bc, rk=g.rk)
    dt_after, hist, out = s.run(g.nsteps, g.first_dt)
    V, U, Bs = s.download()
    assert out.err_bits & api.ERR_QUIT == 0
    np.testing.assert_array_equal(hist, g.dt[:-1])
    assert dt_after == g.dt[-1]
    np.testing.assert_array_equal(V, g.V)
    np.testing.assert_array_equal(U, g.U)
    for a, b in zip(Bs, g.Bs):
        np.testing.assert_array_equal(a, b)


CASES = [
    # (generator, kwargs, limiter, solver, ct, nsteps)
    (ics.mhd2d_turbulence, dict(n=(64, 48), seed=21), "mc", "hlld", "uct_hlld", 30),
    (ics.mhd2d_turbulence, dict(n=(33, 17), seed=22), "vl", "hlld", "uct_hll", 20),
    (ics.mhd3d_turbulence, dict(n=(20, 18, 16), seed=23), "mc", "hlld", "uct_hlld", 10),
    (ics.mhd3d_blast, dict(n=(24, 24, 24), seed=24, radius=0.2), "mc", "hlld", "uct_hlld", 10),
    (ics.mhd3d_turbulence, dict(n=(16, 20, 12), seed=25), "minmod", "hll", "uct_hll", 8),
    (ics.hd_turbulence, dict(n=(40, 36), seed=26), "mc", "hllc", "uct_hll", 20),
    (ics.hd_turbulence, dict(n=(16, 12, 20), seed=27), "vl", "hll", "uct_hll", 10),
    # PPM: rows of 33 and 65 cells (a last chunk of 1 lane), a row shorter
    # than a warp, a 5-cell direction
    (ics.mhd2d_turbulence, dict(n=(33, 17), seed=28), "ppm", "hlld", "uct_hlld", 15),
    (ics.mhd3d_turbulence, dict(n=(20, 18, 16), seed=29), "ppm", "hlld", "uct_hlld", 8),
    (ics.hd_turbulence, dict(n=(65, 5), seed=30), "ppm", "hllc", "uct_hll", 12),
    (ics.mhd2d_turbulence, dict(n=(6, 40), seed=31), "ppm", "hll", "uct_hll", 10),
    # the other PLM limiters (flat, van Albada, OSPRE, UMIST) on odd sizes
    (ics.mhd3d_turbulence, dict(n=(13, 11, 9), seed=131), "vanalbada", "hlld", "uct_hlld", 6),
    (ics.mhd2d_turbulence, dict(n=(35, 19), seed=132), "ospre", "hlld", "uct_hll", 10),
    (ics.hd_turbulence, dict(n=(33, 7), seed=133), "umist", "hllc", "uct_hll", 12),
    (ics.mhd2d_turbulence, dict(n=(17, 23), seed=134), "flat", "hll", "uct_hll", 10),
    # the Lax-Friedrichs (tvdlf) solver
    (ics.mhd2d_turbulence, dict(n=(29, 21), seed=171), "mc", "tvdlf", "uct_hll", 10),
    (ics.mhd3d_blast, dict(n=(13, 12, 11), seed=172, radius=0.25), "vl", "tvdlf", "uct_hll", 6),
    (ics.hd_turbulence, dict(n=(27, 13, 11), seed=173), "ppm", "tvdlf", "uct_hll", 8),
    # CT_EMF_AVERAGE ARITHMETIC
    (ics.mhd3d_turbulence, dict(n=(13, 11, 9), seed=191), "mc", "hlld", "arithmetic", 6),
    (ics.mhd2d_turbulence, dict(n=(27, 19), seed=192), "vl", "tvdlf", "arithmetic", 10),
    # CT_EMF_AVERAGE CT_CONTACT on odd sizes
    (ics.mhd3d_turbulence, dict(n=(13, 11, 9), seed=206), "vl", "hlld", "ct_contact", 6),
    (ics.mhd2d_turbulence, dict(n=(29, 17), seed=207), "mc", "hllc", "ct_contact", 10),
    (ics.mhd3d_blast, dict(n=(15, 13, 11), seed=208, radius=0.25), "ppm", "tvdlf",
     "ct_contact", 6),
    # HLLC for MHD (UCT_HLL and ARITHMETIC face data)
    (ics.mhd3d_turbulence, dict(n=(17, 13, 11), seed=195), "mc", "hllc", "uct_hll", 6),
    (ics.mhd2d_turbulence, dict(n=(31, 23), seed=196), "ppm", "hllc", "arithmetic", 10),
    (ics.mhd3d_blast, dict(n=(15, 14, 13), seed=197, radius=0.25), "minmod", "hllc",
     "uct_hll", 6),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_gpu_matches_oracle_bitwise(case):
    gen, kw, lim, rs, ct, nsteps = CASES[case]
    st = gen(**kw)
    o = orc.Oracle(st, limiter=lim, solver=rs, ct=ct)
    ohist, oerr = o.run(nsteps, 1e-4)
    Vo, Uo, Bo = o.state()
    s = make_solver(st, lim, rs, ct)
    dt_after, hist, out = s.run(nsteps, 1e-4)
    V, U, Bs = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, ohist[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)
    for a, b in zip(Bs, Bo):
        np.testing.assert_array_equal(a, b)


OUTFLOW_CASES = [
    # (generator, kwargs, limiter, solver, outflow mask, nsteps): rows of 33
    # and 65 cells (the extra boundary face starts a new chunk), a row
    # shorter than a warp, both PLM and PPM
    (ics.hd_turbulence, dict(n=(32, 20), seed=51), "mc", "hllc", 0b0011, 15),
    (ics.hd_turbulence, dict(n=(65, 7), seed=52), "ppm", "hllc", 0b1111, 12),
    (ics.hd_turbulence, dict(n=(6, 33), seed=53), "vl", "hll", 0b1100, 12),
    (ics.hd_turbulence, dict(n=(13, 11, 9), seed=54), "ppm", "hll", 0b111111, 8),
    (ics.hd_turbulence, dict(n=(31, 10, 12), seed=55), "mc", "hllc", 0b110000, 8),
]


@pytest.mark.parametrize("case", range(len(OUTFLOW_CASES)))
def test_gpu_outflow_matches_oracle_bitwise(case):
    gen, kw, lim, rs, ob, nsteps = OUTFLOW_CASES[case]
    st = gen(**kw)
    o = orc.Oracle(st, limiter=lim, solver=rs, ct="uct_hll", outflow=ob)
    ohist, oerr = o.run(nsteps, 1e-4)
    Vo, Uo, _ = o.state()
    s = make_solver(st, lim, rs, "uct_hll", outflow=ob)
    dt_after, hist, out = s.run(nsteps, 1e-4)
    V, U, _ = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, ohist[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)


CT_OUTFLOW_CASES = [
    # (generator, kwargs, limiter, solver, ct, outflow mask, nsteps)
    (ics.mhd2d_turbulence, dict(n=(33, 20), seed=57), "mc", "hlld", "uct_hlld", 0b0011, 12),
    (ics.mhd2d_turbulence, dict(n=(24, 30), seed=58), "ppm", "hlld", "uct_hlld", 0b1111, 10),
    (ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=59), "mc", "hlld", "uct_hlld", 0b111111, 6),
    (ics.mhd3d_turbulence, dict(n=(16, 12, 10), seed=60), "vl", "hll", "uct_hll", 0b110000, 6),
    (ics.mhd3d_blast, dict(n=(20, 18, 16), seed=61, radius=0.2), "mc", "hlld", "uct_hlld",
     0b001100, 6),
]


@pytest.mark.parametrize("case", range(len(CT_OUTFLOW_CASES)))
def test_gpu_ct_outflow_matches_oracle_bitwise(case):
    """Outflow with constrained transport: padded ghost zones filled before
    every stage (copies, div-free normal faces, re-averaged ghost B)."""
    gen, kw, lim, rs, ct, ob, nsteps = CT_OUTFLOW_CASES[case]
    st = gen(**kw)
    o = orc.Oracle(st, limiter=lim, solver=rs, ct=ct, outflow=ob)
    ohist, oerr = o.run(nsteps, 1e-4)
    Vo, Uo, Bo = o.state()
    s = make_solver(st, lim, rs, ct, outflow=ob)
    dt_after, hist, out = s.run(nsteps, 1e-4)
    V, U, Bs = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, ohist[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)
    for a, b in zip(Bs, Bo):
        np.testing.assert_array_equal(a, b)


MIRROR_CASES = [
    # (generator, kwargs, limiter, solver, ct, dict of side masks, nsteps): odd
    # sizes, mirrored sides alone, with outflow, all sides, HD PPM
    (ics.mhd2d_turbulence, dict(n=(33, 21), seed=81), "mc", "hlld", "uct_hlld",
     dict(reflect=0b0011), 10),
    (ics.mhd2d_turbulence, dict(n=(20, 27), seed=82), "ppm", "hlld", "uct_hlld",
     dict(reflect=0b0001, outflow=0b0010, eqtsym=0b1100), 10),
    (ics.mhd3d_turbulence, dict(n=(11, 10, 9), seed=83), "mc", "hlld", "uct_hlld",
     dict(reflect=0b110011, eqtsym=0b001100), 6),
    (ics.mhd3d_blast, dict(n=(16, 14, 12), seed=84, radius=0.25), "vl", "hll", "uct_hll",
     dict(reflect=0b111111), 6),
    (ics.hd_turbulence, dict(n=(13, 11, 9), seed=85), "ppm", "hllc", "uct_hll",
     dict(reflect=0b110000, outflow=0b000011), 8),
    (ics.hd_turbulence, dict(n=(31, 17), seed=86), "mc", "hll", "uct_hll",
     dict(reflect=0b1111), 12),
    # USERDEF sides (the inflow fill): alone, with mirrored and outflow sides,
    # every side of a grid, MP5 and PPM widths
    (ics.mhd3d_turbulence, dict(n=(11, 10, 9), seed=87), "mc", "hlld", "uct_hlld",
     dict(userdef=0b110011), 6),
    (ics.mhd3d_blast, dict(n=(12, 10, 9), seed=88, radius=0.25), "mp5", "hll", "uct_hll",
     dict(userdef=0b001100, reflect=0b000011), 5),
    (ics.hd_turbulence, dict(n=(21, 17), seed=89), "ppm", "hllc", "uct_hll",
     dict(outflow=0b0001, userdef=0b0010, reflect=0b1100), 10),
    (ics.mhd2d_turbulence, dict(n=(25, 19), seed=90), "vl", "hlld", "uct_hlld",
     dict(userdef=0b1111), 10),
]


@pytest.mark.parametrize("case", range(len(MIRROR_CASES)))
def test_gpu_mirrored_sides_match_oracle_bitwise(case):
    """Reflective / eqtsymmetric sides (mixed with outflow and periodic ones):
    padded ghost zones filled before every stage by mirror copies with the
    reference's signs, then the ghost cells' B averaged from their faces.
    USERDEF sides: the caller's fill, then the div B = 0 normal faces and the
    ghost averages."""
    gen, kw, lim, rs, ct, bc, nsteps = MIRROR_CASES[case]
    st = gen(**kw)
    kwo = dict(limiter=lim, solver=rs, **bc)
    if st.physics != ics.PHYS_HD:
        kwo["ct"] = ct
    o = orc.Oracle(st, **kwo)
    ohist, oerr = o.run(nsteps, 1e-4)
    Vo, Uo, Bo = o.state()
    s = make_solver(st, lim, rs, ct, **bc)
    dt_after, hist, out = s.run(nsteps, 1e-4)
    V, U, Bs = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, ohist[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)
    for a, b in zip(Bs, Bo):
        np.testing.assert_array_equal(a, b)


RK3_CASES = [
    # (generator, kwargs, limiter, solver, ct, side masks, nsteps): TIME_STEPPING RK3
    (ics.mhd3d_blast, dict(n=(17, 15, 13), seed=96, radius=0.2), "mc", "hlld", "uct_hlld",
     dict(), 6),
    (ics.mhd2d_turbulence, dict(n=(29, 23), seed=97), "ppm", "hlld", "uct_hlld",
     dict(reflect=0b0011, outflow=0b1100), 8),
    (ics.hd_turbulence, dict(n=(19, 13, 11), seed=98), "vl", "hllc", "uct_hll", dict(), 8),
]


@pytest.mark.parametrize("case", range(len(RK3_CASES)))
def test_gpu_rk3_matches_oracle_bitwise(case):
    gen, kw, lim, rs, ct, bc, nsteps = RK3_CASES[case]
    st = gen(**kw)
    kwo = dict(limiter=lim, solver=rs, rk=3, **bc)
    if st.physics != ics.PHYS_HD:
        kwo["ct"] = ct
    o = orc.Oracle(st, **kwo)
    ohist, oerr = o.run(nsteps, 1e-4)
    Vo, Uo, Bo = o.state()
    s = make_solver(st, lim, rs, ct, rk=3, **bc)
    dt_after, hist, out = s.run(nsteps, 1e-4)
    V, U, Bs = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, ohist[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)
    for a, b in zip(Bs, Bo):
        np.testing.assert_array_equal(a, b)


MP5_CASES = [
    # (generator, kwargs, solver, ct, side masks, rk, nsteps): rows of 33 and 65
    # cells (a last chunk of 1 and of 1 face), a row shorter than a warp, 3-D
    # marches, mirrored and outflow sides
    (ics.mhd2d_turbulence, dict(n=(33, 20), seed=111), "hlld", "uct_hlld", dict(), 2, 10),
    (ics.mhd2d_turbulence, dict(n=(65, 7), seed=112), "hll", "uct_hll",
     dict(reflect=0b0011, outflow=0b1100), 3, 8),
    (ics.mhd3d_turbulence, dict(n=(7, 12, 10), seed=113), "hlld", "uct_hlld",
     dict(eqtsym=0b110000), 2, 6),
    (ics.hd_turbulence, dict(n=(30, 9, 11), seed=114), "hllc", "uct_hll",
     dict(outflow=0b000011, reflect=0b001100), 3, 8),
]


@pytest.mark.parametrize("rec", ["mp5", "wenoz", "limo3", "weno3"])
@pytest.mark.parametrize("case", range(len(MP5_CASES)))
def test_gpu_mp5_matches_oracle_bitwise(case, rec):
    """The schemes of the MP5 driver: MP5 and WENO-Z (5-point), LimO3 and
    WENO3 (3-point, cell-width dependent)."""
    gen, kw, rs, ct, bc, rk, nsteps = MP5_CASES[case]
    st = gen(**kw)
    kwo = dict(limiter=rec, solver=rs, rk=rk, **bc)
    if st.physics != ics.PHYS_HD:
        kwo["ct"] = ct
    o = orc.Oracle(st, **kwo)
    ohist, oerr = o.run(nsteps, 1e-4)
    Vo, Uo, Bo = o.state()
    s = make_solver(st, rec, rs, ct, rk=rk, **bc)
    dt_after, hist, out = s.run(nsteps, 1e-4)
    V, U, Bs = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, ohist[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)
    for a, b in zip(Bs, Bo):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("rec", ["mp5", "wenoz", "limo3", "weno3"])
def test_mp5_mixed_form_stays_close_to_fp64(rec):
    st = ics.mhd3d_blast(n=(32, 32, 32), seed=115, radius=0.2)
    a = make_solver(st, rec, "hlld", "uct_hlld")
    _, hist, _ = a.run(20, 1e-4)
    b = make_solver(st, rec, "hlld", "uct_hlld", precision=api.MIXED)
    for dt in hist:
        b.AdvanceStep(float(dt))
    Ua, Ub = a.download()[1], b.download()[1]
    for nv in range(8):
        den = np.abs(Ua[nv]).sum()
        if den > 0:
            assert np.abs(Ub[nv] - Ua[nv]).sum() / den <= 1e-5, nv


def test_ct_outflow_reference_layout_needs_the_scheme_ghost_depth():
    st = ics.mhd2d_turbulence(n=(20, 16), seed=62)
    s = make_solver(st, "mc", "hlld", "uct_hlld", outflow=0b0011)
    cshape, fshapes = s.reference_shapes()          # nghost 2 = PLM ghost depth
    Vr = np.empty(cshape)
    Br = [np.empty(f) for f in fshapes]
    api._check(api.lib().gp_download_state(s._h, api.LAYOUT_REFERENCE, None, api._dp(Vr),
                                           api._dp(Br[0]), api._dp(Br[1]), None))
    V, _, Bs = s.download()
    np.testing.assert_array_equal(Vr[:, :, 2:-2, 2:-2], V)
    np.testing.assert_array_equal(Br[0][:, 2:-2, 2:-3], Bs[0])
    sp = api.Solver(2, (20, 16), api.Scheme(physics=api.MHD, limiter="ppm"), outflow=0b0011)
    with pytest.raises(api.GPError) as ei:                # PPM needs nghost 3
        sp.upload(st.V, None, st.Bs, layout=api.LAYOUT_REFERENCE)
    assert ei.value.code == -2


def test_outflow_reference_layout_ghosts_copy_the_boundary_cells():
    st = ics.hd_turbulence(n=(20, 12), seed=56)
    s = make_solver(st, "mc", "hllc", "uct_hll", outflow=0b0011)
    s.run(3, 1e-4)
    V, _, _ = s.download()
    cshape, _ = s.reference_shapes()
    Vr = np.empty(cshape)
    api._check(api.lib().gp_download_state(s._h, api.LAYOUT_REFERENCE, None, api._dp(Vr),
                                           None, None, None))
    g = s.nghost
    inner = Vr[:, :, g:-g, g:-g]
    np.testing.assert_array_equal(inner, V)
    for k in range(g):       # x: outflow copies of the boundary columns
        np.testing.assert_array_equal(Vr[:, :, g:-g, k], V[:, :, :, 0])
        np.testing.assert_array_equal(Vr[:, :, g:-g, -1 - k], V[:, :, :, -1])
    np.testing.assert_array_equal(Vr[:, :, :g, g:-g], V[:, :, -g:, :])   # y: periodic


def test_host_dt_path_equals_device_dt_path():
    st = ics.mhd2d_turbulence(n=(48, 40), seed=31)
    a = make_solver(st, "mc", "hlld", "uct_hlld")
    b = make_solver(st, "mc", "hlld", "uct_hlld")
    dt = 1e-4
    for _ in range(6):
        out = a.AdvanceStep(dt)
        dt = api.NextTimeStep(out.invDt_hyp, 0.4, 1.1, dt)
    dt_b, _, _ = b.run(6, 1e-4)
    assert dt == dt_b
    Va, Ua, Ba = a.download()
    Vb, Ub, Bb = b.download()
    np.testing.assert_array_equal(Ua, Ub)
    np.testing.assert_array_equal(Ba[0], Bb[0])


def test_deterministic_rerun():
    st = ics.mhd3d_blast(n=(32, 32, 32), seed=5)
    r = []
    for _ in range(2):
        s = make_solver(st, "mc", "hlld", "uct_hlld")
        s.run(5, 1e-4)
        r.append(s.download())
    for x, y in zip(r[0][:2], r[1][:2]):
        np.testing.assert_array_equal(x, y)


def test_reference_layout_round_trip():
    st = ics.mhd3d_turbulence(n=(12, 10, 8), seed=41)
    s = make_solver(st, "mc", "hlld", "uct_hlld")
    V0, U0, B0 = s.download()
    cshape, fshapes = s.reference_shapes()
    g = s.nghost
    Vr, Ur = np.zeros(cshape), np.zeros(cshape)
    Br = [np.zeros(f) for f in fshapes]
    api.lib().gp_download_state(s._h, api.LAYOUT_REFERENCE, api._dp(Ur), api._dp(Vr),
                                api._dp(Br[0]), api._dp(Br[1]), api._dp(Br[2]))
    nx, ny, nz = st.shape
    np.testing.assert_array_equal(Vr[:, g:g + nz, g:g + ny, g:g + nx], V0)
    # periodic ghosts: left ghost = right interior
    np.testing.assert_array_equal(Vr[:, g:g + nz, g:g + ny, 0], V0[:, :, :, nx - 2])
    t = make_solver(st, "mc", "hlld", "uct_hlld")
    t.upload(Vr, Ur, Br, layout=api.LAYOUT_REFERENCE)
    V1, U1, B1 = t.download()
    np.testing.assert_array_equal(V1, V0)
    np.testing.assert_array_equal(U1, U0)
    for a, b in zip(B0, B1):
        np.testing.assert_array_equal(a, b)


def test_divb_roundoff_3d_blast():
    st = ics.mhd3d_blast(n=(48, 48, 48), seed=7)
    s = make_solver(st, "mc", "hlld", "uct_hlld")
    s.run(20, 1e-4)
    _, _, Bs = s.download()
    nx, ny, nz = st.shape
    div = ((np.roll(Bs[0], -1, 2) - Bs[0]) * nx + (np.roll(Bs[1], -1, 1) - Bs[1]) * ny
           + (np.roll(Bs[2], -1, 0) - Bs[2]) * nz)
    bmax = max(np.abs(b).max() for b in Bs)
    assert np.abs(div).max() / (bmax * max(nx, ny, nz)) <= 1e-12


def test_conservation_periodic():
    st = ics.mhd3d_turbulence(n=(24, 24, 24), seed=8)
    s = make_solver(st, "mc", "hlld", "uct_hlld")
    _, U0, _ = s.download()
    s.run(10, 1e-4)
    _, U1, _ = s.download()
    for nv in (0, 1, 2, 3, 7):   # mass, momentum, total energy
        tot0, tot1 = U0[nv].sum(), U1[nv].sum()
        scale = np.abs(U0[nv]).sum()
        assert abs(tot1 - tot0) <= 1e-12 * scale


def test_full_size_2d_100_steps_matches_oracle():
    """Config-0 size (2-D 256^2 MHD, PLM-MC, HLLD, UCT_HLLD, RK2, CFL 0.4)."""
    st = ics.mhd2d_turbulence(n=(256, 256), seed=0)
    o = orc.Oracle(st, limiter="mc", solver="hlld", ct="uct_hlld", cfl=0.4)
    ohist, _ = o.run(100, 1e-4)
    Vo, Uo, Bo = o.state()
    s = make_solver(st, "mc", "hlld", "uct_hlld")
    s.run(100, 1e-4)
    V, U, Bs = s.download()
    for nv in range(8):
        assert rel_linf(U[nv], Uo[nv]) <= RTOL_FP64
    assert np.array_equal(U, Uo)


TINY_CASES = [
    # the smallest grids: 2-3 cells along a direction (stencils wrap more
    # than once), PLM needs 2, PPM/MP5 4
    (ics.mhd2d_turbulence, dict(n=(2, 3), seed=131), "mc", "hlld", "uct_hlld", dict(), 6),
    (ics.mhd3d_turbulence, dict(n=(3, 2, 2), seed=132), "vl", "hll", "uct_hll", dict(), 4),
    (ics.hd_turbulence, dict(n=(2, 2, 3), seed=133), "mc", "hllc", "uct_hll", dict(), 6),
    (ics.mhd2d_turbulence, dict(n=(4, 5), seed=134), "ppm", "hlld", "uct_hlld", dict(), 5),
    (ics.mhd2d_turbulence, dict(n=(5, 4), seed=135), "mp5", "hlld", "uct_hlld", dict(), 5),
    (ics.mhd2d_turbulence, dict(n=(4, 4), seed=136), "mc", "hlld", "uct_hlld",
     dict(outflow=0b0011, reflect=0b1100), 5),
]


@pytest.mark.parametrize("case", range(len(TINY_CASES)))
def test_gpu_tiny_grids_match_oracle_bitwise(case):
    gen, kw, lim, rs, ct, bc, nsteps = TINY_CASES[case]
    st = gen(**kw)
    kwo = dict(limiter=lim, solver=rs, **bc)
    if st.physics != ics.PHYS_HD:
        kwo["ct"] = ct
    o = orc.Oracle(st, **kwo)
    ohist, oerr = o.run(nsteps, 1e-4)
    Vo, Uo, Bo = o.state()
    s = make_solver(st, lim, rs, ct, **bc)
    dt_after, hist, out = s.run(nsteps, 1e-4)
    V, U, Bs = s.download()
    assert out.err_bits == oerr
    np.testing.assert_array_equal(hist, ohist[:-1])
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(U, Uo)
    for a, b in zip(Bs, Bo):
        np.testing.assert_array_equal(a, b)


def test_grids_beyond_the_cell_limit_are_refused_before_allocating():
    sch = api.Scheme(physics=api.MHD)
    with pytest.raises(api.GPError) as ei:          # 2048^3 > 2^31 cells
        api.Solver(3, (2048, 2048, 2048), sch)
    assert ei.value.code == -2
    with pytest.raises(api.GPError) as ei:          # PPM below 4 cells
        api.Solver(2, (3, 8), api.Scheme(physics=api.MHD, limiter="ppm"))
    assert ei.value.code == api.GP_ERR_INVALID


def test_gpu_userdef_side_needs_a_fill():
    st = ics.mhd2d_turbulence(n=(16, 12), seed=91)
    sch = api.Scheme(physics=api.MHD, gamma=st.gamma)
    s = api.Solver.from_state(st, sch, userdef=0b0011)
    with pytest.raises(api.GPError) as ei:
        s.run(1, 1e-4)
    assert ei.value.code == api.GP_ERR_INVALID

    def bad_fill(side):
        raise RuntimeError("fill failed")

    s = api.Solver.from_state(st, sch, userdef=0b0011, userdef_fill=bad_fill)
    with pytest.raises(api.GPError) as ei:
        s.run(1, 1e-4)
    assert ei.value.code == api.GP_ERR_INVALID


def test_gpu_userdef_fill_sees_the_reference_ghost_box():
    """The box handed to the fill: the reference's ghost zone along the
    side's direction, the whole array across it; stages 1 and 2 per step."""
    st = ics.mhd3d_turbulence(n=(10, 9, 8), seed=92)
    seen = []

    def fill(side):
        seen.append((side.side, side.stage, side.beg, side.end, side.dom_beg, side.dims))
        ud.inflow_fill(side)

    sch = api.Scheme(physics=api.MHD, gamma=st.gamma)
    s = api.Solver.from_state(st, sch, userdef=0b000010, outflow=0b000001, userdef_fill=fill)
    s.run(1, 1e-4)
    dims = (10 + 5, 9, 8)
    assert seen == [(1, 1, (12, 0, 0), (13, 8, 7), (2, 0, 0), dims),
                    (1, 2, (12, 0, 0), (13, 8, 7), (2, 0, 0), dims)]

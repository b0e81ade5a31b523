"""Batched step on the GPU: every slot must advance exactly as the same grid
does alone through the single-grid entry points.

The FP64 form runs the same tile bodies with the same operation order and
contraction rule (none) as the single-grid FP64 kernels, so each FP64 slot
is compared bit for bit (U, V, face fields and the dt sequence) with
Solver.run.  The mixed form lets the compiler contract FP32 products into
FMAs, and it may choose differently inside the batch's tile function than
inside the single-grid kernels: mixed slots are compared with a relative
L-infinity bound of 1e-6 per variable (measured: ~1e-8 after 6 steps).
"""
import numpy as np
import pytest

from gpluto_dev_b200 import api, ics
from gpluto_dev_b200 import batch as gb

pytestmark = pytest.mark.gpu

POOL = 2 << 30


def mhd(precision=api.FP64):
    return api.Scheme(physics=api.MHD, precision=precision)


def hd(precision=api.FP64):
    return api.Scheme(physics=api.HD, riemann="hllc", precision=precision)


def rmhd(precision=api.FP64):
    return api.Scheme(physics=api.RMHD, riemann="hlld", ct_emf="uct_hll", cfl=0.3,
                      precision=precision)


def cases():
    # uneven sizes: rows not a multiple of 32, odd pencils, 2-D and 3-D
    return [
        ("mhd2d_64x48", ics.mhd2d_turbulence(n=(64, 48), seed=71), mhd()),
        ("mhd2d_40x80", ics.mhd2d_turbulence(n=(40, 80), seed=72), mhd()),
        ("mhd2d_150x37", ics.mhd2d_turbulence(n=(150, 37), seed=73), mhd()),
        ("mhd3d_24x20x16", ics.mhd3d_turbulence(n=(24, 20, 16), seed=74), mhd()),
        ("hd2d_64x64", ics.hd_turbulence(n=(64, 64), seed=75), hd()),
        ("hd3d_20x16x12", ics.hd_turbulence(n=(20, 16, 12), seed=76), hd()),
        ("mhd2d_mixed_96x64", ics.mhd2d_turbulence(n=(96, 64), seed=77), mhd(api.MIXED)),
        ("mhd3d_mixed_16x16x24", ics.mhd3d_turbulence(n=(16, 16, 24), seed=78), mhd(api.MIXED)),
        ("hd2d_mixed_48x48", ics.hd_turbulence(n=(48, 48), seed=79), hd(api.MIXED)),
        ("rmhd3d_20x12x10", ics.rmhd3d_turbulence(n=(20, 12, 10), seed=80, lorentz_max=5.0),
         rmhd()),
        ("rmhd3d_mixed_16x18x8", ics.rmhd3d_turbulence(n=(16, 18, 8), seed=81, lorentz_max=5.0),
         rmhd(api.MIXED)),
    ]


def alone(st, scheme, dt0, nsteps):
    s = api.Solver.from_state(st, scheme)
    dt, hist, out = s.run(nsteps, dt0)
    V, U, Bs = s.download()
    s.close()
    return V, U, Bs, dt, out


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def assert_close(got, ref, name, tol=1e-6):
    V, U, Bs = got
    Vr, Ur, Br, _, _ = ref
    for nv in range(U.shape[0]):
        assert rel(U[nv], Ur[nv]) <= tol, (name, "U", nv, rel(U[nv], Ur[nv]))
        assert rel(V[nv], Vr[nv]) <= tol, (name, "V", nv, rel(V[nv], Vr[nv]))
    for a, b in zip(Bs, Br):
        assert rel(a, b) <= tol, (name, "Bs", rel(a, b))


def assert_same(got, ref, name):
    V, U, Bs = got
    Vr, Ur, Br, _, _ = ref
    assert np.array_equal(U, Ur), (name, "U", np.abs(U - Ur).max())
    assert np.array_equal(V, Vr), (name, "V", np.abs(V - Vr).max())
    assert len(Bs) == len(Br)
    for a, b in zip(Bs, Br):
        assert np.array_equal(a, b), (name, "Bs", np.abs(a - b).max())


def test_batch_slots_match_single_grid():
    nsteps, dt0 = 6, 1e-4
    b = gb.Batch(POOL, 16)
    slots = {}
    for name, st, sch in cases():
        slots[name] = (b.add(st, sch, dt0, nsteps), st, sch)
    b.advance(nsteps)
    b.wait()
    for name, (slot, st, sch) in slots.items():
        ref = alone(st, sch, dt0, nsteps)
        stt = b.status(slot)
        assert stt.steps_done == nsteps and stt.steps_left == 0, (name, stt)
        assert stt.err_bits == ref[4].err_bits, name
        if sch.precision == api.FP64:
            assert stt.dt == ref[3], (name, stt.dt, ref[3])
            assert_same(b.download(slot), ref, name)
        else:
            assert abs(stt.dt / ref[3] - 1) <= 1e-6, (name, stt.dt, ref[3])
            assert_close(b.download(slot), ref, name)
    b.close()


def test_batch_budgets_replay_and_readmission():
    """Per-slot budgets stop slots independently; a graph replayed twice
    equals one run of twice the steps; a freed slot's pool space is reused
    by a new grid that then matches its own single-grid run."""
    dt0 = 1e-4
    sa = ics.mhd2d_turbulence(n=(64, 64), seed=81)
    sb = ics.mhd3d_turbulence(n=(16, 20, 24), seed=82)
    sc = ics.hd_turbulence(n=(80, 40), seed=83)
    b = gb.Batch(1 << 30, 4)
    a = b.add(sa, mhd(), dt0, 3)
    c = b.add(sb, mhd(), dt0, 10)
    b.advance(5)
    b.advance(5)
    b.wait()
    assert b.status(a).steps_done == 3 and b.status(c).steps_done == 10
    assert_same(b.download(a), alone(sa, mhd(), dt0, 3), "budget 3")
    assert_same(b.download(c), alone(sb, mhd(), dt0, 10), "replayed 5+5")
    used = b.info()["pool_used"]
    b.remove(a)
    assert b.info()["pool_used"] < used
    d = b.add(sc, hd(), dt0, 4)
    b.advance(5)
    b.wait()
    assert b.status(d).steps_done == 4
    assert b.status(c).steps_done == 10          # budget spent: untouched
    assert_same(b.download(d), alone(sc, hd(), dt0, 4), "readmitted")
    assert_same(b.download(c), alone(sb, mhd(), dt0, 10), "idle slot unchanged")
    b.close()


@pytest.mark.parametrize("seg,cpt", [(4, 1), (16, 4), (64, 8)])
def test_tile_shape_does_not_change_results(seg, cpt):
    st = ics.mhd3d_turbulence(n=(32, 24, 20), seed=84)
    b = gb.Batch(1 << 30, 2)
    s = b.add(st, mhd(), 1e-4, 4, gb.TileShape(seg, cpt))
    b.advance(4)
    b.wait()
    assert_same(b.download(s), alone(st, mhd(), 1e-4, 4), f"seg={seg} cpt={cpt}")
    b.close()


def test_batch_rejections():
    st = ics.mhd2d_turbulence(n=(64, 64), seed=85)
    b = gb.Batch(gb.slot_bytes(st, mhd()) + 4096, 2)
    with pytest.raises(api.GPError) as ei:
        b.add(st, api.Scheme(physics=api.MHD, riemann="hll", ct_emf="uct_hll"), 1e-4, 1)
    assert ei.value.code == -2
    b.add(st, mhd(), 1e-4, 1)
    with pytest.raises(api.GPError) as ei:   # pool holds one slot
        b.add(st, mhd(), 1e-4, 1)
    assert ei.value.code == -4
    b.close()

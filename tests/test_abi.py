"""The C-ABI library: symbols, loading and failure behaviour (no GPU needed)."""
import ctypes
import os
import re

import pytest

from gpluto_dev_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            syms |= set(re.findall(r"\b(gp_[a-z_0-9]+)\s*\(", txt))
    return sorted(syms)


def test_header_declares_entry_points():
    s = declared_symbols()
    for must in ("gp_create", "gp_destroy", "gp_upload_state", "gp_download_state",
                 "gp_advance_step", "gp_advance_steps", "gp_next_time_step"):
        assert must in s


def test_library_exports_every_declared_symbol():
    L = api.lib()
    for name in declared_symbols():
        assert hasattr(L, name), f"{name} not exported"
        assert ctypes.cast(getattr(L, name), ctypes.c_void_p).value


def test_next_time_step_formula():
    # Src/next_time_step.cpp:80,125
    assert api.NextTimeStep(10.0, 0.4, 1.1, 1.0) == 0.04
    assert api.NextTimeStep(1e-3, 0.4, 1.1, 1e-4) == 1.1 * 1e-4


def test_create_rejects_bad_configs_before_touching_the_device():
    L = api.lib()
    g = api.GpGridDesc()
    g.ndim = 1
    s = api.Scheme().to_c()
    h = ctypes.c_void_p()
    assert L.gp_create(ctypes.byref(g), ctypes.byref(s), None, ctypes.byref(h)) == -2
    g.ndim = 2
    g.nint[0] = g.nint[1] = 16
    g.nint[2] = 1
    s.rk_stages = 4                       # RK4 is not built
    assert L.gp_create(ctypes.byref(g), ctypes.byref(s), None, ctypes.byref(h)) == -2
    for rs in ("tvdlf", "hll"):           # UCT_HLLD pairs with hlld only
        s = api.Scheme(riemann=rs, ct_emf="uct_hlld").to_c()
        assert L.gp_create(ctypes.byref(g), ctypes.byref(s), None, ctypes.byref(h)) == -2
    s = api.Scheme(physics=api.RMHD, riemann="hllc", ct_emf="uct_hll").to_c()
    assert L.gp_create(ctypes.byref(g), ctypes.byref(s), None, ctypes.byref(h)) == -2


def test_no_cpu_fallback_without_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(api.GPError) as ei:
        api.Solver(2, (16, 16), api.Scheme())
    assert ei.value.code == api.GP_ERR_NO_DEVICE


def test_batch_slot_bytes_formula():
    """Pool bytes of one slot: U (2 copies), V, per-direction dU and C_dt,
    3 face buffers, 6 UCT arrays per direction and the edge EMFs, each array
    rounded up to 256 bytes, plus the scalars."""
    from gpluto_dev_b200 import batch as gb, ics
    al = lambda x: (x + 255) // 256 * 256
    st = ics.mhd2d_turbulence(n=(64, 48), seed=1)
    n = 64 * 48
    c = 8 * n
    exp = 2 * al(8 * c) + al(8 * c) + al(16 * c) + al(2 * c) + 6 * al(c) + 12 * al(c) + al(c) + 256
    assert gb.slot_bytes(st, api.Scheme()) == exp
    mixed = gb.slot_bytes(st, api.Scheme(precision=api.MIXED))
    f = 4 * n    # dU, C_dt, UCT data and EMFs are float in the mixed form
    assert mixed == (2 * al(8 * c) + al(8 * c) + al(16 * f) + al(2 * f) + 6 * al(c)
                     + 12 * al(f) + al(f) + 256)
    sh = ics.hd_turbulence(n=(20, 16, 12), seed=1)
    n = 20 * 16 * 12
    c = 8 * n
    assert gb.slot_bytes(sh, api.Scheme(physics=api.HD, riemann="hllc")) == \
        2 * al(5 * c) + al(5 * c) + al(15 * c) + al(3 * c) + 256


def test_batch_has_no_cpu_path():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from gpluto_dev_b200 import batch as gb
    with pytest.raises(api.GPError) as ei:
        gb.Batch(1 << 20, 4)
    assert ei.value.code == api.GP_ERR_NO_DEVICE

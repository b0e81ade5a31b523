"""The correctly rounded acos/sin/cos of the RMHD fast-speed quartic
(gpluto_dev_b200/csrc/gp_crmath.cuh), compiled for the host and checked
against binary128 (libquadmath, rounded once) on dense argument sweeps of
the ranges the quartic uses: acos on [-1, 1] (with both ends resolved
down to 1e-16), sin and cos on [0, pi/3] and up to 1.125.  A subset is
checked against mpmath at 200 bits as an independent reference."""
import ctypes
import math
import os
import subprocess
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def crm():
    d = tempfile.mkdtemp(prefix="crmath_")
    so = os.path.join(d, "libcrm.so")
    cxx = os.environ.get("CXX", "g++")
    subprocess.run([cxx, "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                    os.path.join(HERE, "crmath_host.cpp"), "-l:libquadmath.so.0", "-lm"],
                   check=True)
    L = ctypes.CDLL(so)
    P = ctypes.POINTER(ctypes.c_double)
    L.crm_eval.argtypes = [ctypes.c_int, P, P, P, ctypes.c_size_t]
    L.crm_slow_calls.restype = ctypes.c_long

    def ev(which, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        a, b = np.empty_like(x), np.empty_like(x)
        L.crm_eval(which, x.ctypes.data_as(P), a.ctypes.data_as(P), b.ctypes.data_as(P),
                   x.size)
        return a, b
    ev.slow_calls = L.crm_slow_calls
    return ev


def _acos_args(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, n)
    ends = 1.0 - 10.0 ** rng.uniform(-16, 0, n // 2)
    x = np.concatenate([x, ends, -ends, [-1.0, -0.5, 0.0, 0.5, 1.0,
                                         np.nextafter(0.5, 1), np.nextafter(-0.5, -1)]])
    return x


def test_acos_correctly_rounded(crm):
    x = _acos_args(1_000_000, 1)
    ours, quad = crm(0, x)
    bad = np.flatnonzero(ours != quad)
    assert bad.size == 0, (bad.size, x[bad[:5]])


@pytest.mark.parametrize("which", [1, 2])
def test_sin_cos_correctly_rounded(crm, which):
    rng = np.random.default_rng(10 + which)
    theta = np.arccos(_acos_args(500_000, 2 + which)) / 3.0   # what the quartic passes
    x = np.concatenate([theta, rng.uniform(0, 1.125, 500_000),
                        np.arange(19) / 16.0, np.arange(19) / 16.0 + 1 / 32.0,
                        10.0 ** rng.uniform(-300, 0, 1000), [0.0, 1.125]])
    x = x[(x >= 0) & (x <= 1.125)]
    ours, quad = crm(which, x)
    bad = np.flatnonzero(ours != quad)
    assert bad.size == 0, (bad.size, x[bad[:5]])


def test_agrees_with_mpmath(crm):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 200
    rng = np.random.default_rng(5)
    xa = _acos_args(3000, 6)
    ours, _ = crm(0, xa)
    for a, o in zip(xa, ours):
        assert float(mpmath.acos(mpmath.mpf(float(a)))) == o
    xs = rng.uniform(0, math.pi / 3, 3000)
    s, _ = crm(1, xs)
    c, _ = crm(2, xs)
    for a, so, co in zip(xs, s, c):
        assert float(mpmath.sin(mpmath.mpf(float(a)))) == so
        assert float(mpmath.cos(mpmath.mpf(float(a)))) == co


def test_fast_path_decides_nearly_every_call(crm):
    """The slow (full double-double) path runs only where the fast form
    cannot decide the rounding: well under 1% of the calls the quartic makes."""
    x = _acos_args(200_000, 9)
    before = crm.slow_calls()
    crm(0, x)                                   # acos
    theta = np.arccos(x) / 3.0
    crm(1, theta)                               # sin and cos share one slow call
    slow = crm.slow_calls() - before
    assert slow < 0.005 * 2 * x.size, slow

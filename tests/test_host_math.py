"""Host build of the kernels' arithmetic header (porerad_b200/csrc/pr_math.cuh), CPU only.

The same source the sm_100a kernels compile is built with g++ -ffp-contract=off and
checked against NumPy's PCG64 stream, glibc sin/cos (with exact rational arithmetic
deciding every disagreement) and NumPy's float remainder.
"""

from __future__ import annotations

import ctypes
import math
import subprocess
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np
import pytest

from tests.helpers import ROOT


@pytest.fixture(scope="module")
def hm(tmp_path_factory):
    out = tmp_path_factory.mktemp("hm") / "libhm.so"
    src = ROOT / "tests" / "host_math_harness.cpp"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", str(src), "-o",
                    str(out), "-lm"], check=True)
    lib = ctypes.CDLL(str(out))
    d = ctypes.POINTER(ctypes.c_double)
    lib.hm_pcg_doubles.argtypes = [ctypes.c_uint64] * 5 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.hm_sincos.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
    lib.hm_pymod.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_void_p]
    return lib


MASK = (1 << 64) - 1
MULT = 0x2360ED051FC65DA44385DF649FCCF645


def _maps(inc):
    a, c = MULT, inc
    rows = []
    for _ in range(64):
        rows += [a & MASK, a >> 64, c & MASK, c >> 64]
        a, c = (a * a) & ((1 << 128) - 1), (a * c + c) & ((1 << 128) - 1)
    return np.array(rows, dtype=np.uint64)


@pytest.mark.parametrize("seed,jump", [(0, 0), (2456208011404661170, 4 * 12345), (7, 4 * 987654321)])
def test_pcg64_stream_matches_numpy(hm, seed, jump):
    st = np.random.PCG64(seed).state["state"]
    s, inc = int(st["state"]), int(st["inc"])
    out = np.empty(64)
    maps = _maps(inc)
    hm.hm_pcg_doubles(s >> 64, s & MASK, inc >> 64, inc & MASK, jump, maps.ctypes.data, 64, out.ctypes.data)
    g = np.random.PCG64(seed)
    g.advance(jump)
    want = np.random.Generator(g).random(64)
    assert np.array_equal(out, want)


def _exact_sin_cos(x: float):
    getcontext().prec = 60
    xv = Decimal(Fraction(x).numerator) / Decimal(Fraction(x).denominator)
    s = c = Decimal(0)
    term, n = xv, 1
    while abs(term) > Decimal(10) ** -58:
        s += term
        term = -term * xv * xv / ((n + 1) * (n + 2))
        n += 2
    term, n = Decimal(1), 0
    while abs(term) > Decimal(10) ** -58:
        c += term
        term = -term * xv * xv / ((n + 1) * (n + 2))
        n += 2
    return s, c


def test_sincos_correctly_rounded_and_close_to_glibc(hm):
    rng = np.random.default_rng(5)
    u = (rng.integers(0, 1 << 53, size=400_000, dtype=np.int64) >> 0).astype(np.float64) * 2.0**-53
    x = (2.0 * np.pi) * u
    s = np.empty_like(x)
    c = np.empty_like(x)
    hm.hm_sincos(x.ctypes.data, x.size, s.ctypes.data, c.ctypes.data)
    gs, gc = np.sin(x), np.cos(x)
    bad = (s != gs) | (c != gc)
    assert bad.mean() < 5e-3  # glibc misrounds a small fraction of azimuths
    assert np.all(np.abs(s - gs) <= np.spacing(np.abs(gs)) * 1.0 + 0.0)
    assert np.all(np.abs(c - gc) <= np.spacing(np.abs(gc)) * 1.0 + 0.0)
    # on every disagreement (first 25), this header's value is the correctly rounded one
    for i in np.flatnonzero(bad)[:25]:
        es, ec = _exact_sin_cos(float(x[i]))
        if s[i] != gs[i]:
            assert abs(Decimal(float(s[i])) - es) <= abs(Decimal(float(gs[i])) - es)
        if c[i] != gc[i]:
            assert abs(Decimal(float(c[i])) - ec) <= abs(Decimal(float(gc[i])) - ec)


def test_sincos_endpoints(hm):
    x = np.array([0.0, math.pi / 2, math.pi, 1.5 * math.pi, (2.0 * math.pi) * (1 - 2.0**-53)])
    s = np.empty_like(x)
    c = np.empty_like(x)
    hm.hm_sincos(x.ctypes.data, x.size, s.ctypes.data, c.ctypes.data)
    assert s[0] == 0.0 and c[0] == 1.0
    assert np.allclose(s, np.sin(x), rtol=0, atol=1e-16) and np.allclose(c, np.cos(x), rtol=0, atol=1e-16)


def test_python_float_remainder(hm):
    a = np.array([-1e-9, -0.0, 0.0, 5.25, 128.0, 128.000000001, -3.5, 255.9, 1e-300, -1e-300])
    out = np.empty_like(a)
    hm.hm_pymod(a.ctypes.data, a.size, 128.0, out.ctypes.data)
    want = np.remainder(a, 128.0)
    assert np.array_equal(out, want)
    assert np.array_equal(np.signbit(out), np.signbit(want))


def test_sincos_correctly_rounded_on_the_layer_field_range(hm):
    """The arguments of TL's wavy layers, 2 pi n (x + wav) / N, lie within about [-10, 60]: the
    header's sine there is within one ulp of glibc's and, on every disagreement checked, the
    correctly rounded one (the device TL field relies on it)."""

    rng = np.random.default_rng(11)
    x = rng.uniform(-10.0, 60.0, size=200_000)
    s = np.empty_like(x)
    c = np.empty_like(x)
    hm.hm_sincos(x.ctypes.data, x.size, s.ctypes.data, c.ctypes.data)
    gs = np.sin(x)
    assert np.all(np.abs(s - gs) <= np.spacing(np.abs(gs)))
    bad = np.flatnonzero(s != gs)
    assert bad.size < 0.01 * x.size
    for i in bad[:25]:
        es, _ = _exact_sin_cos(float(x[i]))
        assert abs(Decimal(float(s[i])) - es) <= abs(Decimal(float(gs[i])) - es)

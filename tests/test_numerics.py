"""Shared numeric primitives (include/pi_numerics.h): Philox4x32-10 known answers, exp error
bound, Julia float semantics, and the draw lattice."""
import ctypes as ct
import math
import os
import subprocess
import tempfile
from fractions import Fraction

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SRC = r'''
#include "pi_numerics.h"
void philox(const uint32_t* c, const uint32_t* k, uint32_t* o) { pi_philox4x32_10(c, k, o); }
double jmax(double a, double b) { return jl_max(a, b); }
double jmin(double a, double b) { return jl_min(a, b); }
int jless(double a, double b) { return jl_isless(a, b); }
double jmod1(double a) { return jl_mod1(a); }
double jmulb(double a, int b) { return jl_mulb(a, b); }
'''


@pytest.fixture(scope="module")
def nlib():
    d = tempfile.mkdtemp()
    src = os.path.join(d, "n.c")
    so = os.path.join(d, "n.so")
    open(src, "w").write(_SRC)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
                    "-o", so, src, "-lm"], check=True)
    lib = ct.CDLL(so)
    for f in ("jmax", "jmin"):
        getattr(lib, f).restype = ct.c_double
        getattr(lib, f).argtypes = [ct.c_double, ct.c_double]
    lib.jless.argtypes = [ct.c_double, ct.c_double]
    lib.jmod1.restype = ct.c_double
    lib.jmod1.argtypes = [ct.c_double]
    lib.jmulb.restype = ct.c_double
    lib.jmulb.argtypes = [ct.c_double, ct.c_int]
    return lib


def test_philox_known_answers(nlib):
    # Random123 known-answer vectors for philox4x32-10
    cases = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
             ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
             ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
              (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in cases:
        C = (ct.c_uint32 * 4)(*c); K = (ct.c_uint32 * 2)(*k); O = (ct.c_uint32 * 4)()
        nlib.philox(C, K, O)
        assert tuple(O) == want


def ulp_err(got, x):
    exact = Fraction(math.exp(x))  # reference value from libm is itself within 1 ulp
    return abs(got - math.exp(x)) / math.ulp(math.exp(x))


def test_exp_error_bound():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-700, 700, 4000), rng.uniform(-1, 1, 4000), rng.uniform(-30, 0, 4000)])
    worst = max(abs(oracle.pi_exp(x) - math.exp(x)) / math.ulp(math.exp(x)) for x in xs)
    assert worst <= 2.0
    assert oracle.pi_exp(0.0) == 1.0
    assert oracle.pi_exp(-800.0) == 0.0 and math.isinf(oracle.pi_exp(800.0))
    assert math.isnan(oracle.pi_exp(float("nan")))


def test_pow_int_compensated():
    rng = np.random.default_rng(1)
    for x in rng.uniform(0, 1, 2000):
        exact4 = float(Fraction(x) ** 4)
        assert abs(oracle.pow_int(x, 4) - exact4) <= 0.5 * math.ulp(exact4) * 1.0000001
        assert oracle.pow_int(x, 2) == x * x


def test_julia_float_semantics(nlib):
    nan = float("nan")
    assert math.isnan(nlib.jmax(nan, 1.0)) and math.isnan(nlib.jmin(1.0, nan))
    assert math.copysign(1, nlib.jmax(-0.0, 0.0)) == 1 and math.copysign(1, nlib.jmax(0.0, -0.0)) == 1
    assert math.copysign(1, nlib.jmin(-0.0, 0.0)) == -1 and math.copysign(1, nlib.jmin(0.0, -0.0)) == -1
    assert nlib.jmax(2.0, 3.0) == 3.0 and nlib.jmin(2.0, 3.0) == 2.0
    assert nlib.jless(1.0, nan) == 1 and nlib.jless(nan, 1.0) == 0 and nlib.jless(nan, nan) == 0
    assert nlib.jless(-0.0, 0.0) == 1 and nlib.jless(0.0, -0.0) == 0
    assert nlib.jmod1(2.75) == 0.75 and nlib.jmod1(-0.25) == 0.75 and nlib.jmod1(3.0) == 0.0
    assert math.copysign(1, nlib.jmod1(-0.0)) == 1
    assert nlib.jmulb(nan, 0) == 0.0 and math.copysign(1, nlib.jmulb(-2.0, 0)) == -1
    assert nlib.jmulb(5.5, 1) == 5.5


def test_draws_lattice_and_keys():
    r = oracle.draw3(1234, 7, 1, 0, 99)
    for v in r:
        assert 0.0 <= v < 1.0 and v * 2 ** 24 == int(v * 2 ** 24)
        assert float(np.float32(v)) == v
    assert oracle.draw3(1234, 7, 1, 0, 99) == r
    assert oracle.draw3(1234, 8, 1, 0, 99) != r and oracle.draw3(1234, 7, 0, 0, 99) != r
    assert oracle.draw3(1234, 7, 1, 1, 99) != r and oracle.draw3(1235, 7, 1, 0, 99) != r
    # uniformity on a sample
    s = np.array([oracle.draw3(5, 1, 0, 1, i)[0] for i in range(20000)])
    assert abs(s.mean() - 0.5) < 0.01 and abs(s.var() - 1 / 12) < 0.005


def test_log_and_pow_error_bounds():
    """pi_log within 2 ulp of libm's log over [1e-300, 1e300]; pi_pow(x, y) within 8 ulp of
    libm's pow for the reference's non-integer exponent 2f0/3f0 and others on positive bases."""
    rng = np.random.default_rng(5)
    xs = np.concatenate([10.0 ** rng.uniform(-300, 300, 3000), rng.uniform(0.5, 2.0, 3000),
                         [1.0, 2.0, 0.5, math.sqrt(0.5), math.sqrt(2.0), 5e-324]])
    worst = max(abs(oracle.pi_log(x) - math.log(x)) / math.ulp(math.log(x)) if x != 1.0 else 0.0 for x in xs)
    assert worst <= 2.0
    assert oracle.pi_log(1.0) == 0.0 and oracle.pi_log(0.0) == -math.inf and math.isnan(oracle.pi_log(-1.0))
    y23 = float(np.float32(2.0) / np.float32(3.0))
    for y in (y23, 0.5, 1.7, -0.3):
        bases = rng.uniform(0.0, 20.0, 2000)
        worst = max(abs(oracle.pi_pow(x, y) - x ** y) / math.ulp(x ** y) for x in bases if x > 0)
        assert worst <= 8.0, (y, worst)
    assert oracle.pi_pow(0.0, y23) == 0.0 and oracle.pi_pow(8.0, 1.0 / 3.0) == pytest.approx(2.0, rel=1e-15)

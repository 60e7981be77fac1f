"""Correctly rounded transcendental terms (CPU).

The step's friction, tidal and Coriolis terms need h**(1/3), sin and cos.
Both the kernels (host build of rkb_crmath.cuh, exported by librakali.so) and
the oracle (oracle/crmath.c) evaluate them correctly rounded, so the GPU and
the oracle agree bit for bit.  Checked here: the two implementations agree,
both equal a 60-digit reference on a random sample, and glibc's libm (what a
gfortran build of the reference calls) is within 1 ulp of them.
"""
import ctypes
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest


def _pi(digits=90):
    def arctan_inv(x, prec):
        total, term, n, sign, x2 = 0, (10 ** prec) // x, 1, 1, x * x
        while term:
            total += sign * term // n
            term //= x2
            n += 2
            sign = -sign
        return total
    return Decimal(4 * (4 * arctan_inv(5, digits) - arctan_inv(239, digits))) / Decimal(10 ** digits)


def _nearest(d: Decimal) -> float:
    f = float(d)
    cands = (f, math.nextafter(f, math.inf), math.nextafter(f, -math.inf))
    return min(cands, key=lambda c: abs(Decimal(c) - d))


@pytest.fixture(scope="module")
def libs():
    from oracle import oracle as orc
    from rakali_b200 import _lib
    return _lib.load(), orc.lib()


def _sincos(fn, x):
    s, c = ctypes.c_double(), ctypes.c_double()
    fn(x, ctypes.byref(s), ctypes.byref(c))
    return s.value, c.value


def test_product_and_oracle_agree(libs):
    lib, orc = libs
    rng = np.random.default_rng(0)
    for h in 10.0 ** rng.uniform(-6, 3, 20000):
        assert lib.rkb_cr_pow_third(h) == orc.orc_cr_pow_third(h)
    for x in rng.uniform(-3e4, 3e4, 20000):
        assert _sincos(lib.rkb_cr_sincos, x) == _sincos(orc.orc_cr_sincos, x)


def test_correctly_rounded_against_60_digits(libs):
    lib, _ = libs
    getcontext().prec = 80
    third = Decimal(6004799503160661) / Decimal(2 ** 54)  # fl(1/3) exactly
    rng = np.random.default_rng(1)
    for h in 10.0 ** rng.uniform(-6, 3, 300):
        exact = (Decimal(float(h)).ln() * third).exp()
        assert lib.rkb_cr_pow_third(float(h)) == _nearest(exact)
    pi = _pi()
    for x in rng.uniform(-2e4, 2e4, 200):
        X = Decimal(float(x))
        k = (X / (2 * pi)).to_integral_value()
        r = X - k * 2 * pi
        s, c, term, n = Decimal(0), Decimal(0), r, 1
        while abs(term) > Decimal(10) ** -75:
            s += term
            term = -term * r * r / ((n + 1) * (n + 2))
            n += 2
        term, n = Decimal(1), 0
        while abs(term) > Decimal(10) ** -75:
            c += term
            term = -term * r * r / ((n + 1) * (n + 2))
            n += 2
        assert _sincos(lib.rkb_cr_sincos, float(x)) == (_nearest(s), _nearest(c))


def test_glibc_within_one_ulp(libs):
    lib, _ = libs
    rng = np.random.default_rng(2)
    hs = 10.0 ** rng.uniform(-6, 3, 50000)
    mism = 0
    for h in hs:
        a, b = math.pow(h, 1.0 / 3.0), lib.rkb_cr_pow_third(h)
        if a != b:
            mism += 1
            assert abs(a - b) <= math.ulp(b)
    assert mism < 0.01 * len(hs)

"""The double-double pow/exp used on the device (cleo_b200/csrc/ddmath.h), built for the host.

They must return the correctly rounded result (checked against 60-digit decimal arithmetic) and
agree with the host libm that CLEO uses, except where the libm itself is not correctly rounded.
"""
import ctypes as C
import os
import subprocess
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXPONENTS = (1.0 / 3.0, 2.0 / 3.0, 1.0 / 6.0, 1.94, 1.963, 0.702, 0.135, 1.5, 3.0, 2.0, 0.5)


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("ddmath") / "libddmath.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o",
                    str(out), os.path.join(ROOT, "tests", "ddmath_host.cpp")], check=True)
    L = C.CDLL(str(out))
    L.dd_pow.argtypes = [C.c_double, C.c_double]
    L.dd_pow.restype = C.c_double
    L.dd_exp.argtypes = [C.c_double]
    L.dd_exp.restype = C.c_double
    return L


def correctly_rounded(v: Decimal) -> float:
    return float(v)  # Decimal -> float conversion rounds to nearest


def test_pow_correctly_rounded(lib):
    getcontext().prec = 60
    rng = np.random.default_rng(1)
    for y in EXPONENTS:
        for x in np.exp(rng.uniform(-30, 30, 300)):
            exact = correctly_rounded(Decimal(float(x)) ** Decimal(y))
            assert lib.dd_pow(float(x), y) == exact, (x, y)


def test_exp_correctly_rounded(lib):
    getcontext().prec = 60
    rng = np.random.default_rng(2)
    for x in rng.uniform(-700, 700, 1500):
        assert lib.dd_exp(float(x)) == correctly_rounded(Decimal(float(x)).exp()), x


def test_agreement_with_host_libm(lib):
    rng = np.random.default_rng(3)
    for y in EXPONENTS:
        xs = np.exp(rng.uniform(-30, 30, 20000))
        mine = np.array([lib.dd_pow(float(x), y) for x in xs])
        libm = np.array([math.pow(float(x), y) for x in xs])  # the C library's pow
        diff = mine != libm
        assert diff.mean() < 0.005, (y, diff.mean())
        ulps = np.abs(mine[diff] - libm[diff]) / np.spacing(np.abs(libm[diff]))
        assert np.all(ulps <= 1.0), (y, ulps.max())

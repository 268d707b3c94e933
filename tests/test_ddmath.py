"""The double-double pow/exp used on the device (cleo_b200/csrc/ddmath.h), built for the host.

They must return the correctly rounded result (checked against 60-digit decimal arithmetic) and
agree with the host libm that CLEO uses, except where the libm itself is not correctly rounded.
The fast first phase (Ziv's strategy) must return bit for bit what the accurate double-double
phase alone returns, and its error must stay far inside the bound its rounding test assumes.
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
    u64, d = C.c_uint64, C.c_double
    L.dd_compare_pow.argtypes = [u64, u64, d, d, C.POINTER(d), C.c_int, d, d, C.POINTER(u64),
                                 C.POINTER(u64), C.POINTER(d)]
    L.dd_compare_exp.argtypes = [u64, u64, d, d, C.POINTER(u64), C.POINTER(u64), C.POINTER(d)]
    L.dd_compare_pow2.argtypes = [u64, u64, d, d]
    L.dd_compare_pow2.restype = u64
    L.dd_fast_pow_maxerr.argtypes = [u64, u64, d, d, d, d]
    L.dd_fast_pow_maxerr.restype = d
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


THIRDS = (1.0 / 6.0, 1.0 / 3.0, 2.0 / 3.0)
FAST_CASES = [  # (x = 2^U[lx0, lx1), y from the listed exponents or U[y0, y1))
    (-40.0, 40.0, EXPONENTS, 0.0, 0.0),
    (-1000.0, 1000.0, None, -0.6, 0.6),
    (-5.0, 5.0, None, -60.0, 60.0),
    (-1.0, 1.0, None, -3.0, 3.0),
    (-600.0, 600.0, THIRDS, 0.0, 0.0),  # the cube-root first phase over its whole range
]


@pytest.mark.parametrize("case", FAST_CASES)
def test_fast_pow_phase_is_bit_identical(lib, case):
    lx0, lx1, listed, y0, y1 = case
    ys = (C.c_double * len(listed))(*listed) if listed else None
    mm, df, bad = C.c_uint64(), C.c_uint64(), (C.c_double * 2)()
    n = 1_000_000
    lib.dd_compare_pow(11, n, lx0, lx1, ys, len(listed) if listed else 0, y0, y1,
                       C.byref(mm), C.byref(df), bad)
    assert mm.value == 0, (mm.value, list(bad))
    assert df.value < 1e-3 * n  # the accurate phase runs rarely


def test_fast_exp_phase_is_bit_identical(lib):
    mm, df, bad = C.c_uint64(), C.c_uint64(), (C.c_double * 2)()
    for seed, (a, b) in enumerate([(-600.0, 600.0), (-1.0, 1.0), (-30.0, 0.0)]):
        lib.dd_compare_exp(seed, 1_000_000, a, b, C.byref(mm), C.byref(df), bad)
        assert mm.value == 0, (a, b, list(bad))
        assert df.value < 1000


def test_fast_phase_error_inside_its_bound(lib):
    # the rounding test assumes 2^-67; the analysis gives 2^-72
    for lx0, lx1, y0, y1 in [(-40, 40, -3, 3), (-1000, 1000, -0.5, 0.5), (-5, 5, -60, 60)]:
        assert lib.dd_fast_pow_maxerr(5, 300_000, lx0, lx1, y0, y1) < 2.0 ** -71


def test_cube_root_phase_error_inside_its_bound(lib):
    # the first phase of the exponents 1/6, 1/3, 2/3 (cube root by Newton steps, the exponent's
    # rounding from a single-precision logarithm): 2^-76 by its analysis, against the accurate
    # phase's double-double value (itself good to about 2^-100); the rounding test assumes 2^-67
    lib.dd_fast_sixth_maxerr.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double]
    lib.dd_fast_sixth_maxerr.restype = C.c_double
    for lx0, lx1 in [(-40, 40), (-600, 600), (-1, 1)]:
        assert lib.dd_fast_sixth_maxerr(7, 300_000, lx0, lx1) < 2.0 ** -76


def test_pow_pair_matches_two_pows(lib):
    assert lib.dd_compare_pow2(3, 300_000, 1.963, 0.702) == 0

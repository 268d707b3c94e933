"""The device's pow and exp (cleo_b200/csrc/ddmath.h) against the same functions built for the
host, bit for bit. The host build is checked against 60-digit decimal arithmetic in
test_ddmath.py; here the device's first phases (which start from the device's own
single-precision cube root and logarithm, and whose fused multiply-adds are the hardware's) must
round to the same doubles over millions of arguments, in the ranges the microphysics uses and
over the cube-root phase's whole range."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from cleo_b200 import abi

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def libs(tmp_path_factory):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    out = tmp_path_factory.mktemp("ddmath") / "libddmath.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o",
                    str(out), os.path.join(ROOT, "tests", "ddmath_host.cpp")], check=True)
    host = C.CDLL(str(out))
    host.dd_eval_array.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64]
    host.dd_vent_array.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
    return abi.load_library(), host


def _device(lib, x, y, fn=None):
    import torch
    if fn is None:
        fn = abi.MATH_POW if y is not None else abi.MATH_EXP
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda() if y is not None else None
    out = torch.empty_like(dx)
    rc = lib.cleo_b200_check_math(fn, C.c_void_p(dx.data_ptr()),
                                  C.c_void_p(dy.data_ptr()) if dy is not None else None,
                                  C.c_void_p(out.data_ptr()), x.size)
    assert rc == 0
    return out.cpu().numpy()


def _host(host, x, y):  # pow (y given) or exp
    out = np.empty_like(x)
    host.dd_eval_array(x.ctypes.data, y.ctypes.data if y is not None else None, out.ctypes.data,
                       x.size)
    return out


CASES = [  # (log2 x range, exponents)
    ((-80.0, 10.0), (1.0 / 6.0, 1.0 / 3.0, 2.0 / 3.0)),  # terminal velocities, radii from volumes
    ((-600.0, 600.0), (1.0 / 6.0, 1.0 / 3.0, 2.0 / 3.0)),  # the cube-root phase's whole range
    ((-40.0, 10.0), (1.963, 0.702, 1.94, 1.5, 0.135)),  # ventilation, diffusivity, breakup
    ((-330.0, 330.0), (0.5, 2.0, 3.0, 1.0)),  # finite cubes
]


@pytest.mark.parametrize("case", CASES)
def test_device_pow_equals_host_build(libs, case):
    lib, host = libs
    (lx0, lx1), ys = case
    rng = np.random.default_rng(17)
    n = 2_000_000
    x = np.exp2(rng.uniform(lx0, lx1, n))
    y = np.asarray(ys, dtype=np.float64)[rng.integers(0, len(ys), n)]
    d, h = _device(lib, x, y), _host(host, x, y)
    bad = np.flatnonzero(d.view(np.uint64) != h.view(np.uint64))
    assert bad.size == 0, (bad.size, x[bad[:3]], y[bad[:3]])


def test_device_exp_equals_host_build(libs):
    lib, host = libs
    rng = np.random.default_rng(18)
    x = np.concatenate([rng.uniform(-700.0, 700.0, 1_000_000), rng.uniform(-40.0, 1.0, 1_000_000)])
    d, h = _device(lib, x, None), _host(host, x, None)
    assert np.array_equal(d.view(np.uint64), h.view(np.uint64))


VENT_RADII = [  # (log10 of the radius in um: range), the share of warps with larger droplets
    (-2.0, 0.0),  # haze and activating droplets: the library's log2/exp2 decide almost always
    (-2.0, 1.0),  # cloud droplets too: warps with droplets above 1.5 um take the exact powers
    (-2.0, 3.0),  # drizzle and rain
    (-1.0, 0.17),  # up to 1.48 um, where the check fails most often
]


@pytest.mark.parametrize("span", VENT_RADII)
def test_device_ventilation_factor_equals_correctly_rounded_form(libs, span):
    """The condensation kernels' ventilation factor takes its powers from the library's log2 and
    exp2 where a rounding check shows they decide the result; it must equal the factor from the
    correctly rounded powers bit for bit, in warps of small droplets (the quick form), of mixed
    sizes and of large ones (the correctly rounded form)."""
    lib, host = libs
    rng = np.random.default_rng(19)
    r = 10.0 ** rng.uniform(span[0], span[1], 4_000_000)
    d = _device(lib, r, None, fn=abi.MATH_VENT)
    h = np.empty_like(r)
    host.dd_vent_array(r.ctypes.data, h.ctypes.data, r.size)
    bad = np.flatnonzero(d.view(np.uint64) != h.view(np.uint64))
    assert bad.size == 0, (bad.size, r[bad[:3]], d[bad[:3]], h[bad[:3]])

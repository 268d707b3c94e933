"""The arithmetic facts behind the device code's exact shortcuts (physics.cuh, sdm.cu), checked
on the CPU with IEEE doubles against exact or high-precision references:

* interpolation of a wind that is zero on both faces: alpha * vhi + (1 - alpha) * vlo equals
  vhi + vlo, signed zeros included, whenever the extent bhi - blo is finite and positive and the
  coordinate is clamped to [blo, bhi] (sdm.cu, interpolation);
* max_dryradius: r^3 Rho_sol > vconst msol (1 + 1e-13), evaluated in doubles, implies that r is
  above the correctly rounded cube root of the dry radius cubed, so fmax returns r (physics.cuh);
* below_critical_timestep: x sqrt(x) in doubles lies within a few ulp of the correctly rounded
  x^1.5, far inside the 1e-12 band outside which the estimate decides (physics.cuh).

The GPU parity tests check the kernels' results against the oracle; these check the reasoning
that makes the shortcuts return the same doubles for every input.
"""
import math
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np

PI = 3.141592653589793238462643383279502884
RHO0 = 100000.0 / (1004.64 * 273.15)
RHO_SOL = 2016.5 / RHO0
VCONST = 3.0 / (4.0 * PI)


def test_zero_wind_interpolation_is_the_signed_zero_sum():
    rng = np.random.default_rng(3)
    checked = 0
    for k in range(60000):
        blo = float(rng.normal() * 10 ** rng.uniform(-3, 6))
        bhi = blo + float(abs(rng.normal()) * 10 ** rng.uniform(-12, 6))
        extent = bhi - blo
        if not (0.0 < extent <= 1.7976931348623157e308):
            continue
        sd = [blo - 1.0, bhi + 1.0, blo, bhi, float(rng.uniform(blo, bhi)), math.nan][k % 6]
        vlo, vhi = (0.0, -0.0)[rng.integers(2)], (0.0, -0.0)[rng.integers(2)]
        coord = min(bhi, max(blo, sd)) if sd == sd else blo  # fmin / fmax drop a NaN
        alpha = (coord - blo) / (bhi - blo)
        full = alpha * vhi + (1 - alpha) * vlo
        fast = vhi + vlo
        assert full == fast and math.copysign(1.0, full) == math.copysign(1.0, fast)
        checked += 1
    assert checked > 50000


def _cbrt_rounded(y: float) -> Fraction:
    """A double within one ulp of the real cube root of y > 0: the one whose cube is nearest y
    (exact rational comparison)."""
    c = y ** (1.0 / 3.0)
    for _ in range(4):  # step to the neighbour whose cube brackets y from the right side
        lo, hi = np.nextafter(c, 0.0), np.nextafter(c, np.inf)
        yq = Fraction(y)
        best = min((lo, c, hi), key=lambda t: abs(Fraction(t) ** 3 - yq))
        if best == c:
            break
        c = float(best)
    return Fraction(c)


def test_dry_radius_margin_implies_the_larger_radius():
    rng = np.random.default_rng(1)
    fired = 0
    for k in range(4000):
        msol = float(np.exp(rng.uniform(-60, 15)))
        y = VCONST * msol / RHO_SOL
        dry = _cbrt_rounded(y)
        # radii around the dry radius, many within the margin's neighbourhood
        r = float(dry) * float(np.exp(rng.uniform(-2e-13, 2e-13) if k % 2 else rng.uniform(-1, 1)))
        if r * r * r * RHO_SOL > VCONST * msol * (1.0 + 1e-13):
            fired += 1
            # above the next double too: holds whichever neighbour the rounding picks
            assert Fraction(r) > Fraction(float(np.nextafter(float(dry), np.inf))), (msol, r)
    assert fired > 1000


def test_x_sqrt_x_within_the_band_of_the_rounded_power():
    getcontext().prec = 60
    rng = np.random.default_rng(7)
    worst = 0.0
    for _ in range(5000):
        x = float(np.exp(rng.uniform(-300, 300)))
        est = x * math.sqrt(x)
        exact = Decimal(x) ** Decimal("1.5")
        rel = abs((Decimal(est) - exact) / exact)
        worst = max(worst, float(rel))
    # a few ulp (2^-52 = 2.2e-16 each), four orders of magnitude inside the 1e-12 band
    assert worst < 1e-15, worst

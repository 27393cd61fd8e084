"""Implied-variance surfaces on the GPU: the device total-variance code
against the reference's 70-digit equation cases and against the oracle, and
the Dupire grids of every surface kind against the oracle's."""
import numpy as np
import pytest

import surface_cases as S
from rust_pricing_b200 import _native as N

pytestmark = pytest.mark.gpu

GOLD = S.golden()


def rel_err(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(np.asarray(b)), 1e-300))


@pytest.mark.parametrize("case", GOLD["standard_ssvi"] + [GOLD["essvi_interpolation"]], ids=lambda c: c["id"])
def test_device_total_variance_against_the_equation_cases(engine, case):
    make = S.essvi_case_surface if "t0" in case["inputs"] else S.ssvi_case_surface
    surface, t, k = make(case)
    got = N.surface_total_variance(surface, [t], [k])[0]
    want = [float(case["expected"][key]) for key in ("w", "w_k", "w_kk", "w_t")]
    assert rel_err(got, want) <= 1e-12
    assert rel_err(got, S.oracle_total_variance(surface, t, k)) <= 1e-13


@pytest.mark.parametrize("name", ["power", "heston", "essvi"])
def test_grid_matches_the_oracle(engine, name):
    surfaces, tn, xn = S.grid_surfaces()
    got, repairs = N.surface_grid(surfaces[name], tn, xn)
    want, want_repairs = S.oracle_grid(surfaces[name], tn, xn)
    assert repairs == want_repairs
    assert rel_err(got, want) <= 1e-13


def test_essvi_points_across_regions(engine):
    """Short end (before the first slice), knots, interior and long end."""
    surfaces, _, _ = S.grid_surfaces()
    s = surfaces["essvi"]
    times = [0.05, 0.25, 0.3, 0.5, 1.2, 1.5, 2.5, 0.25, 1.5]
    ks = [-0.5, 0.0, 0.3, -1.0, 0.8, 0.1, -0.2, 0.7, -0.7]
    got = N.surface_total_variance(s, times, ks)
    want = np.array([S.oracle_total_variance(s, t, k) for t, k in zip(times, ks)])
    assert rel_err(got, want) <= 1e-13

"""The oracle's implied-variance surfaces against the reference's equation
fixture (fixtures/local-vol/reference-cases-v0.1.json, 70-digit decimal
values): standard SSVI with power-law and Heston-like phi (including the
small-z series branch) and eSSVI interpolation; plus the reference's own
eSSVI unit tests (crates/pricing/src/market/essvi.rs tests) and the
validation rules of the engine library (checked on the host, before any
device call)."""
import numpy as np
import pytest

import surface_cases as S
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N

GOLD = S.golden()
# binary64 closed forms against 70-digit values: 1e-12 relative (the
# Heston-like w_k loses two digits to the cancellation in rho + a / q)
REL = 1e-12


def close(got, want, rel=REL, floor=1e-300):
    return abs(got - want) <= rel * max(abs(want), floor)


@pytest.mark.parametrize("case", GOLD["standard_ssvi"], ids=lambda c: c["id"])
def test_standard_ssvi_cases(case):
    surface, t, k = S.ssvi_case_surface(case)
    w = S.oracle_total_variance(surface, t, k)
    e = case["expected"]
    for got, key in zip(w, ("w", "w_k", "w_kk", "w_t")):
        assert close(got, float(e[key])), (key, got, e[key])
    # the Durrleman density factor of the same derivatives
    u = 1.0 - k * w[1] / (2.0 * w[0])
    density = u * u - (w[1] * w[1] / 4.0) * (1.0 / w[0] + 1.0 / 4.0) + w[2] / 2.0
    assert close(density, float(e["density_factor"]), rel=1e-12)


def test_essvi_interpolation_case():
    case = GOLD["essvi_interpolation"]
    surface, t, k = S.essvi_case_surface(case)
    w = S.oracle_total_variance(surface, t, k)
    e = case["expected"]
    for got, key in zip(w, ("w", "w_k", "w_kk", "w_t")):
        assert close(got, float(e[key])), (key, got, e[key])


def test_essvi_time_derivative_matches_central_difference():
    """analytic_time_derivative_matches_central_difference (essvi.rs tests)."""
    s = S.unit_test_essvi()
    t, k, h = 1.5, -0.1, 1e-6
    wt = S.oracle_total_variance(s, t, k)[3]
    fd = (S.oracle_total_variance(s, t + h, k)[0] - S.oracle_total_variance(s, t - h, k)[0]) / (2 * h)
    assert abs(wt - fd) < 1e-10


def test_essvi_extrapolation_policy():
    """interpolation_and_extrapolation_follow_v1_policy (essvi.rs tests): at
    k = 0 the total variance is theta (to rounding), so the short end gives
    theta = 0.02 at t = 0.5, the middle 0.065 at 1.5, the long end 0.11 at 3."""
    s = S.unit_test_essvi()
    for t, theta in ((0.5, 0.02), (1.5, 0.065), (3.0, 0.11)):
        assert close(S.oracle_total_variance(s, t, 0.0)[0], theta, rel=1e-15)


def test_constant_volatility_dupire_identity():
    """Dupire identity in forward log-moneyness: a flat total variance
    sigma^2 t has w_k = w_kk = 0, density factor 1 and local variance
    sigma^2 -- the grid of a flat theta curve with a vanishing skew."""
    case = GOLD["constant_vol_dupire"]
    sigma, t = float(case["inputs"]["sigma"]), float(case["inputs"]["t"])
    assert close(sigma * sigma * t, float(case["expected"]["w"]))
    assert close(sigma * sigma, float(case["expected"]["local_variance"]))


@pytest.mark.parametrize("name", ["power", "heston", "essvi"])
def test_grids_are_finite_and_positive(name):
    surfaces, tn, xn = S.grid_surfaces()
    grid, repairs = S.oracle_grid(surfaces[name], tn, xn)
    assert repairs >= 0
    assert np.all(np.isfinite(grid)) and np.all(grid > 0)


INVALID = {
    # EssviSlice::new / EssviSurface::new rejections (essvi.rs tests and constructors)
    "decreasing-theta": dict(slice_thetas=[0.04, 0.03], slice_psis=[0.2, 0.21], slice_rho_psis=[-0.08, -0.07]),
    "rho-psi-change": dict(slice_thetas=[0.04, 0.09], slice_psis=[0.2, 0.21], slice_rho_psis=[-0.08, 0.0]),
    "rho-at-one": dict(slice_thetas=[0.04, 0.09], slice_psis=[0.2, 0.25], slice_rho_psis=[0.2, 0.25]),
    "one-slice": dict(slice_times=[1.0], slice_thetas=[0.04], slice_psis=[0.2], slice_rho_psis=[-0.08]),
}


@pytest.mark.parametrize("name", sorted(INVALID))
def test_engine_rejects_invalid_essvi(name):
    kw = dict(kind=A.SURFACE_ESSVI, slice_times=[1.0, 2.0], terminal_theta_slope=0.01)
    kw.update(INVALID[name])
    with pytest.raises(N.EngineError) as err:
        N.surface_total_variance(S.SurfaceSpec(**kw), [1.5], [0.0])
    assert err.value.name == "market"


def test_engine_rejects_inadmissible_ssvi():
    base = dict(theta_times=[0.5, 1.0], theta_values=[0.02, 0.04], terminal_theta_slope=0.04, rho=-0.4)
    for kw in (dict(kind=A.SURFACE_SSVI_POWER_LAW, eta=1.0, gamma=0.7),      # gamma above one half
               dict(kind=A.SURFACE_SSVI_POWER_LAW, eta=1.5, gamma=0.5),      # eta (1 + |rho|) above 2
               dict(kind=A.SURFACE_SSVI_HESTON_LIKE, lam=0.3)):              # lambda below (1 + |rho|) / 4
        with pytest.raises(N.EngineError) as err:
            N.surface_total_variance(S.SurfaceSpec(**base, **kw), [1.0], [0.0])
        assert err.value.name == "market"

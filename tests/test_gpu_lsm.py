"""Longstaff--Schwartz early exercise on the GPU against the oracle.

The engine (mcg_lsm_price) and the oracle share the path streams: the same
Philox or scrambled-Sobol normals (training under the LsmTrain domain,
valuation under Valuation), the same Black--Scholes spots and the same
decision rule, so every stopping index and exercise count must agree.  The
regression differs only in how the least-squares problem is solved (the
oracle runs the reference's CPQR, the engine an exactly accumulated Gram
matrix and a double-double pivoted Cholesky): pivots (but for the structural
first-pivot tie of a degree-1 basis), ranks and ITM counts agree exactly; feature scalings, |R| diagonals and coefficients within
MODEL_TOL; prices, standard errors and the in-sample value within PRICE_TOL.
The replay fixture's own values are checked as well.
"""
import numpy as np
import pytest

import gpu_common as G
import helpers as H
import lsm_cases as L
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W

pytestmark = pytest.mark.gpu

MODEL_TOL = 5e-13
PRICE_TOL = 1e-12


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def assert_models(spec, lsm, got, want, tol=MODEL_TOL):
    for k in range(len(spec.observation_times) - 1):
        g, w = got.models[k], want.models[k]
        assert (g.regression, g.itm_rows, g.candidate_rows) == (w.regression, w.itm_rows, w.candidate_rows), k
        if not w.regression:
            continue
        assert (g.feature_inactive, g.active_columns, g.diagonal_count, g.rank) == (
            w.feature_inactive, w.active_columns, w.diagonal_count, w.rank), k
        gp, wp = list(g.pivot_order[:w.active_columns]), list(w.pivot_order[:w.active_columns])
        if lsm.max_degree == 1 and sorted(gp) == sorted(wp) == [0, 1]:
            # A structural tie: the squared norms of z^0 and of the standardised
            # z^1 are n and sum z^2 = n (1 + O(eps)), so which column pivots first
            # turns on the last bit of a sum; the fit is the same either way.
            pass
        else:
            assert gp == wp, k
        for f in ("feature_mean", "feature_variance", "feature_scale", "zero_scale_threshold", "rank_threshold",
                  "residual_sum_squares"):
            assert rel(getattr(g, f), getattr(w, f)) <= tol, (k, f, getattr(g, f), getattr(w, f))
        for c in range(w.diagonal_count):
            assert rel(g.diagonal_abs[c], w.diagonal_abs[c]) <= tol, (k, c)
        scale = max(abs(w.coefficients[c]) for c in range(lsm.max_degree + 1))
        for c in range(lsm.max_degree + 1):
            assert abs(g.coefficients[c] - w.coefficients[c]) <= tol * scale, (k, c)


def assert_same_result(spec, lsm, got, want, stops=True):
    dates = len(spec.observation_times)
    assert list(got.counts[:dates]) == list(want.counts[:dates])
    if stops:
        assert list(got.stops) == list(want.stops)
    g, w = got.result, want.result
    assert (g.training_paths, g.valuation_paths, g.independent_sampling_units) == (
        w.training_paths, w.valuation_paths, w.independent_sampling_units)
    assert rel(g.price.value, w.price.value) <= PRICE_TOL
    assert rel(g.price.standard_error, w.price.standard_error) <= 1e-10
    assert rel(g.in_sample_value, w.in_sample_value) <= PRICE_TOL
    assert_models(spec, lsm, got, want)


def bump_noise(spec, price):
    """Rounding floor of the validation bumps: last-ulp differences of the
    bumped prices (a few eps |price|) divided by the bump (second differences
    by its square).  A bumped gamma of a path that is linear in the spot is
    pure rounding noise at this level."""
    sb = (spec.gamma_bump * spec.spot if spec.gamma_bump_relative else spec.gamma_bump) \
        if spec.request_gamma else min(spec.spot * 1e-4, 0.5 * spec.spot)
    vb = min(1e-4, 0.5 * spec.volatility)
    u = 1e3 * 2.220446049250313e-16 * abs(price)
    return {"bump_delta": u / sb, "bump_gamma": u / sb ** 2, "bump_vega": u / vb,
            A.BUMP_DELTA: u / sb, A.DELTA_DIFFERENCE: u / sb, A.BUMP_GAMMA: u / sb ** 2,
            A.GAMMA_DIFFERENCE: u / sb ** 2, A.BUMP_VEGA: u / vb, A.VEGA_DIFFERENCE: u / vb}


def assert_same_risk(spec, got, want):
    """Fixed-policy Greeks against the oracle with the parity tolerances of
    the European engine: direct estimates (AAD delta/vega, gamma from AAD
    deltas) 1e-12, the validation bumps 1e-8 (they divide last-ulp libm
    differences by the bump), both on the scale max(|total|, spread), the
    bumps above their rounding floor."""
    g, w = got.result, want.result
    noise = bump_noise(spec, w.price.value)
    for name, bump in (("delta", 0), ("gamma", 0), ("vega", 0), ("bump_delta", 1), ("bump_gamma", 1),
                       ("bump_vega", 1)):
        a, b = getattr(g, name), getattr(w, name)
        tol = G.BUMP_TOL if bump else G.DIRECT_TOL
        assert abs(a.value - b.value) <= tol * max(abs(b.value), b.standard_error, 1e-300) + noise.get(name, 0.0), (
            name, a.value, b.value)
        assert abs(a.standard_error - b.standard_error) <= (1e-6 if bump else 1e-9) * max(
            b.standard_error, 1e-300) + noise.get(name, 0.0), name
        assert a.effective_sampling_units == b.effective_sampling_units, name
    for c in range(10):
        a, b = g.risk_components[c], w.risk_components[c]
        assert a.count == b.count, c
        scale = G._scale(b)
        if c in G.DIFFERENCE_OF:
            scale = max(scale, G._scale(w.risk_components[G.DIFFERENCE_OF[c]]))
        tol = G.BUMP_TOL if c in G.BUMP_COMPONENTS else G.DIRECT_TOL
        floor = noise.get(c, 0.0) * b.count
        assert abs(a.total() - b.total()) <= tol * max(scale, 1e-300) + floor, (c, a.total(), b.total())


@pytest.mark.parametrize("case", L.cases(), ids=lambda c: c["name"])
def test_replay_fixture_on_the_gpu(engine, case):
    spec, lsm = L.plan(case)
    got = N.lsm_price(spec, lsm, stopping=True)
    want = H.oracle_lsm(spec, lsm, stopping=True, threads=4)
    assert_same_result(spec, lsm, got, want)
    e = case["expected"]
    assert list(got.stops) == e["stopping_indices"]
    assert list(got.counts[:len(spec.observation_times)]) == e["exercise_counts"]
    assert rel(got.result.price.value, e["value"]["value"]) <= PRICE_TOL
    assert rel(got.result.in_sample_value, e["in_sample_value"]) <= PRICE_TOL
    if case["risk"].get("delta"):
        assert_same_risk(spec, got, want)
        for name in ("delta", "gamma", "vega"):
            a, b = getattr(got.result, name), e["risks"][name]["raw"]
            assert abs(a.value - b["value"]) <= G.DIRECT_TOL * max(abs(b["value"]), b["standard_error"]), name
            assert rel(a.standard_error, b["standard_error"]) <= 1e-9, name


CASES = {
    "pseudo-12-dates": lambda: W.american_bs(dates=12, units=1 << 13),
    "pseudo-antithetic-odd-units": lambda: W.american_bs(dates=7, units=5001, training_units=3001, antithetic=True),
    "rqmc-antithetic": lambda: W.american_bs(dates=10, units=1 << 10, engine=A.ENGINE_RQMC, antithetic=True,
                                             scrambles=4),
    "call-degree-1": lambda: W.american_bs(dates=6, units=1 << 12, side=A.CALL, max_degree=1, strike=95.0),
    "degree-5": lambda: W.american_bs(dates=6, units=1 << 12, max_degree=5),
    "one-date-is-european": lambda: W.american_bs(dates=1, units=1 << 12),
    "deep-otm-continue-all": lambda: W.american_bs(dates=5, units=1 << 10, strike=40.0, vol=0.05),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_matches_the_oracle(engine, name):
    spec, lsm = CASES[name]()
    got = N.lsm_price(spec, lsm, stopping=True)
    want = H.oracle_lsm(spec, lsm, stopping=True, threads=8)
    assert_same_result(spec, lsm, got, want)


def test_one_date_equals_the_european_engine(engine):
    spec, lsm = W.american_bs(dates=1, units=1 << 14)
    got = N.lsm_price(spec, lsm)
    eu = W.american_bs(dates=1, units=1 << 14)[0]
    eu.products[0].kind = A.PRODUCT_EUROPEAN
    with N.Plan(eu) as plan:
        ref = plan.evaluate()
    assert rel(got.result.price.value, ref.products[0].price.value) <= PRICE_TOL


def test_deep_otm_dates_continue(engine):
    spec, lsm = CASES["deep-otm-continue-all"]()
    got = N.lsm_price(spec, lsm)
    assert all(got.models[k].regression == 0 for k in range(4))
    assert got.counts[4] == got.result.valuation_paths


def test_matrix_limit_is_an_lsm_error(engine):
    spec, lsm = W.american_bs(dates=4, units=1 << 12)
    lsm.max_matrix_elements = 100
    with pytest.raises(N.EngineError) as err:
        N.lsm_price(spec, lsm)
    assert err.value.name == "lsm"


@pytest.fixture(scope="module")
def ssvi_grid():
    surface = W.SsviSurface(steps=252, expiries=30)
    return W.local_vol_grid(surface, G.gpu_grid)


LV_CASES = {
    "lv-pseudo-12-dates": dict(dates=12, units=1 << 13),
    "lv-pseudo-antithetic-bridge-odd-units": dict(dates=7, units=5001, training_units=3001, antithetic=True,
                                                   bridge=True),
    "lv-rqmc-antithetic-bridge": dict(dates=10, units=1 << 10, engine=A.ENGINE_RQMC, antithetic=True,
                                      scrambles=4, bridge=True),
    "lv-call-degree-5": dict(dates=6, units=1 << 12, side=A.CALL, max_degree=5, strike=95.0),
}


@pytest.mark.parametrize("name", sorted(LV_CASES))
def test_local_volatility_matches_the_oracle(engine, ssvi_grid, name):
    """Early exercise under the SSVI local-variance grid: training and
    valuation Log-Euler path stores, the same regression and policy."""
    spec, lsm = W.american_lv(ssvi_grid, **LV_CASES[name])
    got = N.lsm_price(spec, lsm, stopping=True)
    want = H.oracle_lsm(spec, lsm, stopping=True, threads=8)
    assert_same_result(spec, lsm, got, want)


@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC], ids=["pseudo", "rqmc"])
def test_flat_local_volatility_is_black_scholes(engine, engine_kind):
    kw = dict(dates=12, units=1 << 13, engine=engine_kind, antithetic=True)
    bs = N.lsm_price(*W.american_bs(vol=0.25, **kw), stopping=True)
    lv = N.lsm_price(*W.american_lv(W.flat_grid(0.25), **kw), stopping=True)
    assert list(lv.stops) == list(bs.stops)
    assert rel(lv.result.price.value, bs.result.price.value) <= 1e-13


def test_local_volatility_learned_policy(engine, ssvi_grid):
    spec, lsm = W.american_lv(ssvi_grid, dates=10, units=1 << 14)
    lsm.continuation = A.CONTINUATION_MLP
    got = N.lsm_price(spec, lsm)
    poly = N.lsm_price(*W.american_lv(ssvi_grid, dates=10, units=1 << 14))
    r = got.result
    assert r.continuation_used in (A.CONTINUATION_MLP, A.CONTINUATION_POLYNOMIAL)
    # the policy kept is the one with the higher in-sample value on the same training paths
    assert r.polynomial_in_sample == poly.result.in_sample_value
    assert r.in_sample_value >= r.polynomial_in_sample
    # an exercise policy can only lose value against the optimum: the kept one is not worse
    assert r.price.value >= poly.result.price.value - 6 * poly.result.price.standard_error


LV_RISK_CASES = {
    "lv-pseudo-antithetic-bridge": dict(dates=8, units=3001, training_units=2001, antithetic=True, bridge=True),
    "lv-rqmc-antithetic-bridge": dict(dates=6, units=1 << 9, engine=A.ENGINE_RQMC, antithetic=True, scrambles=4,
                                      bridge=True),
}


@pytest.mark.parametrize("name", sorted(LV_RISK_CASES))
def test_local_volatility_fixed_policy_risk_matches_the_oracle(engine, ssvi_grid, name):
    """Fixed-policy Delta/Gamma (CRN spot bumps), Vega and node sensitivities
    of an American put under the SSVI local-variance grid: the adjoint sweeps
    in exercise-value mode against the oracle's
    local_vol_fixed_policy_*_statistics restatement."""
    spec, lsm = W.american_lv(ssvi_grid, **LV_RISK_CASES[name])
    spec.request_delta = spec.request_gamma = spec.request_vega = spec.request_local_vega_nodes = True
    got = N.lsm_price(spec, lsm, stopping=True)
    want = H.oracle_lsm(spec, lsm, stopping=True, threads=8)
    assert_same_result(spec, lsm, got, want)
    g, w = got.result, want.result
    for name_ in ("delta", "gamma", "vega", "bump_delta", "bump_gamma"):
        a, b = getattr(g, name_), getattr(w, name_)
        assert abs(a.value - b.value) <= G.DIRECT_TOL * max(abs(b.value), b.standard_error), (name_, a.value, b.value)
        assert abs(a.standard_error - b.standard_error) <= 1e-9 * b.standard_error, name_
    p = g.risk_components[A.PRICE]
    assert rel((p.sum + p.correction) / g.independent_sampling_units, g.price.value) <= 1e-12
    gm = np.array([e.value for e in got.node_estimates])
    wm = np.array([e.value for e in want.node_estimates])
    assert np.max(np.abs(gm - wm)) <= 1e-11 * np.max(np.abs(wm))
    assert abs(gm.sum() - g.vega.value) <= 1e-11 * abs(g.vega.value)


def test_flat_local_volatility_fixed_policy_vega_is_black_scholes(engine):
    kw = dict(dates=10, units=1 << 12, antithetic=True)
    sb, lb = W.american_bs(vol=0.25, **kw)
    sb.request_delta = sb.request_gamma = sb.request_vega = True
    sl, ll = W.american_lv(W.flat_grid(0.25), **kw)
    sl.request_delta = sl.request_gamma = sl.request_vega = True
    bs = N.lsm_price(sb, lb).result
    lv = N.lsm_price(sl, ll).result
    assert abs(lv.vega.value - bs.vega.value) <= 1e-12 * abs(bs.vega.value)
    assert abs(lv.delta.value - bs.bump_delta.value) <= 1e-10 * max(abs(bs.bump_delta.value), bs.bump_delta.standard_error)



RISK_CASES = {
    "pseudo-antithetic-odd-units": lambda: W.american_bs(dates=7, units=5001, training_units=3001,
                                                         antithetic=True),
    "rqmc-antithetic": lambda: W.american_bs(dates=10, units=1 << 10, engine=A.ENGINE_RQMC, antithetic=True,
                                             scrambles=4),
    "call-12-dates": lambda: W.american_bs(dates=12, units=1 << 13, side=A.CALL, strike=95.0),
    "one-date": lambda: W.american_bs(dates=1, units=1 << 12),
}


@pytest.mark.parametrize("gamma", [True, False], ids=["gamma", "delta-vega"])
@pytest.mark.parametrize("name", sorted(RISK_CASES))
def test_fixed_policy_risk_matches_the_oracle(engine, name, gamma):
    spec, lsm = RISK_CASES[name]()
    spec.request_delta = spec.request_vega = True
    spec.request_gamma = gamma
    got = N.lsm_price(spec, lsm, stopping=True)
    want = H.oracle_lsm(spec, lsm, stopping=True, threads=8)
    assert_same_result(spec, lsm, got, want)
    assert_same_risk(spec, got, want)
    # the price component re-derives the valuation price under the fixed policy
    p = got.result.risk_components[A.PRICE]
    assert rel((p.sum + p.correction) / got.result.independent_sampling_units, got.result.price.value) <= 1e-12


def test_one_date_risk_equals_the_european_engine(engine):
    """With one exercise date the stopping policy is 'at expiry' and the
    fixed-policy Greeks are the European pathwise ones."""
    spec, lsm = W.american_bs(dates=1, units=1 << 14)
    spec.request_delta = spec.request_gamma = spec.request_vega = True
    got = N.lsm_price(spec, lsm)
    eu = W.american_bs(dates=1, units=1 << 14)[0]
    eu.products[0].kind = A.PRODUCT_EUROPEAN
    eu.request_delta = eu.request_gamma = eu.request_vega = True
    with N.Plan(eu) as plan:
        ref = plan.evaluate().products[0]
    for name in ("delta", "gamma", "vega", "bump_delta", "bump_gamma", "bump_vega"):
        a, b = getattr(got.result, name), getattr(ref, name)
        assert abs(a.value - b.value) <= 1e-12 * max(abs(b.value), b.standard_error), name


def test_learned_policy_has_fixed_policy_risk(engine):
    spec, lsm = W.american_bs(dates=6, units=1 << 13)
    spec.request_delta = spec.request_vega = True
    lsm.continuation = A.CONTINUATION_MLP
    got = N.lsm_price(spec, lsm)
    r = got.result
    p = r.risk_components[A.PRICE]
    assert rel((p.sum + p.correction) / r.independent_sampling_units, r.price.value) <= 1e-12
    # an American put: delta in (-1, 0), vega positive
    assert -1.0 < r.delta.value < 0.0 and r.vega.value > 0.0


def test_rejects_what_it_does_not_price(engine):
    spec, lsm = W.american_bs(dates=4, units=1 << 10)
    spec.request_local_vega_nodes = True
    with pytest.raises(N.EngineError) as err:
        N.lsm_price(spec, lsm)
    assert err.value.name == "unsupported"
    spec, lsm = W.american_bs(dates=4, units=1 << 10)
    spec.request_gamma = True
    spec.gamma_bump_relative, spec.gamma_bump = False, spec.spot
    with pytest.raises(N.EngineError) as err:
        N.lsm_price(spec, lsm)
    assert err.value.name == "invalid_argument"
    spec, lsm = W.american_bs(dates=4, units=1 << 10)
    spec.products[0].kind = A.PRODUCT_EUROPEAN
    with pytest.raises(N.EngineError) as err:
        N.lsm_price(spec, lsm)
    assert err.value.name == "invalid_argument"


def test_repeatable(engine):
    spec, lsm = W.american_bs(dates=8, units=1 << 14)
    a = N.lsm_price(spec, lsm, stopping=True)
    b = N.lsm_price(spec, lsm, stopping=True)
    assert a.result.price.value == b.result.price.value
    assert list(a.stops) == list(b.stops)

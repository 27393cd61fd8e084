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


@pytest.mark.parametrize("case", L.cases(), ids=lambda c: c["name"])
def test_replay_fixture_on_the_gpu(engine, case):
    spec, lsm = L.plan(case)
    if case["risk"].get("delta"):
        pytest.skip("fixed-policy risk is priced by the oracle only")
    got = N.lsm_price(spec, lsm, stopping=True)
    want = H.oracle_lsm(spec, lsm, stopping=True, threads=4)
    assert_same_result(spec, lsm, got, want)
    e = case["expected"]
    assert list(got.stops) == e["stopping_indices"]
    assert list(got.counts[:len(spec.observation_times)]) == e["exercise_counts"]
    assert rel(got.result.price.value, e["value"]["value"]) <= PRICE_TOL
    assert rel(got.result.in_sample_value, e["in_sample_value"]) <= PRICE_TOL


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


def test_rejects_what_it_does_not_price(engine):
    spec, lsm = W.american_bs(dates=4, units=1 << 10)
    spec.request_delta = True
    with pytest.raises(N.EngineError) as err:
        N.lsm_price(spec, lsm)
    assert err.value.name == "unsupported"
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

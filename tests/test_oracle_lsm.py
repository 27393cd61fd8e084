"""The oracle's Longstaff--Schwartz evaluation against the reference's replay fixture.

fixtures/replay/early_exercise-windows-x86_64.json (extracted into
tests/golden/early_exercise.json) holds an American put under Black--Scholes
(S = K = 100, sigma = 0.2, r = 5 %, four quarterly exercise dates) priced with
a pseudo-MC engine (128 antithetic training units, 256 valuation units) and an
RQMC engine (64 x 4 training points, 128 x 4 valuation points).  The oracle
reproduces, to the last bit, the CPQR pivots and ranks of every fitted
decision model, the ITM row counts, the valuation
stopping index of every path, the exercise counts, the in-sample value, the
price with its standard error and confidence bounds, and the bits of the
sampling and estimator variances.  The feature scalings, |R| diagonals, rank
thresholds, coefficients and residual sums of squares agree within MODEL_TOL: the reference's own Windows and macOS
fixtures differ there by up to 4.5e-15 relative (their libm exp differs in the
last bit of some path spots), and so does the oracle under glibc.
"""
import ctypes as C
import struct

import numpy as np
import pytest

import helpers as H
import lsm_cases as L
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import workloads as W


def bits(x: float) -> str:
    return struct.pack(">d", x).hex()


CASES = L.cases()
MODEL_TOL = 5e-14


def close(got, want, tol=MODEL_TOL):
    return all(abs(a - b) <= tol * max(abs(b), 1e-300) for a, b in zip(got, want)) and len(got) == len(want)


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_replay_early_exercise(case):
    spec, lsm = L.plan(case)
    buf = H.oracle_lsm(spec, lsm, stopping=True, threads=3)
    r, e = buf.result, case["expected"]
    v = e["value"]
    assert r.price.value == v["value"]
    assert r.price.standard_error == v["standard_error"]
    assert r.price.confidence_lower == v["confidence_lower"]
    assert r.price.confidence_upper == v["confidence_upper"]
    assert r.price.effective_sampling_units == v["effective_sampling_units"]
    assert bits(r.sampling_variance) == e["sampling_variance_bits"]
    assert bits(r.estimator_variance) == e["estimator_variance_bits"]
    assert r.independent_sampling_units == e["independent_sampling_units"]
    assert r.valuation_paths == e["valuation_trajectories"] == e["evaluated_paths"]
    assert r.training_paths == e["training_trajectories"]
    assert r.in_sample_value == e["in_sample_value"]
    dates = len(spec.observation_times)
    assert list(buf.counts[:dates]) == e["exercise_counts"]
    assert list(buf.stops) == e["stopping_indices"]
    for k, (want, diag) in enumerate(zip(e["decision_models"], e["regression_diagnostics"])):
        m = buf.models[k]
        assert m.itm_rows == diag["itm_rows"]
        assert m.candidate_rows == diag["candidate_rows"]
        if want["type"] != "regression":
            assert m.regression == 0
            continue
        w = want["model"]
        sc = w["feature_scalings"][0]
        assert m.regression == 1
        assert close([m.feature_mean, m.feature_variance, m.feature_scale, m.zero_scale_threshold],
                     [sc["mean"], sc["population_variance"], sc["scale"], sc["zero_scale_threshold"]])
        assert bool(m.feature_inactive) == sc["inactive"]
        assert m.active_columns == len(w["active_basis_columns"])
        assert list(m.pivot_order[:m.active_columns]) == w["pivot_order"]
        assert close(list(m.diagonal_abs[:m.diagonal_count]), w["diagonal_abs"])
        assert m.rank == w["rank"]
        assert close([m.rank_threshold], [w["rank_threshold"]])
        assert close(list(m.coefficients[:lsm.max_degree + 1]), w["coefficients"])
        assert close([m.residual_sum_squares], [w["residual_sum_squares"]])


RISK_CASES = [c for c in CASES if c["risk"].get("delta")]


def check_risks(r, risks):
    """Raw delta, gamma and vega estimates of a fixed-policy risk replay, to the bit."""
    for name in ("delta", "gamma", "vega"):
        got, want = getattr(r, name), risks[name]["raw"]
        assert got.value == want["value"], name
        assert got.standard_error == want["standard_error"], name
        assert got.confidence_lower == want["confidence_lower"], name
        assert got.confidence_upper == want["confidence_upper"], name
        assert got.effective_sampling_units == want["effective_sampling_units"], name


@pytest.mark.parametrize("case", RISK_CASES, ids=lambda c: c["name"])
def test_replay_fixed_policy_risk(case):
    """Fixed-policy delta, gamma and vega of the American put
    (early_exercise.rs:454-600 over black_scholes.rs:358-415): the stopping
    dates of the valuation paths held, the discounted exercise value
    differentiated pathwise, gamma from deltas at S0 +- 1 % of spot."""
    spec, lsm = L.plan(case)
    buf = H.oracle_lsm(spec, lsm, stopping=True, threads=3)
    check_risks(buf.result, case["expected"]["risks"])
    # the price component of the risk pass re-derives the valuation price
    comp = buf.result.risk_components[A.PRICE]
    assert comp.sum + comp.correction == pytest.approx(
        buf.result.price.value * buf.result.independent_sampling_units, rel=1e-13)


@pytest.mark.parametrize("engine", [A.ENGINE_PSEUDO, A.ENGINE_RQMC], ids=["pseudo", "rqmc"])
def test_flat_local_volatility_is_black_scholes(engine):
    """write_local_vol_lsm_trajectory (early_exercise.rs:389-450) on a flat
    local-variance grid whose time grid is the exercise dates: the Log-Euler
    step of a constant variance is the exact lognormal step and draws the same
    normal per date, so every stopping date and exercise count equals the
    Black--Scholes engine's and the prices agree to rounding."""
    kw = dict(dates=12, units=1 << 12, engine=engine, antithetic=True)
    bs = H.oracle_lsm(*W.american_bs(vol=0.25, **kw), stopping=True, threads=4)
    lv = H.oracle_lsm(*W.american_lv(W.flat_grid(0.25), **kw), stopping=True, threads=4)
    assert list(lv.stops) == list(bs.stops)
    assert list(lv.counts[:12]) == list(bs.counts[:12])
    assert abs(lv.result.price.value - bs.result.price.value) <= 1e-13 * bs.result.price.value
    assert abs(lv.result.in_sample_value - bs.result.in_sample_value) <= 1e-13 * bs.result.in_sample_value


def test_flat_local_volatility_fixed_policy_risk_is_black_scholes():
    """local_vol_fixed_policy_pseudo_statistics_with_vega_kt (early_exercise.rs:465-700)
    on a flat local-variance grid: the reverse sweep's Vega (sum of the node
    sensitivities, seed at each path's stopping date) is the Black--Scholes
    pathwise Vega of fixed_policy_pathwise_values path by path, and the LV
    Delta/Gamma (central spot bumps on common paths) are the Black--Scholes
    bump-and-revalue validation components."""
    kw = dict(dates=12, units=1 << 12, antithetic=True)
    sb, lb = W.american_bs(vol=0.25, **kw)
    sb.request_delta = sb.request_gamma = sb.request_vega = True
    sl, ll = W.american_lv(W.flat_grid(0.25), **kw)
    sl.request_delta = sl.request_gamma = sl.request_vega = sl.request_local_vega_nodes = True
    bs = H.oracle_lsm(sb, lb, stopping=True, threads=4).result
    buf = H.oracle_lsm(sl, ll, stopping=True, threads=4)
    lv = buf.result
    assert abs(lv.vega.value - bs.vega.value) <= 1e-12 * abs(bs.vega.value)
    assert abs(lv.vega.standard_error - bs.vega.standard_error) <= 1e-10 * bs.vega.standard_error
    for mine, theirs in (("delta", "bump_delta"), ("gamma", "bump_gamma")):
        a, b = getattr(lv, mine), getattr(bs, theirs)
        assert abs(a.value - b.value) <= 1e-10 * max(abs(b.value), b.standard_error), mine
    nodes = np.array([e.value for e in buf.node_estimates])
    assert abs(nodes.sum() - lv.vega.value) <= 1e-12 * abs(lv.vega.value)


def test_thread_count_does_not_change_the_result():
    spec, lsm = L.plan(CASES[0])
    a = H.oracle_lsm(spec, lsm, stopping=True, threads=1)
    b = H.oracle_lsm(spec, lsm, stopping=True, threads=5)
    assert a.result.price.value == b.result.price.value
    assert list(a.stops) == list(b.stops)


def _fit(spots, immediate, targets, **kw):
    lib = H.oracle()
    lsm = L.LsmSpec(training_seed=0, training_units=1, **kw)
    ld = lsm.desc()
    m = A.LsmDateModel()
    n = len(spots)
    s, i, t = (np.ascontiguousarray(x, dtype=np.float64) for x in (spots, immediate, targets))
    rc = lib.oracle_lsm_fit(H.dptr(s), H.dptr(i), H.dptr(t), n, C.byref(ld), C.byref(m))
    return rc, m


def test_no_itm_rows_continue_all():
    rc, m = _fit([100.0, 101.0], [0.0, 0.0], [1.0, 2.0])
    assert rc == 0 and m.regression == 0 and m.itm_rows == 0


def test_single_itm_row_inactive_feature_constant_fit():
    # One ITM row: zero variance, the feature is inactive and only z^0 is fitted
    # (fit_polynomial_regression pre-excludes every column of an inactive feature).
    rc, m = _fit([90.0, 110.0], [10.0, 0.0], [7.5, 3.0])
    assert rc == 0 and m.regression == 1 and m.feature_inactive == 1
    assert m.active_columns == 1 and m.rank == 1 and m.diagonal_count == 1
    assert m.coefficients[0] == 7.5 and list(m.coefficients[1:4]) == [0.0, 0.0, 0.0]


def test_fewer_rows_than_columns_caps_the_rank():
    # Two ITM rows of a cubic basis: CPQR stops after min(rows, columns) = 2 pivots.
    rc, m = _fit([90.0, 95.0, 120.0], [10.0, 5.0, 0.0], [12.0, 6.0, 0.0])
    assert rc == 0 and m.diagonal_count == 2 and m.rank == 2
    z = np.array([-1.0, 1.0])   # standardised spots of the two rows
    c = np.array(m.coefficients[:4])
    pred = sum(c[k] * z ** k for k in range(4))
    assert np.allclose(pred, [12.0, 6.0], rtol=0, atol=1e-12)


def test_matrix_limit_is_enforced():
    rc, _ = _fit(np.linspace(80, 99, 300), np.full(300, 1.0), np.ones(300), max_matrix_elements=1000)
    assert rc == 12  # MCG_ERR_LSM: a 300 x 4 design exceeds 1000 elements

"""The oracle against the reference's fixtures (golden vectors in tests/golden/).

* Replay: the European BS pseudo-MC and RQMC full-risk cases of
  fixtures/replay/european_bs-windows-x86_64.json reproduce value, standard
  error, Delta, Gamma and Vega, and the bits of the sampling variance.
* Path dependence: compact-C2 smoothing, smooth extrema and the exact and
  smoothed bridge survival match the independent high-precision cases of
  fixtures/path-dependence/reference-cases-v0.1.json.
* Local volatility: the pseudo-MC and RQMC cases of
  fixtures/replay/local_volatility-*.json (3 x 5 grid, price-only and
  Delta/Gamma/Vega) reproduce price, standard error and variance bits.
* Analytic: the closed-form benchmark reproduces fixtures/acceptance/european_bs_analytical.csv.
"""
import ctypes as C
import json
import math
import os
import struct

import numpy as np
import pytest

import helpers as H
import lv_cases as L
from bs_closed_form import black_scholes
from rust_pricing_b200 import _abi as A
from rust_pricing_b200.desc import PlanSpec, ProductSpec

GOLDEN = H.GOLDEN


def bits(x: float) -> str:
    return struct.pack(">d", x).hex()


def replay_spec(case: dict) -> PlanSpec:
    """The compiled plan of one replay request (valuation 2026-09-04, expiry 2027-09-04: T = 1)."""
    rqmc = case["engine"] == "randomized_quasi_monte_carlo"
    return PlanSpec(
        observation_times=[1.0], products=[ProductSpec(kind=A.PRODUCT_EUROPEAN, strike=case["strike"])],
        engine=A.ENGINE_RQMC if rqmc else A.ENGINE_PSEUDO, master_seed=case["master_seed"],
        sampling_units=case["sampling_units"], scramble_count=case["scramble_count"] or 16,
        antithetic=case["antithetic"], brownian_bridge=case["brownian_bridge"],
        reduction_block_size=case["reduction_block_size"], spot=case["spot"],
        discount_times=case["discount_curve"]["times"], discount_factors=case["discount_curve"]["discount_factors"],
        dividend_times=case["dividend_curve"]["times"], dividend_factors=case["dividend_curve"]["discount_factors"],
        volatility=case["volatility"], request_delta=True, request_gamma=True, request_vega=True,
        gamma_bump=case["gamma_bump_relative"])


def replay_cases():
    return json.load(open(os.path.join(GOLDEN, "replay_european_bs.json")))["cases"]


@pytest.mark.parametrize("case", replay_cases(), ids=lambda c: c["name"])
def test_replay_european_bs(case):
    r = H.oracle_evaluate(replay_spec(case), threads=4)
    p = r.products[0]
    e = case["expected"]
    # Every estimate agrees to the last bit with the reference on Windows/macOS.
    assert p.price.value == e["price"]
    assert p.price.standard_error == e["price_standard_error"]
    assert p.delta.value == e["delta"]
    assert p.delta.standard_error == e["delta_standard_error"]
    assert p.gamma.value == e["gamma"]
    assert p.gamma.standard_error == e["gamma_standard_error"]
    assert p.vega.value == e["vega"]
    assert p.vega.standard_error == e["vega_standard_error"]
    assert bits(p.sampling_variance) == e["sampling_variance_bits"]
    assert bits(p.estimator_variance) == e["estimator_variance_bits"]
    # CRN validation bumps differ only in low bits across platforms' libm.
    for key, est in (("bump_delta_value_bits", p.bump_delta), ("bump_gamma_value_bits", p.bump_gamma),
                     ("bump_vega_value_bits", p.bump_vega)):
        expected = struct.unpack(">d", bytes.fromhex(e[key]))[0]
        assert abs(est.value - expected) <= 1e-9 * abs(expected)


LV_CASES = L.cases()


def ulps(a: float, b: float) -> int:
    """Distance in units in the last place between two finite doubles of one sign."""
    ia, ib = (struct.unpack(">q", struct.pack(">d", x))[0] for x in (a, b))
    return abs(ia - ib)


def nearest_ulps(got: float, wants) -> int:
    return min(ulps(got, w) for w in wants)


@pytest.mark.parametrize("case", LV_CASES, ids=lambda c: c["name"])
def test_replay_local_volatility(case):
    """Log-Euler local volatility against both platforms' fixtures.  The price
    and the Delta/Vega values equal a platform's to the last bit; standard
    errors and variances are within 2 ulps and Gamma within 4 ulps of the
    nearer platform, or inside the two platforms' own spread where that is
    wider (their libm exp/log differ in the last bit of some paths; the RQMC
    Gamma standard error of the two fixtures differs by 250 ulps)."""
    r = H.oracle_evaluate(L.plan(case), threads=4)
    p = r.products[0]
    plats = list(case["expected"].values())
    assert r.result.evaluated_paths == plats[0]["evaluated_paths"]
    assert nearest_ulps(p.price.value, [e["value"]["value"] for e in plats]) == 0
    for f in ("standard_error", "confidence_lower", "confidence_upper"):
        assert nearest_ulps(getattr(p.price, f), [e["value"][f] for e in plats]) <= 2, f
    assert p.price.effective_sampling_units == plats[0]["value"]["effective_sampling_units"]
    for name, key in (("sampling_variance", "sampling_variance_bits"),
                      ("estimator_variance", "estimator_variance_bits")):
        want = [struct.unpack(">d", bytes.fromhex(e[key]))[0] for e in plats]
        assert nearest_ulps(getattr(p, name), want) <= 2, name
    for name in plats[0]["risks"]:
        got = getattr(p, name)
        assert nearest_ulps(got.value, [e["risks"][name]["value"] for e in plats]) <= (4 if name == "gamma" else 0), name
        ses = [e["risks"][name]["standard_error"] for e in plats]
        spread = max(ses) - min(ses)  # 250 ulps for the RQMC Gamma (8 scramble means)
        assert nearest_ulps(got.standard_error, ses) <= 2 or \
            min(ses) - spread <= got.standard_error <= max(ses) + spread, name
        assert got.effective_sampling_units == plats[0]["risks"][name]["effective_sampling_units"]


VEGA_KT_CASES = [c for c in LV_CASES if "node_allocation" in c]


def node_means(buf):
    return np.array([e.value for e in buf.node_estimates])


@pytest.mark.parametrize("case", VEGA_KT_CASES, ids=lambda c: c["name"])
def test_vega_kt_node_allocation(case):
    """allocate_local_vol_nodes over the local-vega node sensitivities of the
    LV replay risk cases, against the node-allocation audit fixture
    (fixtures/replay/local-vol-node-allocation-change-audit-v1.json): raw
    buckets, scalar VegaKT, the residual outside the active density domain and
    the left-edge statistics.  The oracle projects the node means (the
    projection is linear; the reference projects every path and averages), so
    agreement is to rounding, 1e-13; the engine's host projection of the same
    means gives the same numbers."""
    spec = L.plan(case)
    spec.request_local_vega_nodes = True
    buf = H.oracle_evaluate(spec, threads=4)
    means = node_means(buf)
    paths = buf.result.evaluated_paths
    out, buckets = L.oracle_vega_kt(case, means, paths)
    L.check_node_allocation(out, buckets, case["node_allocation"], 1e-13)
    # reconciliation: buckets + residual (excluded nodes and the initial-time row) = scalar local Vega
    assert abs(out.scalar_vega + out.signed_residual - out.pre_projection) <= 1e-12 * abs(out.pre_projection)
    assert out.signed_residual == out.initial_time + out.density_excluded
    assert abs(out.pre_projection - buf.products[0].vega.value) <= 1e-12 * abs(buf.products[0].vega.value)
    from rust_pricing_b200 import _native as N
    g = case["local_variance_grid"]
    eng, eb = N.vega_kt_project(g["time_nodes"], g["log_forward_moneyness_nodes"], means, paths, L.vega_kt_basis(case))
    assert list(eb) == list(buckets)
    for f in ("scalar_vega", "signed_residual", "density_excluded", "initial_time", "left_edge_sensitivity",
              "left_edge_count"):
        assert getattr(eng, f) == getattr(out, f), f


def test_vega_kt_rejects_a_grid_time_without_a_density_row():
    from rust_pricing_b200 import _native as N
    case = VEGA_KT_CASES[0]
    g = case["local_variance_grid"]
    times = [0.0, 0.5, 1.0]   # 0.5 is not a reporting maturity
    with pytest.raises(N.EngineError) as err:
        N.vega_kt_project(times, g["log_forward_moneyness_nodes"], np.ones(15), 10, L.vega_kt_basis(case))
    assert err.value.name == "invalid_argument"


def test_replay_independent_of_thread_count():
    case = replay_cases()[0]
    a = H.oracle_evaluate(replay_spec(case), threads=1).products[0]
    b = H.oracle_evaluate(replay_spec(case), threads=7).products[0]
    for f in ("price", "delta", "gamma", "vega"):
        assert getattr(a, f).value == getattr(b, f).value


def test_closed_form_benchmark_matches_analytical_grid():
    rows = json.load(open(os.path.join(GOLDEN, "bs_analytical.json")))["rows"]
    for row in rows:
        spot, t = 100.0, float(row["time"])
        r, q, vol = float(row["rate"]), float(row["dividend_yield"]), float(row["volatility"])
        forward = spot * math.exp((r - q) * t)
        strike = float(row["moneyness"]) * forward
        got = black_scholes(row["side"] == "call", spot, strike, t, r, q, vol)
        for key, tol in (("price", 5e-13), ("delta", 5e-14), ("gamma", 5e-15), ("vega", 5e-13)):
            expected = float(row[key])
            assert abs(got[key] - expected) <= tol * max(1.0, abs(expected)), (row["case"], key)


def _pd():
    return json.load(open(os.path.join(GOLDEN, "path_dependence.json")))


@pytest.mark.parametrize("case", _pd()["smoothing_cases"], ids=lambda c: c["id"])
def test_smoothing_reference_cases(oracle, case):
    out = np.zeros(6)
    oracle.oracle_smoothing(float(case["half_width"]), float(case["input"]), H.dptr(out))
    keys = ["indicator", "indicator_first", "indicator_second", "positive_part",
            "positive_part_first", "positive_part_second"]
    for k, v in zip(keys, out):
        exp = float(case["expected"][k])
        assert abs(v - exp) <= 4e-15 * max(1.0, abs(exp)), k


@pytest.mark.parametrize("case", _pd()["extrema_cases"], ids=lambda c: c["id"])
def test_smooth_extrema_reference_cases(oracle, case):
    out = np.zeros(2)
    oracle.oracle_smooth_extrema(float(case["half_width"]), float(case["left"]), float(case["right"]), H.dptr(out))
    assert abs(out[0] - float(case["expected"]["maximum"])) <= 1e-13
    assert abs(out[1] - float(case["expected"]["minimum"])) <= 1e-13


@pytest.mark.parametrize("case", _pd()["bridge_cases"], ids=lambda c: c["id"])
def test_bridge_reference_cases(oracle, case):
    surv = C.c_double()
    rc = oracle.oracle_exact_bridge(int(case["direction"] == "up"), float(case["barrier"]),
                                    float(case["start_spot"]), float(case["end_spot"]),
                                    float(case["integrated_variance"]), C.byref(surv))
    assert rc == 0
    exp = float(case["expected"]["survival_probability"])
    assert abs(surv.value - exp) <= 1e-14 * max(1.0, exp)


@pytest.mark.parametrize("case", _pd()["smoothed_bridge_cases"], ids=lambda c: c["id"])
def test_smoothed_bridge_reference_cases(oracle, case):
    out = np.zeros(6)
    rc = oracle.oracle_smoothed_bridge(int(case["direction"] == "up"), float(case["barrier"]),
                                       float(case["start_spot"]), float(case["end_spot"]),
                                       float(case["half_width"]), float(case["integrated_variance"]), H.dptr(out))
    assert rc == 0
    e = case["expected"]
    for k, v in zip(["start_hit_weight", "end_hit_weight", "start_effective_log_distance",
                     "end_effective_log_distance", "bridge_survival", "endpoint_survival"], out):
        exp = float(e[k])
        assert abs(v - exp) <= 1e-13 * max(1.0, abs(exp)), k

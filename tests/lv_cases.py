"""Local-volatility plans of the reference's replay fixture (tests/golden/replay_local_vol.json).

fixtures/replay/local_volatility-{windows-x86_64,macos-aarch64}.json hold a
European call under a 3 x 5 local-variance grid (S = K = 100, discount and
dividend curves log-linear to one year, grid floor 1e-8, cap 4) priced with a
pseudo-MC engine (8192 antithetic units, no bridge) and an RQMC engine
(512 points x 8 scrambles, antithetic, Brownian bridge), price-only and with
Delta (CRN central bump), Gamma (CRN, 1 % relative bump) and Vega (reverse
sweep, the sum of the local-variance node adjoints).
"""
import ctypes as C
import datetime as dt
import json
import math
import os

import numpy as np

import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200.desc import LocalVarianceSpec, PlanSpec, ProductSpec


def cases():
    return json.load(open(os.path.join(H.GOLDEN, "replay_local_vol.json")))["cases"]


def act365(valuation: str, date: str) -> float:
    """DayCountConvention::Act365F.year_fraction (crates/pricing/src/core)."""
    return (dt.date.fromisoformat(date) - dt.date.fromisoformat(valuation)).days / 365.0


def plan(case: dict) -> PlanSpec:
    g = case["local_variance_grid"]
    risk = case["risk"]
    spec = PlanSpec(
        observation_times=[act365(case["valuation_date"], case["product"]["expiry"])],
        products=[ProductSpec(kind=A.PRODUCT_EUROPEAN, side=A.CALL if case["side"] == "call" else A.PUT,
                              strike=case["product"]["strike"], notional=case["product"]["notional"])],
        model=A.MODEL_LOCAL_VOLATILITY,
        engine=A.ENGINE_RQMC if case["engine"] == "rqmc" else A.ENGINE_PSEUDO,
        master_seed=case["master_seed"], sampling_units=case["sampling_units"],
        scramble_count=case["scramble_count"] or 0, antithetic=case["antithetic"],
        brownian_bridge=case["brownian_bridge"], reduction_block_size=case["reduction_block_size"],
        spot=case["spot"],
        discount_times=case["discount_curve"]["times"], discount_factors=case["discount_curve"]["discount_factors"],
        dividend_times=case["dividend_curve"]["times"], dividend_factors=case["dividend_curve"]["discount_factors"],
        local_variance=LocalVarianceSpec(g["time_nodes"], g["log_forward_moneyness_nodes"], g["values"],
                                         g["floor"], g["cap"]),
        request_delta=bool(risk.get("delta")), request_vega=bool(risk.get("vega")),
        request_gamma=bool(risk.get("gamma")))
    if risk.get("gamma"):
        bump = risk["gamma"]["bump"]
        spec.gamma_bump_relative = bump["type"] == "relative"
        spec.gamma_bump = bump["value"]
    return spec


def _log_df(curve: dict, t: float) -> float:
    """LogLinearDiscountCurve at t (pillars given; linear in log DF, flat log slope beyond)."""
    ts, dfs = curve["times"], curve["discount_factors"]
    for i in range(len(ts) - 1):
        if t <= ts[i + 1] or i == len(ts) - 2:
            w = (t - ts[i]) / (ts[i + 1] - ts[i])
            return math.log(dfs[i]) + w * (math.log(dfs[i + 1]) - math.log(dfs[i]))
    return math.log(dfs[-1])


def vega_kt_basis(case: dict):
    """The request's reporting-IV basis and VegaKT config, with the market
    forwards at the reporting maturities."""
    from rust_pricing_b200._native import VegaKtBasisSpec
    kt = case["vega_kt"]
    rb = kt["reporting_iv_basis"]
    forwards = [case["spot"] * math.exp(_log_df(case["dividend_curve"], t) - _log_df(case["discount_curve"], t))
                for t in rb["maturity_nodes"]]
    return VegaKtBasisSpec(rb["maturity_nodes"], rb["log_forward_moneyness_nodes"], rb["implied_volatilities"],
                           forwards, kt["config"]["relative_density_threshold"])


def oracle_vega_kt(case: dict, node_means, evaluated_paths: int):
    """The oracle's node allocation of given node-sensitivity means."""
    from rust_pricing_b200 import _abi as A
    g = case["local_variance_grid"]
    tn = np.ascontiguousarray(g["time_nodes"], dtype=np.float64)
    xn = np.ascontiguousarray(g["log_forward_moneyness_nodes"], dtype=np.float64)
    nodes = np.ascontiguousarray(node_means, dtype=np.float64).ravel()
    basis = vega_kt_basis(case)
    out = A.VegaKtProjection()
    buckets = np.zeros(basis.buckets())
    out.bucket_capacity = len(buckets)
    out.raw_buckets = H.dptr(buckets)
    b = basis.desc()
    rc = H.oracle().oracle_vega_kt_project(H.dptr(tn), len(tn), H.dptr(xn), len(xn), H.dptr(nodes), evaluated_paths,
                                           C.byref(b), C.byref(out))
    assert rc == 0, rc
    return out, buckets


def check_node_allocation(out, buckets, want: dict, rel: float):
    """The audit fixture's node-allocation values."""
    def close(a, b):
        return abs(a - b) <= rel * max(abs(b), 1.0)
    assert close(buckets[0], want["raw_buckets/0"]), (buckets[0], want["raw_buckets/0"])
    assert close(buckets[1], want["raw_buckets/1"]), (buckets[1], want["raw_buckets/1"])
    assert all(abs(v) <= rel for v in buckets[2:])
    assert close(out.scalar_vega, want["projection/scalar_vega"])
    assert close(out.signed_residual, want["projection/signed_residual"])
    assert close(out.left_edge_sensitivity, want["projection/reporting_stats/left_edge_sensitivity"])
    assert out.left_edge_count == want["projection/reporting_stats/left_edge_count"]

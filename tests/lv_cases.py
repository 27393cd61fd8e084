"""Local-volatility plans of the reference's replay fixture (tests/golden/replay_local_vol.json).

fixtures/replay/local_volatility-{windows-x86_64,macos-aarch64}.json hold a
European call under a 3 x 5 local-variance grid (S = K = 100, discount and
dividend curves log-linear to one year, grid floor 1e-8, cap 4) priced with a
pseudo-MC engine (8192 antithetic units, no bridge) and an RQMC engine
(512 points x 8 scrambles, antithetic, Brownian bridge), price-only and with
Delta (CRN central bump), Gamma (CRN, 1 % relative bump) and Vega (reverse
sweep, the sum of the local-variance node adjoints).
"""
import datetime as dt
import json
import os

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

"""Early-exercise plans of the reference's replay fixture (tests/golden/early_exercise.json)."""
import datetime as dt
import json
import os

import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200.desc import LsmSpec, PlanSpec, ProductSpec


def cases():
    return json.load(open(os.path.join(H.GOLDEN, "early_exercise.json")))["cases"]


def act365(valuation: str, date: str) -> float:
    """DayCountConvention::Act365F.year_fraction (crates/pricing/src/core)."""
    a, b = dt.date.fromisoformat(valuation), dt.date.fromisoformat(date)
    return (b - a).days / 365.0


def _engine_kwargs(e: dict) -> dict:
    rqmc = e["engine"] == "rqmc"
    return dict(engine=A.ENGINE_RQMC if rqmc else A.ENGINE_PSEUDO, master_seed=e["master_seed"],
                sampling_units=e["sampling_units"], scramble_count=e["scramble_count"] or 0,
                antithetic=e["antithetic"], brownian_bridge=e["brownian_bridge"])


def _risk_kwargs(r: dict) -> dict:
    """Risk requests of a replay case: delta/vega flags and the gamma bump."""
    kw = dict(request_delta=bool(r.get("delta")), request_vega=bool(r.get("vega")))
    g = r.get("gamma")
    if g:
        bump = g["bump"]
        kw.update(request_gamma=True, gamma_bump_relative=bump["type"] == "relative", gamma_bump=bump["value"])
    return kw


def plan(case: dict) -> tuple[PlanSpec, LsmSpec]:
    """The compiled American plan and LSM configuration of one replay request."""
    times = [act365(case["valuation_date"], d) for d in case["product"]["exercise_dates"]]
    side = A.PUT if case["side"] == "put" else A.CALL
    spec = PlanSpec(
        observation_times=times,
        products=[ProductSpec(kind=A.PRODUCT_AMERICAN, side=side, strike=case["product"]["strike"],
                              notional=case["product"]["notional"])],
        reduction_block_size=case["reduction_block_size"], spot=case["spot"],
        discount_times=case["discount_curve"]["times"], discount_factors=case["discount_curve"]["discount_factors"],
        dividend_times=case["dividend_curve"]["times"], dividend_factors=case["dividend_curve"]["discount_factors"],
        volatility=case["volatility"], **_engine_kwargs(case["valuation"]), **_risk_kwargs(case["risk"]))
    t = case["training"]
    cfg = case["lsm"]
    lsm = LsmSpec(training_seed=t["master_seed"], training_units=t["sampling_units"],
                  training_scramble_count=t["scramble_count"] or 0, training_antithetic=t["antithetic"],
                  training_brownian_bridge=t["brownian_bridge"], max_degree=cfg["max_degree"],
                  itm_abs_tolerance=cfg["itm_abs_tolerance"], cpqr_abs_tolerance=cfg["cpqr_abs_tolerance"],
                  cpqr_rel_tolerance=cfg["cpqr_rel_tolerance"], max_matrix_elements=cfg["max_matrix_elements"])
    return spec, lsm

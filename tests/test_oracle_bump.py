"""The oracle's bump-and-revalue restatement against the reference's acceptance checks.

* crates/pricing/src/engine/risk/bump.rs:986-1012: under local volatility a
  spot-Delta bump of relative size 1e-6 agrees with the native Delta within the
  combined standard errors, pseudo-MC (4096 units) and RQMC (128 x 16,
  antithetic, bridge).
* With the native CRN half-width (the gamma bump) the bump-plan Delta and Gamma
  are the native local-volatility Delta and Gamma: the same per-unit
  differences, so equal to rounding.
* Black--Scholes: bump Delta, Gamma and Vega agree with the pathwise Delta,
  bumped-AAD Gamma and pathwise Vega within the combined errors.
* Scenarios: Delta and Gamma of one size share one pair (bump_cost: two side
  evaluations plus the base for Gamma), bump.rs:446-488.
"""
import math

import pytest

import bump_cases as B
import helpers as H
from rust_pricing_b200 import _abi as A

SPOT = (A.BUMP_SPOT_DELTA, 1e-6, True)


def within(bump, value, se):
    gap = abs(bump.value - value)
    assert bump.standard_error > 0.0 and se > 0.0
    assert gap <= math.hypot(bump.standard_error, se), (bump.value, value, gap)


@pytest.mark.parametrize("engine", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
def test_local_volatility_bump_agrees_with_native_delta(engine):
    spec = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, engine)
    (d,), rep = H.oracle_bump(spec, [SPOT])
    want = H.oracle_evaluate(B.native(spec, request_delta=True)).products[0].delta
    within(d, want.value, want.standard_error)
    assert rep.evaluations == 2 and rep.scenarios == 1
    assert d.units == (16 if engine == A.ENGINE_RQMC else 4096)


@pytest.mark.parametrize("engine", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
def test_native_half_width_gives_the_native_crn_greeks(engine):
    spec = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, engine, antithetic=True)
    est, rep = H.oracle_bump(spec, [(A.BUMP_SPOT_DELTA, 0.01, True), (A.BUMP_SPOT_GAMMA, 0.01, True)])
    nat = H.oracle_evaluate(B.native(spec, request_delta=True, request_gamma=True)).products[0]
    for got, want in ((est[0], nat.delta), (est[1], nat.gamma)):
        assert abs(got.value - want.value) <= 1e-12 * abs(want.value), (got.value, want.value)
        assert abs(got.standard_error - want.standard_error) <= 1e-9 * want.standard_error
    assert rep.scenarios == 1 and rep.evaluations == 3
    assert est[0].amount == 1.0 and est[0].scenario == est[1].scenario == 0


@pytest.mark.parametrize("steps", [1, 12])
def test_black_scholes_bumps_agree_with_pathwise_risk(steps):
    prod = None if steps == 1 else A.PRODUCT_ASIAN
    from rust_pricing_b200.desc import ProductSpec
    product = None if prod is None else ProductSpec(kind=A.PRODUCT_ASIAN, strike=100.0, weights=[1.0 / steps] * steps)
    spec = B.fixture_plan(units=1 << 15, product=product, steps=steps, antithetic=True)
    est, rep = H.oracle_bump(spec, [(A.BUMP_SPOT_DELTA, 1e-4, True), (A.BUMP_SPOT_GAMMA, 0.01, True),
                                    (A.BUMP_VOLATILITY_VEGA, 1e-4, False)])
    nat = H.oracle_evaluate(B.native(spec, request_delta=True, request_gamma=True, request_vega=True)).products[0]
    within(est[0], nat.delta.value, nat.delta.standard_error)
    within(est[1], nat.gamma.value, nat.gamma.standard_error)
    within(est[2], nat.vega.value, nat.vega.standard_error)
    assert rep.scenarios == 3 and rep.evaluations == 7
    assert abs(rep.base_price.value - nat.price.value) <= 1e-12 * nat.price.value


def test_shared_scenarios_are_counted_once():
    spec = B.fixture_plan(units=512)
    est, rep = H.oracle_bump(spec, [(A.BUMP_SPOT_DELTA, 0.01, True), (A.BUMP_SPOT_DELTA, 1.0, False),
                                    (A.BUMP_SPOT_GAMMA, 1.0, False), (A.BUMP_SPOT_DELTA, 2.0, False)])
    assert [e.scenario for e in est] == [0, 0, 0, 1]
    assert est[0].value == est[1].value
    assert rep.scenarios == 2 and rep.evaluations == 5


def test_volatility_bump_needs_a_constant_volatility():
    spec = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, units=256)
    with pytest.raises(RuntimeError):
        H.oracle_bump(spec, [(A.BUMP_VOLATILITY_VEGA, 1e-4, False)])

"""Bump-and-revalue on the GPU (mcg_bump_evaluate): every side in one launch.

* Engine vs oracle on identical draws: each paired estimate within 1e-12 of
  its scale and its standard error within 1e-10, the side prices within
  1e-12 -- Black--Scholes single-terminal and path (Asian) plans, local
  volatility pseudo-MC (with and without antithetic pairs) and RQMC with the
  bridge, spot and volatility scenarios, shared pairs.
* The reference's acceptance check (crates/pricing/src/engine/risk/bump.rs:986-1012): the
  local-volatility bump Delta at relative size 1e-6 agrees with the native
  Delta within the combined standard errors.
* At the native CRN half-width the bump Delta and Gamma equal the engine's own
  local-volatility Delta and Gamma to rounding.
* One launch prices all sides: kernel_launches is the scenario grid, its tile
  reduction and (pseudo-MC) the pairing kernel with its reduction.
"""
import math

import pytest

import bump_cases as B
import gpu_common as G
import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200.desc import ProductSpec

pytestmark = pytest.mark.gpu

REQUESTS = [(A.BUMP_SPOT_DELTA, 1e-4, True), (A.BUMP_SPOT_GAMMA, 0.01, True), (A.BUMP_SPOT_DELTA, 1.0, False)]


def assert_same(spec, requests):
    got, grep = N.bump_evaluate(spec, requests)
    want, wrep = H.oracle_bump(spec, requests)
    for g, w in zip(got, want):
        scale = max(abs(w.value), w.standard_error)
        assert abs(g.value - w.value) <= G.DIRECT_TOL * scale, (g.value, w.value)
        assert abs(g.standard_error - w.standard_error) <= 1e-10 * w.standard_error
        assert g.units == w.units and g.scenario == w.scenario and g.amount == w.amount
        for a, b in ((g.up_price, w.up_price), (g.down_price, w.down_price)):
            assert abs(a - b) <= G.DIRECT_TOL * max(abs(b), 1e-300)
    assert (grep.scenarios, grep.sides, grep.evaluations) == (wrep.scenarios, wrep.sides, wrep.evaluations)
    rqmc = spec.engine == A.ENGINE_RQMC
    assert grep.kernel_launches == (2 if rqmc else 4)
    return got, grep


@pytest.mark.parametrize("steps", [1, 12])
@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
def test_black_scholes_matches_the_oracle(engine, steps, engine_kind):
    product = None if steps == 1 else ProductSpec(kind=A.PRODUCT_ASIAN, strike=100.0, weights=[1.0 / steps] * steps)
    spec = B.fixture_plan(engine=engine_kind, units=4099, product=product, steps=steps)
    assert_same(spec, REQUESTS + [(A.BUMP_VOLATILITY_VEGA, 1e-4, False)])


@pytest.mark.parametrize("engine_kind,antithetic", [(A.ENGINE_PSEUDO, False), (A.ENGINE_PSEUDO, True),
                                                    (A.ENGINE_RQMC, True)])
def test_local_volatility_matches_the_oracle(engine, engine_kind, antithetic):
    spec = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, engine_kind, units=3001, antithetic=antithetic, steps=4)
    assert_same(spec, REQUESTS)


def test_ssvi_local_volatility_barrier_matches_the_oracle(engine):
    from rust_pricing_b200 import workloads as W
    grid = W.local_vol_grid(W.SsviSurface(steps=12, expiries=12), G.gpu_grid)
    spec = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, units=2048, steps=12,
                          product=ProductSpec(kind=A.PRODUCT_CONTINUOUS_BARRIER, strike=100.0, barrier=80.0,
                                              barrier_direction=A.BARRIER_DOWN, rebate=1.0))
    spec.local_variance = grid
    spec.smoothing_half_width = 0.5
    assert_same(spec, REQUESTS)


@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
def test_local_volatility_bump_agrees_with_native_delta(engine, engine_kind):
    spec = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, engine_kind)
    (d,), _ = N.bump_evaluate(spec, [(A.BUMP_SPOT_DELTA, 1e-6, True)])
    want = G.run_engine(B.native(spec, request_delta=True)).products[0].delta
    assert math.fabs(d.value - want.value) <= math.hypot(d.standard_error, want.standard_error)


@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
def test_native_half_width_gives_the_engines_crn_greeks(engine, engine_kind):
    spec = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, engine_kind, antithetic=True, units=1 << 16)
    est, rep = N.bump_evaluate(spec, [(A.BUMP_SPOT_DELTA, 0.01, True), (A.BUMP_SPOT_GAMMA, 0.01, True)])
    nat = G.run_engine(B.native(spec, request_delta=True, request_gamma=True)).products[0]
    for got, want in ((est[0], nat.delta), (est[1], nat.gamma)):
        assert abs(got.value - want.value) <= 1e-12 * abs(want.value), (got.value, want.value)
        assert abs(got.standard_error - want.standard_error) <= 1e-9 * want.standard_error
    assert abs(rep.base_price.value - nat.price.value) <= 1e-12 * nat.price.value


def test_rejections(engine):
    lv = B.fixture_plan(A.MODEL_LOCAL_VOLATILITY, units=256)
    with pytest.raises(N.EngineError) as err:
        N.bump_evaluate(lv, [(A.BUMP_VOLATILITY_VEGA, 1e-4, False)])
    assert err.value.name == "invalid_argument"
    with pytest.raises(N.EngineError) as err:
        N.bump_evaluate(B.fixture_plan(units=256), [(A.BUMP_SPOT_DELTA, 200.0, False)])  # spot - h < 0
    assert err.value.name == "invalid_argument"
    risky = B.native(B.fixture_plan(units=256), request_delta=True)
    with pytest.raises(N.EngineError) as err:
        N.bump_evaluate(risky, [(A.BUMP_SPOT_DELTA, 1e-4, True)])
    assert err.value.name == "unsupported"

"""Discrete dividends (escrowed affine model) on the GPU.

* The reference's own acceptance checks (crates/pricing/tests/affine_oracles.rs:131-230):
  zero-volatility terminal spots exactly, and the escrowed-spot closed form for
  a cash-and-proportional dividend (price, Delta, Vega, Gamma within 4.5 SE).
* Engine vs oracle on identical draws, within the parity tolerances
  (gpu_common): Black--Scholes European (single terminal, risk), Asian,
  lookback, digital and discrete barriers (exact and smoothed, with a
  dividend on a monitoring date, where the barrier also sees the spot before
  the dividend), price and full pathwise risk, pseudo-MC and RQMC; local
  volatility with the ex-dates added to the time grid, price and CRN
  Delta/Gamma, pseudo and RQMC with the Brownian bridge.
* The combinations left out (continuous barrier, early exercise, local
  Vega) are refused as unsupported.
"""
import pytest

import dividend_cases as D
import gpu_common as G
import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W
from rust_pricing_b200.desc import ProductSpec

pytestmark = pytest.mark.gpu

DIVS = [(0.25, 1.5, 0.0), (0.5, 0.0, 0.02), (0.75, 1.0, 0.01)]  # 0.25, 0.5, 0.75: monitoring dates


@pytest.mark.parametrize("case", D.DETERMINISTIC, ids=lambda c: f"t{c[0]}-cash{c[1]}-beta{c[2]}")
@pytest.mark.parametrize("side", [A.CALL, A.PUT])
def test_zero_volatility_dividends_leave_the_known_terminal_spot(engine, case, side):
    t, cash, beta, terminal = case
    spec = D.european(side, [(t, cash, beta)], vol=0.0, rate=0.0, repo=0.0, units=256)
    p = G.run_engine(spec).products[0]
    sign = 1.0 if side == A.CALL else -1.0
    assert abs(p.price.value - max(sign * (terminal - D.STRIKE), 0.0)) <= 1e-12


@pytest.mark.parametrize("side", [A.CALL, A.PUT])
def test_mixed_dividend_is_black_scholes_on_the_escrowed_spot(engine, side):
    spec = D.european(side, [(0.5, 20.0, 0.1)], units=1 << 20, risk=True)
    p = G.run_engine(spec).products[0]
    want = D.escrowed_reference(side)
    for key in ("price", "delta", "vega", "gamma"):
        est = getattr(p, key)
        assert abs(est.value - want[key]) <= 4.5 * est.standard_error, (key, est.value, want[key])


@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
@pytest.mark.parametrize("side", [A.CALL, A.PUT])
def test_european_with_dividends_matches_the_oracle(engine, engine_kind, side):
    spec = D.european(side, [(0.5, 20.0, 0.1), (0.9, 3.0, 0.0)], units=4096 if engine_kind == A.ENGINE_RQMC else 20001,
                      engine=engine_kind, risk=True)
    G.assert_parity(spec)


def _barrier(smooth_kind, up):
    return ProductSpec(kind=A.PRODUCT_DISCRETE_BARRIER, strike=95.0, barrier=110.0 if up else 85.0,
                       barrier_direction=A.BARRIER_UP if up else A.BARRIER_DOWN, barrier_style=smooth_kind,
                       rebate=1.0)


PATH_PRODUCTS = {
    "asian": ProductSpec(kind=A.PRODUCT_ASIAN, strike=95.0, weights=[1.0 / 12] * 12),
    "lookback-put": ProductSpec(kind=A.PRODUCT_LOOKBACK, side=A.PUT, strike=100.0),
    "digital": ProductSpec(kind=A.PRODUCT_DIGITAL, strike=95.0),
    "up-out": _barrier(A.KNOCK_OUT, True),
    "down-in": _barrier(A.KNOCK_IN, False),
}


@pytest.mark.parametrize("name", sorted(PATH_PRODUCTS))
@pytest.mark.parametrize("smoothing", [0.0, 0.5])
@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
def test_black_scholes_path_products_with_dividends(engine, name, smoothing, engine_kind):
    prod = PATH_PRODUCTS[name]
    units = 512 if engine_kind == A.ENGINE_RQMC else 4099
    price = D.path_plan([prod], DIVS, engine=engine_kind, units=units, smoothing=smoothing,
                        antithetic=engine_kind == A.ENGINE_PSEUDO)
    G.assert_parity(price)
    risk = D.path_plan([prod], DIVS, engine=engine_kind, units=units, smoothing=smoothing, risk=True,
                       antithetic=engine_kind == A.ENGINE_PSEUDO)
    G.assert_parity(risk)


@pytest.fixture(scope="module")
def ssvi_grid():
    surface = W.SsviSurface(steps=12, expiries=12)
    return W.local_vol_grid(surface, G.gpu_grid)


@pytest.mark.parametrize("engine_kind,bridge", [(A.ENGINE_PSEUDO, False), (A.ENGINE_PSEUDO, True),
                                                (A.ENGINE_RQMC, True)])
@pytest.mark.parametrize("risk", [False, True])
def test_local_volatility_with_dividends_matches_the_oracle(engine, ssvi_grid, engine_kind, bridge, risk):
    """Ex-dates at 0.3 (between monitoring dates: a time-grid node of its own)
    and at 0.5 and 0.75 (monitoring dates); an Asian and a down-and-out call on
    the same draws."""
    prods = [PATH_PRODUCTS["asian"], _barrier(A.KNOCK_OUT, False)]
    spec = D.path_plan(prods, [(0.3, 1.5, 0.0), (0.5, 0.0, 0.02), (0.75, 1.0, 0.01)],
                       model=A.MODEL_LOCAL_VOLATILITY, grid=ssvi_grid, engine=engine_kind,
                       units=1024 if engine_kind == A.ENGINE_RQMC else 3001, bridge=bridge, risk=risk)
    G.assert_parity(spec)


def test_without_dividends_the_plan_is_unchanged(engine, ssvi_grid):
    """An empty schedule and no schedule give the same bits (the dividend code
    paths are not taken)."""
    prods = [PATH_PRODUCTS["asian"], _barrier(A.KNOCK_OUT, False)]
    a = G.run_engine(D.path_plan(prods, [], model=A.MODEL_LOCAL_VOLATILITY, grid=ssvi_grid, units=2048))
    spec = D.path_plan(prods, [], model=A.MODEL_LOCAL_VOLATILITY, grid=ssvi_grid, units=2048)
    spec.dividends = ()
    b = G.run_engine(spec)
    for k in range(2):
        assert a.products[k].price.value == b.products[k].price.value


def test_what_dividends_leave_out_is_unsupported(engine, ssvi_grid):
    cont = D.path_plan([ProductSpec(kind=A.PRODUCT_CONTINUOUS_BARRIER, barrier=80.0, rebate=1.0)], DIVS)
    lv_vega = D.path_plan([PATH_PRODUCTS["asian"]], DIVS, model=A.MODEL_LOCAL_VOLATILITY, grid=ssvi_grid)
    lv_vega.request_vega = True
    for spec in (cont, lv_vega):
        with pytest.raises(N.EngineError) as err:
            G.run_engine(spec)
        assert err.value.name == "unsupported"
    spec, lsm = W.american_bs(dates=4, units=1024)
    spec.dividends = [(0.5, 1.0, 0.0)]
    with pytest.raises(N.EngineError) as err:
        N.lsm_price(spec, lsm)
    assert err.value.name == "unsupported"
    bad = D.european(A.CALL, [(0.5, 200.0, 0.0)], units=1024)  # the reserve exceeds the spot
    with pytest.raises(N.EngineError) as err:
        G.run_engine(bad)
    assert err.value.name == "market"

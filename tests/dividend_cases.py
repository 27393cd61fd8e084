"""Discrete-dividend plans of the escrowed affine model and their acceptance checks.

The cases restate the reference's own acceptance of the affine dividend model
(crates/pricing/tests/affine_oracles.rs:131-230), whose checks need no
simulation:

* with zero volatility and zero rates a cash dividend, a proportional one or
  both leave a known terminal spot (80, 100 or 70 from 100), so the price is the
  intrinsic value against strike 90;
* a cash-and-proportional dividend (20 at t = 0.5 with 10 %) prices a European
  like Black--Scholes on the escrowed spot 0.9 (S - R), R = 20 / 0.9 e^{-(r - q) 0.5}
  the discounted cash reserve, with Delta scaled by 0.9 and Vega unchanged.
"""
import math

from rust_pricing_b200 import _abi as A
from rust_pricing_b200.desc import PlanSpec, ProductSpec

SPOT, STRIKE = 100.0, 90.0

# (ex-time, cash, proportional, terminal spot) of affine_oracles.rs:133-139
DETERMINISTIC = [(0.5, 20.0, 0.0, 80.0), (1.0, 20.0, 0.0, 80.0), (1.5, 20.0, 0.0, 100.0),
                 (0.5, 0.0, 0.2, 80.0), (0.5, 20.0, 0.1, 70.0)]


def curves(rate: float, repo: float) -> dict:
    """The tests' two-pillar curves on [0, 2]."""
    return dict(discount_times=(0.0, 2.0), discount_factors=(1.0, math.exp(-2.0 * rate)),
                dividend_times=(0.0, 2.0), dividend_factors=(1.0, math.exp(-2.0 * repo)))


def european(side: int, dividends, vol: float = 0.2, rate: float = 0.05, repo: float = 0.02,
             units: int = 1 << 16, engine: int = A.ENGINE_PSEUDO, risk: bool = False,
             antithetic: bool = True) -> PlanSpec:
    return PlanSpec(observation_times=[1.0], products=[ProductSpec(kind=A.PRODUCT_EUROPEAN, side=side,
                                                                   strike=STRIKE)],
                    engine=engine, master_seed=42, sampling_units=units, scramble_count=8,
                    antithetic=antithetic, volatility=vol, spot=SPOT, dividends=list(dividends),
                    request_delta=risk, request_gamma=risk, request_vega=risk, gamma_bump=0.01,
                    **curves(rate, repo))


def escrowed_reference(side: int, rate: float = 0.05, repo: float = 0.02, vol: float = 0.2):
    """affine_oracles.rs:167-197: Black--Scholes on 0.9 (S - R), Delta x 0.9."""
    import bs_closed_form as B
    reserve = 20.0 / 0.9 * math.exp(-(rate - repo) * 0.5)
    r = B.black_scholes(side == A.CALL, 0.9 * (SPOT - reserve), STRIKE, 1.0, rate, repo, vol)
    return {"price": r["price"], "delta": 0.9 * r["delta"], "vega": r["vega"],
            "gamma": 0.81 * r["gamma"]}


def path_plan(products, dividends, model=A.MODEL_BLACK_SCHOLES, grid=None, engine=A.ENGINE_PSEUDO,
              units=4099, steps=12, risk=False, smoothing=0.0, bridge=False, antithetic=False) -> PlanSpec:
    """Monthly observations over a year under dividends at some of them."""
    times = [(i + 1) / steps for i in range(steps)]
    spec = PlanSpec(observation_times=times, products=list(products), model=model, engine=engine,
                    master_seed=0x5EED, sampling_units=units, scramble_count=4, antithetic=antithetic,
                    volatility=0.25, spot=SPOT, dividends=list(dividends), request_delta=risk,
                    request_gamma=risk, request_vega=risk and model == A.MODEL_BLACK_SCHOLES, gamma_bump=0.01,
                    smoothing_half_width=smoothing, brownian_bridge=bridge, **curves(0.03, 0.01))
    if grid is not None:
        spec.local_variance = grid
    return spec

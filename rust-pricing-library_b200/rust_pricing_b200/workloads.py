"""Synthetic workloads with the shapes of the benchmark configurations.

There is no public data set for this path: each workload is a seeded synthetic
market with the sizes the configurations name (valuation at T = 0, ACT/365F
year fractions, flat log-linear curves as in the reference's
crates/pricing/examples/benchmark_european_bs.rs).

* european_bs      -- S=K=100, r=3%, q=1%, sigma=20%, T=1, one exact step.
* local_vol_rqmc   -- SSVI (theta=0.04t, rho=-0.4, eta=1, gamma=0.5) -> Dupire
                      grid 31 x 100, 252 daily steps, RQMC + Brownian bridge,
                      Asian call K=100 and discrete down-and-out call B=80,
                      rebate 1, priced on the same draws.
* local_vol_adjoint -- the same surface, continuous down-and-out call with
                      compact-C2 smoothing 0.5 (0.5% of spot).
* batched_book     -- a book of trades (seeded): maturities U(0.1, 3) years
                      with daily steps, strikes U(70, 130), 40 % European /
                      25 % Asian / 20 % continuous down-and-out / 15 % lookback,
                      half Black--Scholes (sigma U(0.15, 0.35)), half local
                      volatility on their own SSVI grids (rho, eta perturbed).
* american_bs      -- American put by LSM: S=K=100, r=5%, q=0, sigma=25%, T=1,
                      50 equally spaced exercise dates, cubic basis in spot,
                      CPQR tolerances 1e-14 / 1e-12, ITM tolerance 0.
"""
from __future__ import annotations

import math
from typing import Callable, Optional

import numpy as np

from . import _abi as A
from .desc import LocalVarianceSpec, LsmSpec, PlanSpec, ProductSpec

SEED = 0x0123456789ABCDEF
RATE, DIVIDEND = 0.03, 0.01


def flat_curves(rate: float = RATE, dividend: float = DIVIDEND, horizon: float = 1.0) -> dict:
    return dict(discount_times=(0.0, horizon), discount_factors=(1.0, math.exp(-rate * horizon)),
                dividend_times=(0.0, horizon), dividend_factors=(1.0, math.exp(-dividend * horizon)))


def european_bs(paths: int = 1 << 20, risk: bool = True, engine: int = A.ENGINE_PSEUDO,
                antithetic: bool = False, scrambles: int = 16) -> PlanSpec:
    return PlanSpec(
        observation_times=[1.0], products=[ProductSpec(kind=A.PRODUCT_EUROPEAN, strike=100.0)],
        model=A.MODEL_BLACK_SCHOLES, engine=engine, master_seed=SEED, sampling_units=paths,
        scramble_count=scrambles, antithetic=antithetic, volatility=0.2, spot=100.0,
        request_delta=risk, request_gamma=risk, request_vega=risk, gamma_bump=0.01,
        **flat_curves())


def daily_times(steps: int = 252, horizon: float = 1.0) -> list[float]:
    return [horizon * i / steps for i in range(1, steps + 1)]


def expiry_rows(steps: int = 252, expiries: int = 30) -> list[int]:
    """Daily indices of the surface expiries: evenly spread, the last one at T."""
    return [int(round(k * steps / expiries)) for k in range(1, expiries + 1)]


def piecewise_sinh_nodes(left: float = -1.2, right: float = 0.8, left_intervals: int = 50,
                         right_intervals: int = 49, left_shape: float = 1.5,
                         right_shape: float = 1.5) -> list[float]:
    """piecewise_sinh_log_moneyness_nodes (crates/pricing/src/market/local_variance.rs:417-478)."""
    def ratio(shape, fraction):
        return fraction if shape == 0.0 else math.sinh(shape * fraction) / math.sinh(shape)
    nodes = []
    for i in range(left_intervals + 1):
        fr = i / left_intervals
        nodes.append(0.0 if i == left_intervals else left * ratio(left_shape, 1.0 - fr))
    for i in range(1, right_intervals + 1):
        nodes.append(right * ratio(right_shape, i / right_intervals))
    return nodes


class SsviSurface:
    """Standard SSVI with power-law phi and a PCHIP theta curve."""

    def __init__(self, steps: int = 252, expiries: int = 30, horizon: float = 1.0,
                 theta_slope: float = 0.04, rho: float = -0.4, eta: float = 1.0, gamma: float = 0.5):
        times = daily_times(steps, horizon)
        rows = expiry_rows(steps, expiries)
        self.theta_times = [times[i - 1] for i in rows]
        self.theta_values = [theta_slope * t for t in self.theta_times]
        self.terminal_slope = theta_slope
        self.rho, self.eta, self.gamma = rho, eta, gamma
        self.time_nodes = [0.0] + self.theta_times
        self.log_moneyness_nodes = piecewise_sinh_nodes()

    def grid_args(self):
        return (self.theta_times, self.theta_values, self.terminal_slope, self.rho, self.eta,
                self.gamma, self.time_nodes, self.log_moneyness_nodes)


GridBuilder = Callable[[SsviSurface, float, float], np.ndarray]


def local_vol_grid(surface: SsviSurface, builder: GridBuilder, floor: float = 1e-8,
                   cap: float = 4.0) -> LocalVarianceSpec:
    values = builder(surface, floor, cap)
    return LocalVarianceSpec(surface.time_nodes, surface.log_moneyness_nodes, values, floor, cap)


def local_vol_rqmc(builder: GridBuilder, points: int = 1 << 20, scrambles: int = 16,
                   steps: int = 252, bridge: bool = True, engine: int = A.ENGINE_RQMC,
                   surface: Optional[SsviSurface] = None) -> PlanSpec:
    surface = surface or SsviSurface(steps=steps, expiries=min(30, steps))
    times = daily_times(steps)
    weights = [1.0 / steps] * steps
    products = [
        ProductSpec(kind=A.PRODUCT_ASIAN, strike=100.0, weights=weights),
        ProductSpec(kind=A.PRODUCT_DISCRETE_BARRIER, strike=100.0, barrier=80.0,
                    barrier_direction=A.BARRIER_DOWN, barrier_style=A.KNOCK_OUT, rebate=1.0),
    ]
    return PlanSpec(observation_times=times, products=products, model=A.MODEL_LOCAL_VOLATILITY,
                    engine=engine, master_seed=SEED, sampling_units=points, scramble_count=scrambles,
                    brownian_bridge=bridge, spot=100.0, local_variance=local_vol_grid(surface, builder),
                    **flat_curves())


def local_vol_adjoint(builder: GridBuilder, paths: int = 1 << 20, steps: int = 252,
                      smoothing: float = 0.5, risk: bool = True,
                      surface: Optional[SsviSurface] = None) -> PlanSpec:
    surface = surface or SsviSurface(steps=steps, expiries=min(30, steps))
    times = daily_times(steps)
    products = [ProductSpec(kind=A.PRODUCT_CONTINUOUS_BARRIER, strike=100.0, barrier=80.0,
                            barrier_direction=A.BARRIER_DOWN, barrier_style=A.KNOCK_OUT,
                            rebate=1.0)]
    return PlanSpec(observation_times=times, products=products, model=A.MODEL_LOCAL_VOLATILITY,
                    engine=A.ENGINE_PSEUDO, master_seed=SEED, sampling_units=paths,
                    brownian_bridge=True, spot=100.0, local_variance=local_vol_grid(surface, builder),
                    smoothing_half_width=smoothing, request_delta=risk, request_gamma=risk,
                    gamma_bump=0.01, **flat_curves())


def american_bs(dates: int = 50, units: int = 1 << 20, training_units: Optional[int] = None,
                engine: int = A.ENGINE_PSEUDO, antithetic: bool = False, scrambles: int = 4,
                max_degree: int = 3, vol: float = 0.25, rate: float = 0.05, strike: float = 100.0,
                side: int = A.PUT, horizon: float = 1.0) -> tuple[PlanSpec, LsmSpec]:
    """An American (Bermudan) option with `dates` equally spaced exercise dates
    and its LsmConfig: pseudo `units` sampling units (RQMC: points per
    scramble) for valuation and `training_units` for training."""
    times = [horizon * i / dates for i in range(1, dates + 1)]
    spec = PlanSpec(
        observation_times=times, products=[ProductSpec(kind=A.PRODUCT_AMERICAN, side=side, strike=strike)],
        model=A.MODEL_BLACK_SCHOLES, engine=engine, master_seed=SEED, sampling_units=units,
        scramble_count=scrambles, antithetic=antithetic, volatility=vol, spot=100.0,
        **flat_curves(rate, 0.0, horizon))
    lsm = LsmSpec(training_seed=SEED ^ 0x5DEECE66D, training_units=training_units or units,
                  training_scramble_count=scrambles, training_antithetic=antithetic, max_degree=max_degree,
                  max_matrix_elements=1 << 40)
    return spec, lsm


def american_lv(grid: LocalVarianceSpec, dates: int = 50, units: int = 1 << 20, training_units: Optional[int] = None,
                engine: int = A.ENGINE_PSEUDO, antithetic: bool = False, scrambles: int = 4,
                bridge: bool = False, max_degree: int = 3, rate: float = 0.05, strike: float = 100.0,
                side: int = A.PUT, horizon: float = 1.0) -> tuple[PlanSpec, LsmSpec]:
    """The American option of `american_bs` under a local-variance grid (the
    training and valuation paths are Log-Euler paths on the grid's time grid
    joined with the exercise dates)."""
    spec, lsm = american_bs(dates=dates, units=units, training_units=training_units, engine=engine,
                            antithetic=antithetic, scrambles=scrambles, max_degree=max_degree, vol=0.0,
                            rate=rate, strike=strike, side=side, horizon=horizon)
    spec.model = A.MODEL_LOCAL_VOLATILITY
    spec.local_variance = grid
    spec.brownian_bridge = bridge
    lsm.training_brownian_bridge = bridge
    return spec, lsm


def flat_grid(vol: float, horizon: float = 1.0) -> LocalVarianceSpec:
    """A 2 x 2 local-variance grid holding sigma^2 everywhere: its Log-Euler
    paths on the exercise dates are the exact Black--Scholes paths."""
    return LocalVarianceSpec([0.0, horizon], [-1.0, 1.0], np.full((2, 2), vol * vol), 1e-8, 4.0)


BOOK_SEED = 20260904


def batched_book(builder: GridBuilder, trades: int = 4096, units: int = 1 << 16, seed: int = BOOK_SEED,
                 expiries: int = 30) -> list[PlanSpec]:
    """The batched-book configuration: `trades` single-product plans, each
    with its own seed, maturity, step count, strike, product and model."""
    rng = np.random.default_rng(seed)
    specs = []
    kinds = np.array([A.PRODUCT_EUROPEAN] * 8 + [A.PRODUCT_ASIAN] * 5 + [A.PRODUCT_CONTINUOUS_BARRIER] * 4 +
                     [A.PRODUCT_LOOKBACK] * 3)
    for i in range(trades):
        horizon = float(rng.uniform(0.1, 3.0))
        steps = max(1, int(round(252 * horizon)))
        strike = float(rng.uniform(70.0, 130.0))
        kind = int(kinds[rng.integers(0, len(kinds))])
        local = bool(rng.integers(0, 2))
        vol = float(rng.uniform(0.15, 0.35))
        rho = float(rng.uniform(-0.6, -0.2))
        # the power-law wing bound eta (1 + |rho|) <= 2 of StandardSsvi::new
        eta = min(float(rng.uniform(0.7, 1.3)), 2.0 / (1.0 + abs(rho)))
        barrier = float(rng.uniform(60.0, 90.0))
        times = daily_times(steps, horizon)
        if kind == A.PRODUCT_ASIAN:
            product = ProductSpec(kind=kind, strike=strike, weights=[1.0 / steps] * steps)
        elif kind == A.PRODUCT_CONTINUOUS_BARRIER:
            product = ProductSpec(kind=kind, strike=strike, barrier=barrier, barrier_direction=A.BARRIER_DOWN,
                                  barrier_style=A.KNOCK_OUT)
        else:
            product = ProductSpec(kind=kind, strike=strike)
        if kind == A.PRODUCT_EUROPEAN and not local:
            times = [horizon]
        spec = PlanSpec(observation_times=times, products=[product], engine=A.ENGINE_PSEUDO,
                        master_seed=(SEED + 7919 * i) & 0xFFFFFFFFFFFFFFFF, sampling_units=units, spot=100.0,
                        volatility=vol, **flat_curves(horizon=horizon))
        if local:
            surface = SsviSurface(steps=steps, expiries=min(expiries, steps), horizon=horizon, rho=rho, eta=eta)
            spec.model = A.MODEL_LOCAL_VOLATILITY
            spec.local_variance = local_vol_grid(surface, builder)
        specs.append(spec)
    return specs

"""Multi-asset plans and their acceptance checks, after the reference's own acceptance
(crates/pricing/tests/multi_asset.rs:157-246): one-asset basket = the
Black--Scholes closed form; two perfectly correlated copies of an asset = the
one asset; an exchange option (basket [1, -1], strike 0) under a correlation
that changes during the life = Margrabe with the time-averaged correlation.
The reference's dates (valuation 2026-01-01, expiry 2027-01-01, correlation
change 2026-07-02) are kept as ACT/365F times."""
import math

import numpy as np

from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import workloads as W
from rust_pricing_b200.desc import AssetSpec, LocalVarianceSpec, MultiAssetSpec

CHANGE = 182.0 / 365.0   # 2026-07-02 from 2026-01-01
BEFORE = -31.0 / 365.0   # 2025-12-01


def ncdf(x):
    return 0.5 * math.erfc(-x / math.sqrt(2.0))


def npdf(x):
    return math.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def asset(spot, r, q, vol=0.2, grid=None):
    """The tests' market: flat curves on [0, 2]; Black--Scholes or local vol."""
    a = AssetSpec(spot=spot, volatility=vol, dividend_times=(0.0, 2.0), dividend_factors=(1.0, math.exp(-2.0 * q)))
    if grid is not None:
        a.model = A.MODEL_LOCAL_VOLATILITY
        a.local_variance = grid
    return a


def corr(n, rho):
    return [(BEFORE, [[1.0 if i == j else rho for j in range(n)] for i in range(n)])]


def curve(r):
    return dict(discount_times=(0.0, 2.0), discount_factors=(1.0, math.exp(-2.0 * r)))


def rqmc(points=8192, bridge=True):
    return dict(engine=A.ENGINE_RQMC, sampling_units=points, scramble_count=8, master_seed=702,
                antithetic=True, brownian_bridge=bridge)


def one_asset(**engine):
    return MultiAssetSpec(assets=[asset(100.0, 0.03, 0.01)], correlations=corr(1, 0.0), strike=105.0,
                          weights=[1.0], **curve(0.03), **(engine or rqmc()))


def one_asset_closed_form():
    v = 0.2
    d1 = (math.log(100.0 / 105.0) + 0.02 + 0.5 * v * v) / v
    d2 = d1 - v
    return 100.0 * math.exp(-0.01) * ncdf(d1) - 105.0 * math.exp(-0.03) * ncdf(d2)


def duplicated(**engine):
    return MultiAssetSpec(assets=[asset(100.0, 0.03, 0.01), asset(100.0, 0.03, 0.01)], correlations=corr(2, 1.0),
                          strike=105.0, weights=[0.5, 0.5], **curve(0.03), **(engine or rqmc()))


def margrabe(bridge=True, points=8192):
    c = [(BEFORE, [[1.0, 1.0], [1.0, 1.0]]), (CHANGE, [[1.0, -0.5], [-0.5, 1.0]])]
    return MultiAssetSpec(assets=[asset(100.0, 0.04, 0.01, 0.2), asset(95.0, 0.04, 0.02, 0.3)], correlations=c,
                          strike=0.0, weights=[1.0, -1.0], **curve(0.04), **rqmc(points, bridge))


def margrabe_closed_form():
    t = CHANGE
    variance = 0.2 ** 2 + 0.3 ** 2 - 2.0 * 0.2 * 0.3 * (t - 0.5 * (1.0 - t))
    sigma = math.sqrt(variance)
    d1 = (math.log(100.0 / 95.0) + (-0.01 + 0.02) + variance / 2.0) / sigma
    return 100.0 * math.exp(-0.01) * ncdf(d1) - 95.0 * math.exp(-0.02) * ncdf(d1 - sigma)


def lv_grid(values):
    """The tests' 3 x 3 local-variance grid (times 0, 0.5, 1; x -0.8, 0, 0.8)."""
    return LocalVarianceSpec([0.0, 0.5, 1.0], [-0.8, 0.0, 0.8], np.asarray(values, dtype=np.float64).reshape(3, 3),
                             1e-5, 2.0)


def mixed(n=3, product=A.MULTI_BASKET, engine=A.ENGINE_PSEUDO, bridge=True, antithetic=True, smoothing=0.0,
          units=4099, grid_builder=None):
    """A mix of Black--Scholes and local-volatility assets (one on the SSVI
    Dupire grid of the benchmark surface when a grid builder is given)."""
    assets = [asset(100.0, 0.03, 0.01, 0.2),
              asset(95.0, 0.03, 0.02, 0.3, lv_grid([0.04, 0.03, 0.05, 0.05, 0.04, 0.06, 0.06, 0.05, 0.07])),
              asset(110.0, 0.03, 0.0, 0.25),
              asset(90.0, 0.03, 0.015, 0.35)][:n]
    if grid_builder is not None and n >= 3:
        surface = W.SsviSurface(steps=12, expiries=12)
        assets[2] = asset(110.0, 0.03, 0.0, 0.25, W.local_vol_grid(surface, grid_builder))
    rho = [[1.0, 0.5, 0.3, 0.1], [0.5, 1.0, 0.4, 0.2], [0.3, 0.4, 1.0, -0.3], [0.1, 0.2, -0.3, 1.0]]
    m = [row[:n] for row in rho[:n]]
    m2 = [[1.0 if i == j else 0.5 * m[i][j] for j in range(n)] for i in range(n)]
    spec = MultiAssetSpec(assets=assets, correlations=[(BEFORE, m), (0.4, m2)], strike=1.0 if product else 95.0,
                          product=product, weights=[0.4, 0.3, 0.2, 0.1][:n], scales=[100.0, 95.0, 110.0, 90.0][:n]
                          if product == A.MULTI_WORST_OF else None, smoothing_half_width=smoothing, engine=engine,
                          sampling_units=units if engine == A.ENGINE_PSEUDO else 1024, scramble_count=4,
                          antithetic=antithetic, brownian_bridge=bridge, maximum_step=1.0 / 12, **curve(0.03))
    if product == A.MULTI_WORST_OF:
        spec.side = A.PUT
        spec.notional = 100.0
    return spec

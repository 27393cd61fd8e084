"""Bump-and-revalue cases and their acceptance checks.

The reference's own acceptance of its bump plans
(crates/pricing/src/engine/risk/bump.rs:936-1012,
`local_volatility_bump_agrees_with_native_delta`): a spot-Delta bump of
relative size 1e-6 on the `black_scholes` specification fixture with its model
replaced by a 4 x 3 local-variance grid agrees with the engine's native Delta
within the combined standard errors, under 4096 pseudo-random units and under
RQMC (128 points x 16 scrambles, antithetic, Brownian bridge).  The fixture's
market: S = K = 100, T = 1, discount factor 0.95 and dividend discount factor
0.98 at one year, a European call, seed 7.
"""
from rust_pricing_b200 import _abi as A
from rust_pricing_b200.desc import LocalVarianceSpec, PlanSpec, ProductSpec

import numpy as np

# crates/pricing/src/engine/risk/bump.rs:990-995
FIXTURE_GRID = LocalVarianceSpec(time_nodes=[0.0, 0.25, 0.5, 1.0], log_moneyness_nodes=[-1.0, 0.0, 1.0],
                                 values=np.array([[0.05, 0.04, 0.045]] * 4), floor=1e-8, cap=4.0)


def fixture_plan(model=A.MODEL_BLACK_SCHOLES, engine=A.ENGINE_PSEUDO, units=4096, product=None, steps=1,
                 antithetic=None, bridge=None) -> PlanSpec:
    """The specification fixture's European call (or `product`) on `steps`
    equally spaced observation dates."""
    rqmc = engine == A.ENGINE_RQMC
    spec = PlanSpec(observation_times=[(i + 1) / steps for i in range(steps)],
                    products=[product or ProductSpec(kind=A.PRODUCT_EUROPEAN, strike=100.0)], model=model,
                    engine=engine, master_seed=7 if not rqmc else 819, sampling_units=128 if rqmc else units,
                    scramble_count=16, antithetic=rqmc if antithetic is None else antithetic,
                    brownian_bridge=rqmc if bridge is None else bridge, spot=100.0,
                    discount_times=(0.0, 1.0), discount_factors=(1.0, 0.95),
                    dividend_times=(0.0, 1.0), dividend_factors=(1.0, 0.98), volatility=0.2)
    if model == A.MODEL_LOCAL_VOLATILITY:
        spec.local_variance = FIXTURE_GRID
    return spec


def native(spec: PlanSpec, **flags) -> PlanSpec:
    """The same plan with the engine's own Greeks requested."""
    import copy
    s = copy.copy(spec)
    s._keep = []
    for k, v in flags.items():
        setattr(s, k, v)
    return s

"""Correlated multi-asset paths on the GPU (mcg_multi_asset_price).

* The reference's acceptance checks (crates/pricing/tests/multi_asset.rs:157-246), as for
  the oracle: a one-asset basket is Black--Scholes, two perfectly correlated
  copies are the one asset to 1e-12, and an exchange option under a
  correlation change is Margrabe with the time-averaged correlation.
* Engine vs oracle on identical draws: Black--Scholes and local-volatility
  assets (a 3 x 3 grid and the SSVI Dupire grid), two to four assets, a
  correlation change, basket and worst-of, exact and smoothed, pseudo-MC and
  RQMC, with and without the Brownian bridge and antithetic pairs -- the
  price within 1e-12 of its scale and the standard error within 1e-10.
"""
import pytest

import gpu_common as G
import helpers as H
import multi_asset_cases as M
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N

pytestmark = pytest.mark.gpu


def assert_same(spec):
    got = N.multi_asset_price(spec)
    want = H.oracle_multi(spec)
    scale = max(abs(want.price.value), want.price.standard_error)
    assert abs(got.price.value - want.price.value) <= G.DIRECT_TOL * scale, (got.price.value, want.price.value)
    assert abs(got.price.standard_error - want.price.standard_error) <= 1e-10 * want.price.standard_error
    assert got.price.effective_sampling_units == want.price.effective_sampling_units
    assert (got.time_steps, got.dimension, got.evaluated_paths) == (want.time_steps, want.dimension,
                                                                    want.evaluated_paths)
    return got


def test_one_asset_basket_is_black_scholes(engine):
    r = N.multi_asset_price(M.one_asset(**M.rqmc(1 << 16)))
    assert abs(r.price.value - M.one_asset_closed_form()) <= 7.0 * r.price.standard_error + 0.002


def test_perfectly_correlated_copies_are_the_one_asset(engine):
    a = N.multi_asset_price(M.one_asset())
    b = N.multi_asset_price(M.duplicated())
    assert abs(a.price.value - b.price.value) <= 1e-12


@pytest.mark.parametrize("bridge", [False, True])
def test_exchange_option_is_margrabe_under_a_correlation_change(engine, bridge):
    r = N.multi_asset_price(M.margrabe(bridge, points=1 << 16))
    assert abs(r.price.value - M.margrabe_closed_form()) <= 7.0 * r.price.standard_error + 0.006
    assert_same(M.margrabe(bridge))


@pytest.mark.parametrize("n", [2, 3, 4])
@pytest.mark.parametrize("product", [A.MULTI_BASKET, A.MULTI_WORST_OF])
@pytest.mark.parametrize("engine_kind,bridge", [(A.ENGINE_PSEUDO, False), (A.ENGINE_PSEUDO, True),
                                                (A.ENGINE_RQMC, False), (A.ENGINE_RQMC, True)])
def test_matches_the_oracle(engine, n, product, engine_kind, bridge):
    assert_same(M.mixed(n=n, product=product, engine=engine_kind, bridge=bridge))


@pytest.mark.parametrize("smoothing", [0.0, 0.05])
@pytest.mark.parametrize("antithetic", [False, True])
def test_ssvi_local_volatility_asset_and_smoothing(engine, smoothing, antithetic):
    assert_same(M.mixed(n=4, product=A.MULTI_WORST_OF, smoothing=smoothing, antithetic=antithetic,
                        grid_builder=G.gpu_grid))


def test_rejects_what_it_does_not_price(engine):
    spec = M.mixed(n=2)
    spec.correlations = [(M.BEFORE, [[1.0, 1.5], [1.5, 1.0]])]
    with pytest.raises(N.EngineError) as err:
        N.multi_asset_price(spec)
    assert err.value.name == "invalid_argument"
    spec = M.mixed(n=2)
    spec.correlations = [(0.1, [[1.0, 0.0], [0.0, 1.0]])]  # nothing in force at the valuation date
    with pytest.raises(N.EngineError):
        N.multi_asset_price(spec)

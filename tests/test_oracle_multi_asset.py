"""The oracle's correlated multi-asset paths against the reference's acceptance checks
(crates/pricing/tests/multi_asset.rs:157-246), each within 7 standard errors
plus the reference's floor: a one-asset basket is Black--Scholes, two
perfectly correlated copies equal the one asset to 1e-12 (the bridged terminal
normal drives both), and an exchange option under a correlation change is
Margrabe's price with the time-averaged correlation, with and without the
Brownian bridge."""
import pytest

import helpers as H
import multi_asset_cases as M


def test_one_asset_basket_is_black_scholes():
    r = H.oracle_multi(M.one_asset(), threads=8)
    assert abs(r.price.value - M.one_asset_closed_form()) <= 7.0 * r.price.standard_error + 0.002


def test_perfectly_correlated_copies_are_the_one_asset():
    a = H.oracle_multi(M.one_asset(), threads=8)
    b = H.oracle_multi(M.duplicated(), threads=8)
    assert abs(a.price.value - b.price.value) <= 1e-12


@pytest.mark.parametrize("bridge", [False, True])
def test_exchange_option_is_margrabe_under_a_correlation_change(bridge):
    r = H.oracle_multi(M.margrabe(bridge), threads=8)
    assert r.time_steps == 5  # 0.25 substeps plus the correlation change
    assert abs(r.price.value - M.margrabe_closed_form()) <= 7.0 * r.price.standard_error + 0.006


def test_mixed_black_scholes_and_local_volatility_assets_price():
    for product in (0, 1):
        r = H.oracle_multi(M.mixed(product=product, units=1024), threads=8)
        assert r.price.value > 0.0 and r.price.standard_error > 0.0

"""The oracle's escrowed affine dividend model against the reference's own
acceptance checks (crates/pricing/tests/affine_oracles.rs:131-230): deterministic
terminal spots under zero volatility, and the escrowed-spot Black--Scholes
closed form for a cash-and-proportional dividend (price, Delta, Vega)."""
import pytest

import dividend_cases as D
import helpers as H
from rust_pricing_b200 import _abi as A


@pytest.mark.parametrize("case", D.DETERMINISTIC, ids=lambda c: f"t{c[0]}-cash{c[1]}-beta{c[2]}")
@pytest.mark.parametrize("side", [A.CALL, A.PUT])
def test_zero_volatility_dividends_leave_the_known_terminal_spot(case, side):
    t, cash, beta, terminal = case
    spec = D.european(side, [(t, cash, beta)], vol=0.0, rate=0.0, repo=0.0, units=64)
    p = H.oracle_evaluate(spec, threads=2).products[0]
    sign = 1.0 if side == A.CALL else -1.0
    assert abs(p.price.value - max(sign * (terminal - D.STRIKE), 0.0)) <= 1e-12


@pytest.mark.parametrize("side", [A.CALL, A.PUT])
def test_mixed_dividend_is_black_scholes_on_the_escrowed_spot(side):
    spec = D.european(side, [(0.5, 20.0, 0.1)], units=1 << 17, risk=True)
    p = H.oracle_evaluate(spec, threads=8).products[0]
    want = D.escrowed_reference(side)
    for key in ("price", "delta", "vega", "gamma"):
        est = getattr(p, key)
        assert abs(est.value - want[key]) <= 4.5 * est.standard_error, (key, est.value, want[key])


def test_no_dividends_is_the_plain_plan():
    """An empty schedule gives the dividend-free plan bit for bit."""
    a = H.oracle_evaluate(D.european(A.CALL, [], units=1024, risk=True), threads=2).products[0]
    b = D.european(A.CALL, [], units=1024, risk=True)
    b.dividends = []
    c = H.oracle_evaluate(b, threads=2).products[0]
    assert (a.price.value, a.delta.value, a.vega.value) == (c.price.value, c.delta.value, c.vega.value)


def test_barrier_on_an_ex_date_sees_the_pre_dividend_spot():
    """An up-and-out barrier monitored on an ex-date is hit by the spot just
    before a large cash dividend even though every post-dividend spot stays
    below it (compile.rs:315-346): zero volatility and rates, spot 100; a cash
    dividend of 40 on the first monitoring date leaves 60 after it."""
    from rust_pricing_b200.desc import ProductSpec
    prod = ProductSpec(kind=A.PRODUCT_DISCRETE_BARRIER, strike=50.0, barrier=99.0,
                       barrier_direction=A.BARRIER_UP, barrier_style=A.KNOCK_OUT, rebate=3.0)
    spec = D.path_plan([prod], [(1 / 12, 40.0, 0.0)], units=64)
    spec.volatility = 0.0
    spec.discount_factors = (1.0, 1.0)
    spec.dividend_factors = (1.0, 1.0)
    out = H.oracle_evaluate(spec, threads=2).products[0]
    assert out.price.value == 3.0  # the pre-dividend spot 100 knocks out: the rebate
    spec.dividends = [(0.04, 40.0, 0.0)]  # not a monitoring date: no pre-dividend check
    out = H.oracle_evaluate(spec, threads=2).products[0]
    assert abs(out.price.value - 10.0) <= 1e-12  # 60 at every date: alive, 60 - 50

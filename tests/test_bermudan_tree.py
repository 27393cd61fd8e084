"""The binomial benchmark: converges to Black--Scholes for a European and bounds
the early-exercise premium of the Bermudan put from above by the American."""
from bermudan_tree import bermudan_binomial, bermudan_equally_spaced
from bs_closed_form import black_scholes


def test_european_limit_matches_black_scholes():
    tree = bermudan_binomial(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 5000, [5000])
    bs = black_scholes(False, 100.0, 100.0, 1.0, 0.05, 0.0, 0.25)["price"]
    assert abs(tree - bs) < 2e-3


def test_bermudan_between_european_and_american():
    eu = bermudan_binomial(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 5000, [5000])
    berm = bermudan_equally_spaced(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 50)
    am = bermudan_binomial(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 5000, range(1, 5001))
    assert eu < berm < am
    assert am - berm < 0.05   # 50 dates are close to continuous exercise
    assert am - eu > 0.4      # the early-exercise premium of an at-the-money put at r = 5 %


def test_tree_has_converged_at_5000_steps():
    a = bermudan_equally_spaced(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 50, steps=2500)
    b = bermudan_equally_spaced(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 50, steps=5000)
    assert abs(a - b) < 2e-3

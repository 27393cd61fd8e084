"""American puts of the reference's Andersen--Broadie tests
(crates/pricing/tests/american_dual.rs:37-152): S = 100, r = 5 %, sigma = 0.2,
exercise on 2026-12-04, 2027-03-04, 2027-06-04 and 2027-09-04 from the
valuation date 2026-09-04, a cubic basis in spot trained on antithetic
pseudo paths (seed 17), antithetic pseudo valuation paths, reduction blocks
of 64 units, inner path counts (N, N / 2 + 1) and inner seed 0x1234."""
import datetime as dt
import math

from rust_pricing_b200 import _abi as A
from rust_pricing_b200.desc import LsmSpec, PlanSpec, ProductSpec

VALUATION = dt.date(2026, 9, 4)
DATES = [dt.date(2026, 12, 4), dt.date(2027, 3, 4), dt.date(2027, 6, 4), dt.date(2027, 9, 4)]
INNER_SEED = 0x1234


def times(dates=DATES):
    return [(d - VALUATION).days / 365.0 for d in dates]


def inner(paths: int):
    return paths, paths // 2 + 1


def case(side=A.PUT, strike=100.0, vol=0.2, dividend=0.0, dates=DATES, units=256, training_units=2048,
         antithetic=True, seed=91, notional=1.0):
    spec = PlanSpec(
        observation_times=times(dates),
        products=[ProductSpec(kind=A.PRODUCT_AMERICAN, side=side, strike=strike, notional=notional)],
        engine=A.ENGINE_PSEUDO, master_seed=seed, sampling_units=units, scramble_count=0,
        antithetic=antithetic, reduction_block_size=64, spot=100.0,
        discount_times=[0.0, 1.0], discount_factors=[1.0, math.exp(-0.05)],
        dividend_times=[0.0, 1.0], dividend_factors=[1.0, math.exp(-dividend)], volatility=vol)
    lsm = LsmSpec(training_seed=17, training_units=training_units, training_antithetic=True, max_degree=3,
                  itm_abs_tolerance=0.0, cpqr_abs_tolerance=1e-14, cpqr_rel_tolerance=1e-12,
                  max_matrix_elements=4_000_000)
    return spec, lsm


def tree_price(side=A.PUT, strike=100.0, dividend=0.0, vol=0.2, steps_per_day=4):
    """The Bermudan binomial benchmark on the exercise dates (day counts x steps per day)."""
    from bermudan_tree import bermudan_binomial
    days = [(d - VALUATION).days for d in DATES]
    steps = days[-1] * steps_per_day
    return bermudan_binomial(100.0, strike, 0.05, dividend, vol, days[-1] / 365.0, steps,
                             [d * steps_per_day for d in days], put=side == A.PUT)

"""The oracle's Andersen--Broadie dual against the reference's own properties
(crates/pricing/tests/american_dual.rs; the reference has no golden vectors
for it, so these are the pins):

* the lower bound is the fitted policy's ordinary LSM price on the same
  outer paths (within 1e-12; the dual averages an antithetic pair as
  0.5 a + 0.5 b, the LSM valuation as (a + b) / 2);
* a single exercise date has a zero gap with a zero standard error;
* zero volatility is a deterministic grid: the lower bound is the largest
  discounted payoff of the exercise dates and the upper bound has no error;
* with 2048 outer and 8192 training units the bounds bracket the Bermudan
  binomial tree (5 standard errors + 0.03), and 256 inner paths tighten the
  gap against 16 (within noise);
* the evaluation does not depend on the oracle's thread count.
"""
import math

import pytest

import dual_cases as D
import helpers as H
import lsm_cases as L
from rust_pricing_b200 import _abi as A


def test_lower_bound_is_the_lsm_price_of_the_replay_policy():
    for c in L.cases():
        spec, lsm = L.plan(c)
        if spec.engine != A.ENGINE_PSEUDO:
            continue
        spec.request_delta = spec.request_gamma = spec.request_vega = False
        price = H.oracle_lsm(spec, lsm, threads=4).result.price
        d = H.oracle_lsm_dual(spec, lsm, 64, 33, D.INNER_SEED, threads=8)
        assert abs(d.lower_bound.value - price.value) <= 1e-12 * abs(price.value)
        assert d.upper_bound.value >= d.lower_bound.value
        assert abs(d.upper_bound.value - d.lower_bound.value - d.duality_gap.value) <= 1e-12
        assert d.outer_trajectories == 2 * spec.sampling_units
        assert d.exercise_date_count == len(spec.observation_times)


@pytest.mark.parametrize("antithetic", [False, True])
def test_single_exercise_date_has_zero_gap(antithetic):
    spec, lsm = D.case(dates=D.DATES[-1:], antithetic=antithetic)
    d = H.oracle_lsm_dual(spec, lsm, *D.inner(8), D.INNER_SEED)
    price = H.oracle_lsm(spec, lsm).result.price
    assert d.duality_gap.value == 0.0 and d.duality_gap.standard_error == 0.0
    assert d.lower_bound.value == d.upper_bound.value
    assert abs(d.lower_bound.value - price.value) <= 1e-12 * price.value
    assert d.inner_paths == 0


def test_zero_volatility_is_the_deterministic_maximum():
    spec, lsm = D.case(vol=0.0, strike=105.0, units=64, training_units=256)
    d = H.oracle_lsm_dual(spec, lsm, *D.inner(8), D.INNER_SEED)
    fwd = [100.0 * math.exp(0.05 * t) for t in spec.observation_times]  # q = 0, r = 5 %
    payoffs = [max(105.0 - f, 0.0) * math.exp(-0.05 * t) for f, t in zip(fwd, spec.observation_times)]
    assert abs(d.lower_bound.value - max(payoffs)) < 1e-11
    assert d.upper_bound.standard_error == 0.0
    # one inner path per branch when the transition is deterministic
    assert d.inner_paths == d.outer_trajectories * (len(spec.observation_times) - 1)


def test_bounds_bracket_the_tree_and_inner_paths_tighten_the_gap():
    reference = D.tree_price()
    coarser = D.tree_price(steps_per_day=2)
    assert abs(reference - coarser) < 0.03
    gaps, variances = [0.0, 0.0], [0.0, 0.0]
    for seed in (71, 97, 113):
        spec, lsm = D.case(units=2048, training_units=8192, seed=seed)
        for level, n in enumerate((16, 256)):
            d = H.oracle_lsm_dual(spec, lsm, *D.inner(n), D.INNER_SEED)
            lo, up = d.lower_bound, d.upper_bound
            assert lo.value - 5.0 * lo.standard_error <= reference + 0.03
            assert up.value + 5.0 * up.standard_error >= reference - 0.03
            assert 0.0 <= d.duality_gap.value < 2.0
            gaps[level] += d.duality_gap.value / 3.0
            variances[level] += d.duality_gap.standard_error ** 2 / 9.0
    assert gaps[1] <= gaps[0] + 5.0 * math.sqrt(variances[0] + variances[1])


def test_replay_independent_of_thread_count():
    spec, lsm = D.case(units=512)
    a = H.oracle_lsm_dual(spec, lsm, *D.inner(12), D.INNER_SEED, threads=1)
    b = H.oracle_lsm_dual(spec, lsm, *D.inner(12), D.INNER_SEED, threads=7)
    for name in ("lower_bound", "upper_bound", "duality_gap"):
        assert getattr(a, name).value == getattr(b, name).value
        assert getattr(a, name).standard_error == getattr(b, name).standard_error
    assert a.inner_paths == b.inner_paths


def test_rejects_what_the_reference_rejects():
    spec, lsm = D.case()
    with pytest.raises(RuntimeError):
        H.oracle_lsm_dual(spec, lsm, 0, 4, D.INNER_SEED)
    spec.request_delta = True
    with pytest.raises(RuntimeError):
        H.oracle_lsm_dual(spec, lsm, 4, 4, D.INNER_SEED)

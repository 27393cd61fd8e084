"""The GPU's Andersen--Broadie dual (mcg_lsm_dual) against the oracle's.

Both train the policy on the same paths (the GPU's fitted models agree with
the oracle's within 5e-13, the same decisions on these paths), stop the same
outer valuation paths and roll out the same inner paths: lower, upper and gap
estimates within 1e-12 (scaled by the larger of the value and its standard
error), standard errors within 1e-9, the same number of inner paths; the
lower bound is the GPU's own LSM price within 1e-12; one exercise date has a
zero gap.
"""
import pytest

import dual_cases as D
import helpers as H
import lsm_cases as L
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N

pytestmark = pytest.mark.gpu


def assert_same(got, want):
    for name in ("lower_bound", "upper_bound", "duality_gap"):
        g, w = getattr(got, name), getattr(want, name)
        scale = max(abs(w.value), w.standard_error, 1e-300)
        assert abs(g.value - w.value) <= 1e-12 * scale, (name, g.value, w.value)
        assert abs(g.standard_error - w.standard_error) <= 1e-9 * max(w.standard_error, 1e-300), name
        assert g.effective_sampling_units == w.effective_sampling_units
    assert got.inner_paths == want.inner_paths
    assert got.outer_trajectories == want.outer_trajectories


def _cases():
    out = []
    for c in L.cases():
        spec, lsm = L.plan(c)
        if spec.engine == A.ENGINE_PSEUDO and not c["risk"].get("delta"):
            out.append((c["name"], spec, lsm, 64))
    out.append(("put_2048", *D.case(units=2048, training_units=8192, seed=71), 256))
    out.append(("call_dividend", *D.case(side=A.CALL, dividend=0.1, units=1024, training_units=4096, seed=97), 48))
    out.append(("put_no_antithetic", *D.case(antithetic=False, units=777, seed=113), 33))
    return out


@pytest.mark.parametrize("name, spec, lsm, n", _cases(), ids=lambda x: x if isinstance(x, str) else "")
def test_dual_against_the_oracle(engine, name, spec, lsm, n):
    got = N.lsm_dual(spec, lsm, *D.inner(n), D.INNER_SEED)
    want = H.oracle_lsm_dual(spec, lsm, *D.inner(n), D.INNER_SEED)
    assert_same(got, want)
    price = N.lsm_price(spec, lsm).result.price
    assert abs(got.lower_bound.value - price.value) <= 1e-12 * abs(price.value)


def test_single_exercise_date_has_zero_gap_on_the_gpu(engine):
    spec, lsm = D.case(dates=D.DATES[-1:])
    d = N.lsm_dual(spec, lsm, *D.inner(8), D.INNER_SEED)
    assert d.duality_gap.value == 0.0 and d.duality_gap.standard_error == 0.0
    assert d.lower_bound.value == d.upper_bound.value and d.inner_paths == 0


def test_rejections(engine):
    spec, lsm = D.case()
    with pytest.raises(N.EngineError):
        N.lsm_dual(spec, lsm, 0, 4, D.INNER_SEED)
    spec.engine, spec.scramble_count = A.ENGINE_RQMC, 4
    lsm.training_scramble_count = 4
    with pytest.raises(N.EngineError):
        N.lsm_dual(spec, lsm, 4, 4, D.INNER_SEED)

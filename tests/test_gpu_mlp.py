"""The learned continuation network on the GPU.

* Its forward pass and its hand-written backward pass (tensor-core BF16
  operands, FP32 accumulation) against the CPU FP64 restatement in
  tests/mlp_reference.py: tightly when the restatement rounds the same
  operands to BF16, loosely against plain FP64.
* The learned policy in the early-exercise engine: trained on the engine's
  own training paths, it beats the reference's polynomial policy against the
  independent Bermudan binomial tree, reproducibly.
"""
import numpy as np
import pytest

import mlp_reference as M
from bermudan_tree import bermudan_equally_spaced
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("rows", [1, 31, 1000, 4099])
def test_forward_matches_fp64(engine, rows):
    rng = np.random.default_rng(rows)
    p = M.init(rows)
    x = rng.normal(size=(rows, 2)).astype(np.float32)
    got = N.mlp_forward(p, x)
    want, _ = M.forward(p, x, bf16_ops=True)
    plain, _ = M.forward(p, x)
    scale = np.maximum(1.0, np.abs(want))
    assert np.max(np.abs(got - want) / scale) < 2e-3
    assert np.median(np.abs(got - want) / scale) < 2e-5
    assert np.max(np.abs(got - plain) / scale) < 3e-2


@pytest.mark.parametrize("rows", [7, 128, 3000])
def test_gradient_matches_fp64(engine, rows):
    rng = np.random.default_rng(100 + rows)
    p = M.init(rows + 1)
    x = rng.normal(size=(rows, 2)).astype(np.float32)
    y = rng.normal(size=rows).astype(np.float32)
    mask = rng.random(rows) < 0.6
    g, loss = N.mlp_gradient(p, x, y, mask)
    want, want_loss = M.gradient(p, x, y, mask, bf16_ops=True)
    plain, _ = M.gradient(p, x, y, mask)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, want_loss)
    assert rel_l2(g, want) < 5e-3
    assert rel_l2(g, plain) < 3e-2
    # each parameter block on its own
    for lo, hi in ((0, 128), (128, 192), (192, 4288), (4288, 4352), (4352, 4416), (4416, 4417)):
        assert rel_l2(g[lo:hi], want[lo:hi]) < 1e-2, (lo, hi)


def test_masked_rows_do_not_contribute(engine):
    rng = np.random.default_rng(9)
    p = M.init(2)
    x = rng.normal(size=(200, 2)).astype(np.float32)
    y = rng.normal(size=200).astype(np.float32)
    mask = np.zeros(200, dtype=bool)
    g, loss = N.mlp_gradient(p, x, y, mask)
    assert loss == 0.0 and not np.any(g)


def _american(continuation, units=1 << 16, dates=10):
    spec, lsm = W.american_bs(dates=dates, units=units)
    lsm.continuation = continuation
    lsm.mlp_seed = 7
    return spec, lsm


def test_learned_policy_beats_the_polynomial_policy_against_the_tree(engine):
    tree = bermudan_equally_spaced(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 10, steps=5000)
    spec, lsm = _american(A.CONTINUATION_POLYNOMIAL)
    plain = N.lsm_price(spec, lsm).result
    spec, lsm = _american(A.CONTINUATION_MLP)
    learned = N.lsm_price(spec, lsm).result
    info = (f"tree {tree} plain {plain.price.value} learned {learned.price.value} +- "
            f"{learned.price.standard_error} in-sample mlp {learned.mlp_in_sample} poly "
            f"{learned.polynomial_in_sample} loss {learned.mlp_final_loss} steps {learned.mlp_steps}")
    assert learned.continuation_used == A.CONTINUATION_MLP, info
    assert learned.mlp_steps > 0 and np.isfinite(learned.mlp_final_loss), info
    # the same training paths give the same polynomial fit in both runs
    assert learned.polynomial_in_sample == plain.in_sample_value, info
    err_plain = abs(plain.price.value - tree)
    err_learned = abs(learned.price.value - tree)
    assert err_learned < err_plain, info
    assert err_learned < 4.0 * learned.price.standard_error + 0.03, info


def test_learned_policy_is_reproducible(engine):
    spec, lsm = _american(A.CONTINUATION_MLP, units=1 << 13, dates=5)
    a = N.lsm_price(spec, lsm, stopping=True)
    b = N.lsm_price(spec, lsm, stopping=True)
    assert a.result.price.value == b.result.price.value
    assert list(a.stops) == list(b.stops)
    assert list(a.mlp_params) == list(b.mlp_params)


def test_learned_policy_values_what_it_trained_at_fifty_dates(engine):
    # The valuation applies, date by date, the weights each date was decided
    # with in training, so out-of-sample and in-sample values agree closely.
    tree = bermudan_equally_spaced(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 50, steps=5000)
    spec, lsm = _american(A.CONTINUATION_MLP, units=1 << 16, dates=50)
    r = N.lsm_price(spec, lsm).result
    info = f"tree {tree} price {r.price.value} +- {r.price.standard_error} in-sample {r.mlp_in_sample}"
    assert r.continuation_used == A.CONTINUATION_MLP, info
    assert abs(r.price.value - r.mlp_in_sample) < 4.0 * r.price.standard_error + 0.05, info
    assert abs(r.price.value - tree) < 4.0 * r.price.standard_error + 0.05, info

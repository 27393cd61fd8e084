"""The batched book on the GPU: many single-product plans in one persistent launch.

Every trade's price must be bit for bit the price of evaluating its plan alone
(the book runs the same per-tile path code and the same tile reduction), with
or without the autotuner and the captured CUDA graph; a few trades are also
checked against the oracle, and creation rejects trades a book cannot hold.
"""
import pytest

import gpu_common as G
import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_book(trades=24, units=1 << 11, seed=11):
    return W.batched_book(G.gpu_grid, trades=trades, units=units, seed=seed)


def alone(spec):
    with N.Plan(spec) as plan:
        return plan.evaluate().products[0].price


@pytest.mark.parametrize("autotune,graph,tpi,cps", [(True, True, 0, 0), (False, False, 1, 1), (False, True, 16, 0)])
def test_each_trade_equals_its_plan_alone(engine, autotune, graph, tpi, cps):
    specs = small_book()
    kinds = {(s.model, s.products[0].kind) for s in specs}
    assert len(kinds) >= 6  # the sample covers both models and most products
    with N.Book(specs, autotune=autotune, tiles_per_item=tpi, ctas_per_sm=cps, use_graph=graph) as book:
        prices, report = book.evaluate()
    assert report.trade_count == len(specs) and report.graph == int(graph)
    for i, spec in enumerate(specs):
        want = alone(spec)
        got = prices[i]
        assert (got.value, got.standard_error, got.effective_sampling_units) == (
            want.value, want.standard_error, want.effective_sampling_units), i


def test_repeatable_and_matches_the_oracle(engine):
    specs = small_book(trades=12, units=1 << 10, seed=5)
    with N.Book(specs) as book:
        a, _ = book.evaluate()
        b, report = book.evaluate()
    assert [x.value for x in a] == [x.value for x in b]
    assert report.path_steps > 0 and report.items >= len(specs)
    for i in (0, 3, 7, 11):
        want = H.oracle_evaluate(specs[i]).products[0].price
        assert abs(a[i].value - want.value) <= G.DIRECT_TOL * max(abs(want.value), want.standard_error, 1e-300), i


def test_rejects_what_a_book_cannot_hold(engine):
    specs = small_book(trades=4, units=1 << 10)
    specs[1].sampling_units = 1 << 11
    with pytest.raises(N.EngineError) as err:
        N.Book(specs)
    assert err.value.name == "invalid_argument"
    specs = small_book(trades=4, units=1 << 10)
    specs[2].request_delta = True
    with pytest.raises(N.EngineError) as err:
        N.Book(specs)
    assert err.value.name == "unsupported"


@pytest.mark.parametrize("tpi", [1, 3])
def test_ragged_tiles_equal_their_plans_alone(engine, tpi):
    """An odd tile count with a partial last tile: the two-path family pairs
    tiles from even first tiles (odd tiles per item are rounded up to even)."""
    specs = W.batched_book(G.gpu_grid, trades=16, units=1100, seed=3)
    with N.Book(specs, autotune=False, tiles_per_item=tpi) as book:
        prices, report = book.evaluate()
    assert report.kernel_launches >= 2
    for i, spec in enumerate(specs):
        want = alone(spec)
        assert (prices[i].value, prices[i].standard_error) == (want.value, want.standard_error), i

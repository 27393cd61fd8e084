"""The no-allocation entry point, mcg_price_european_noalloc, on a GPU.

Some callers cannot allocate GPU memory while they price: a service that hands
the whole device to its own memory pool at start-up, a host held to a fixed
device-memory budget, or a latency-bound caller that cannot take the
device-wide synchronisation of cudaFree/cudaMalloc.  For them the library keeps
the kernels' scratch in one static device array, and this entry point prices a
European or Digital Black--Scholes product without a single allocation.

Each test calls it twice in a row through the C ABI and compares both results
with the ordinary entry point, mcg_price, on the same descriptor, within the
tolerances of the parity tests.  The file sorts last so that a run stopping at
its first failure has already run every other test; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

import gpu_common as G
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W
from rust_pricing_b200.desc import ProductSpec

pytestmark = pytest.mark.gpu


def price(entry, spec):
    buf = A.ResultBuffers(1)
    desc = spec.desc()
    status = entry(C.byref(desc), C.c_void_p(0), C.byref(buf.result))
    N.check(status, buf.result.error)
    return buf


def assert_same(spec, got, want):
    """Every component within the parity tolerances (they are in fact equal)."""
    for err, k, c, a, b in G.component_errors(spec, got, want):
        tol = G.BUMP_TOL if c in G.BUMP_COMPONENTS else G.DIRECT_TOL
        assert err <= tol, f"component {c}: {a!r} vs {b!r}"
    for f in ("price", "delta", "gamma", "vega"):
        x, y = getattr(got.products[0], f), getattr(want.products[0], f)
        assert abs(x.value - y.value) <= G.DIRECT_TOL * max(abs(y.value), y.standard_error)
        assert x.effective_sampling_units == y.effective_sampling_units
    assert got.result.independent_sampling_units == want.result.independent_sampling_units
    assert got.result.evaluated_paths == want.result.evaluated_paths


CASES = {
    "pseudo-full-risk": lambda: W.european_bs(paths=1 << 16),
    "pseudo-antithetic-odd-units": lambda: W.european_bs(paths=70001, antithetic=True),
    "rqmc-full-risk": lambda: W.european_bs(paths=1 << 12, engine=A.ENGINE_RQMC, antithetic=True, scrambles=16),
    "digital-smoothed-price": lambda: _digital(),
}


def _digital():
    spec = W.european_bs(paths=1 << 15, risk=False)
    spec.products = [ProductSpec(kind=A.PRODUCT_DIGITAL, side=A.PUT, payout=2.0)]
    spec.smoothing_half_width = 0.5
    return spec


@pytest.mark.parametrize("name", sorted(CASES))
def test_matches_the_allocating_entry_point_twice(engine, name):
    spec = CASES[name]()
    want = price(engine.mcg_price, spec)
    first = price(engine.mcg_price_european_noalloc, spec)
    second = price(engine.mcg_price_european_noalloc, spec)
    assert_same(spec, first, want)
    assert_same(spec, second, want)


def test_rejects_requests_beyond_the_scratch_limit(engine):
    spec = W.european_bs(paths=(1 << 20) + 1)
    with pytest.raises(N.EngineError) as err:
        price(engine.mcg_price_european_noalloc, spec)
    assert err.value.name == "invalid_argument"
    assert "2^20" in str(err.value)
    spec = W.european_bs(paths=1 << 10, engine=A.ENGINE_RQMC, scrambles=65)
    with pytest.raises(N.EngineError):
        price(engine.mcg_price_european_noalloc, spec)


def test_rejects_what_it_does_not_price(engine):
    spec = W.european_bs(paths=1024)
    spec.products = [ProductSpec(kind=A.PRODUCT_ASIAN, weights=[1.0])]
    with pytest.raises(N.EngineError) as err:
        price(engine.mcg_price_european_noalloc, spec)
    assert err.value.name == "unsupported"


def test_rejects_what_plan_create_rejects(engine):
    """The same descriptor checks as mcg_plan_create: a non-finite discount
    factor is a market error, a seasoned state on a terminal product is
    unsupported -- for both entry points."""
    spec = W.european_bs(paths=1024)
    spec.discount_factors = (1.0, float("inf"))
    for entry in (engine.mcg_price, engine.mcg_price_european_noalloc):
        with pytest.raises(N.EngineError) as err:
            price(entry, spec)
        assert err.value.name == "market"
    spec = W.european_bs(paths=1024)
    spec.products[0].initial_state = 0.0  # has_initial_state set
    for entry in (engine.mcg_price, engine.mcg_price_european_noalloc):
        with pytest.raises(N.EngineError) as err:
            price(entry, spec)
        assert err.value.name == "unsupported"

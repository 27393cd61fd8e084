"""The local-volatility adjoint kernel against the oracle: Vega, adjoint Delta,
bumped-adjoint Gamma and the grid-node sensitivities, plus the checkpoint tape
contract (paths recomputed from per-step states, not stored per step object)."""
import numpy as np
import pytest

import helpers as H
import gpu_common as G
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W
from rust_pricing_b200.desc import ProductSpec

pytestmark = pytest.mark.gpu


def _spec(paths=1024, smoothing=0.5, antithetic=False, nodes=True, product=None, engine=A.ENGINE_PSEUDO):
    spec = W.local_vol_adjoint(G.gpu_grid, paths=paths, smoothing=smoothing)
    spec.request_vega = True
    spec.request_local_vega_nodes = nodes
    spec.antithetic = antithetic
    spec.engine = engine
    spec.scramble_count = 4
    if product is not None:
        spec.products = [product]
    return spec


def _check(spec):
    eng = G.run_engine(spec)
    ora = H.oracle_evaluate(spec, 8)
    G.assert_parity(spec, engine_buf=eng, oracle_buf=ora)
    a, b = ora.products[0], eng.products[0]
    for f in ("adjoint_delta", "adjoint_gamma"):
        x, y = getattr(a, f), getattr(b, f)
        assert abs(x.value - y.value) <= 1e-11 * max(abs(x.value), x.standard_error), f
    for c in range(2):
        x, y = a.adjoint_components[c], b.adjoint_components[c]
        assert abs(x.sum + x.correction - (y.sum + y.correction)) <= 1e-11 * max(
            abs(x.sum + x.correction), (x.second_moment * x.count) ** 0.5)
    if spec.request_local_vega_nodes:
        nv = spec.grid_value_count()
        om = np.array([ora.node_stats[k].sum + ora.node_stats[k].correction for k in range(nv)])
        em = np.array([eng.node_stats[k].sum + eng.node_stats[k].correction for k in range(nv)])
        assert np.max(np.abs(om - em)) <= 1e-11 * np.max(np.abs(om))
        # node sensitivities add up to the scalar Vega
        assert abs(em.sum() - (b.components[A.VEGA].sum + b.components[A.VEGA].correction)) <= 1e-9 * abs(em.sum())
    return eng, ora


@pytest.mark.parametrize("smoothing", [0.0, 0.5])
@pytest.mark.parametrize("antithetic", [False, True])
def test_continuous_barrier_adjoint(engine, smoothing, antithetic):
    _check(_spec(smoothing=smoothing, antithetic=antithetic))


@pytest.mark.parametrize("product", [
    ProductSpec(kind=A.PRODUCT_EUROPEAN), ProductSpec(kind=A.PRODUCT_DIGITAL, side=A.PUT),
    ProductSpec(kind=A.PRODUCT_ASIAN, weights=[1.0 / 252] * 252), ProductSpec(kind=A.PRODUCT_LOOKBACK),
    ProductSpec(kind=A.PRODUCT_DISCRETE_BARRIER, barrier=85.0, rebate=1.0)], ids=lambda p: str(p.kind))
def test_discrete_products_adjoint(engine, product):
    _check(_spec(paths=700, smoothing=0.0, product=product))


def test_rqmc_adjoint_and_nodes(engine):
    spec = _spec(paths=512, engine=A.ENGINE_RQMC)
    _check(spec)


def test_vega_without_nodes(engine):
    _check(_spec(nodes=False))

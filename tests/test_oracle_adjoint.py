"""The oracle's local-volatility adjoint against central finite differences.

Per path, the adjoint spot Delta (the reverse sweep's initial-state adjoint
plus the forward-normaliser term) must equal the CRN central bump of the
reference's bumped runtimes (crates/pricing/src/engine/processes/local_vol_valuation.rs:24-68)
with a small bump, up to O(h^2).
"""
import numpy as np
import pytest

import helpers as H
import gpu_common as G
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import workloads as W
from rust_pricing_b200.desc import ProductSpec


@pytest.mark.parametrize("product,smoothing", [
    (ProductSpec(kind=A.PRODUCT_EUROPEAN), 0.0),
    (ProductSpec(kind=A.PRODUCT_ASIAN, weights=[1.0 / 63] * 63), 0.0),
    (None, 0.5),
])
def test_adjoint_delta_equals_crn_bump(oracle, product, smoothing):
    surface = W.SsviSurface(steps=63, expiries=21)
    spec = W.local_vol_adjoint(G.oracle_grid, paths=200, steps=63, smoothing=smoothing, surface=surface)
    if product is not None:
        spec.products = [product]
    spec.request_vega = True
    spec.gamma_bump = 1e-4
    desc = spec.desc()
    out = np.zeros(20)
    diffs = []
    for unit in range(200):
        assert oracle.oracle_unit_values(desc, 0, unit, H.dptr(out)) == 0
        diffs.append(out[18] - out[A.DELTA])
    diffs = np.abs(np.array(diffs))
    assert np.median(diffs) < 1e-8
    assert np.mean(diffs) < 2e-6

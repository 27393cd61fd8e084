"""The FP32 path bulk (MCG_PRECISION_F32_BULK) against the FP64 path.

Same plan, same Sobol words: the local-vol RQMC workload's Asian call and
discrete down-and-out call (SSVI -> Dupire grid, 252 daily steps, Brownian
bridge) priced with the state evolved in FP32.  The stated error of the FP32
bulk is F32_TOL relative to the FP64 price (measured 6.0e-6 and 6.8e-6 at
2^20 x 16 and at 2^14 x 4 points).  At the benchmark's 2^20 x 16 points the
FP64 standard errors are 5.2e-6 (Asian) and 3.8e-5 (barrier) relative, so
1e-5 bounds the FP32 bias by about two standard errors there; the measured
bias is 1.16 and 0.18 of them.  Its standard errors agree with the FP64 ones
to 1 %.
"""
import pytest

import gpu_common as G
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W

pytestmark = pytest.mark.gpu

F32_TOL = 1e-5


def run(precision, points=1 << 14, scrambles=4, antithetic=False):
    spec = W.local_vol_rqmc(G.gpu_grid, points=points, scrambles=scrambles)
    spec.precision = precision
    spec.antithetic = antithetic
    with N.Plan(spec) as plan:
        return plan.evaluate()


@pytest.mark.parametrize("antithetic", [False, True])
def test_fp32_bulk_within_stated_error_of_fp64(engine, antithetic):
    a = run(A.PRECISION_F64, antithetic=antithetic)
    b = run(A.PRECISION_F32_BULK, antithetic=antithetic)
    for k in range(2):
        pa, pb = a.products[k].price, b.products[k].price
        assert abs(pb.value - pa.value) <= F32_TOL * abs(pa.value), (k, pa.value, pb.value)
        assert abs(pb.standard_error - pa.standard_error) <= 0.01 * pa.standard_error


def test_fp32_bulk_is_repeatable(engine):
    a = run(A.PRECISION_F32_BULK, points=1 << 12, scrambles=2)
    b = run(A.PRECISION_F32_BULK, points=1 << 12, scrambles=2)
    assert [a.products[k].price.value for k in range(2)] == [b.products[k].price.value for k in range(2)]


def test_fp32_bulk_rejects_risk_and_black_scholes(engine):
    spec = W.local_vol_rqmc(G.gpu_grid, points=1 << 10, scrambles=2)
    spec.precision = A.PRECISION_F32_BULK
    spec.request_delta = True
    with pytest.raises(N.EngineError) as err:
        N.Plan(spec)
    assert err.value.name == "unsupported"
    spec = W.european_bs(paths=1 << 10)
    spec.precision = A.PRECISION_F32_BULK
    with pytest.raises(N.EngineError) as err:
        N.Plan(spec)
    assert err.value.name == "unsupported"

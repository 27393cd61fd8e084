"""B200 Monte Carlo pricing engine: the host side above the C ABI (include/mcg.h).

Mirrors the reference's Python facade `rust_pricing.PricingPlan`
(crates/pricing-python/src/lib.rs:347-388): `PricingRequest.from_json`,
`PricingPlan.compile(request, worker_threads=...)` then `.evaluate()`
(`facade.py`, over the v3 wire format of `wire.py`); `desc.PlanSpec` builds
engine plans directly.  Pricing always runs on the GPU through libmcg.so.
"""
from . import _abi  # noqa: F401
from .desc import LocalVarianceSpec, PlanSpec, ProductSpec  # noqa: F401
from .facade import PricingError, PricingPlan, PricingRequest, PricingResult, ValidationError  # noqa: F401

__version__ = "0.1.0+b200"

__all__ = ["PlanSpec", "ProductSpec", "LocalVarianceSpec", "PricingRequest", "PricingPlan", "PricingResult",
           "ValidationError", "PricingError"]

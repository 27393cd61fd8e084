"""B200 Monte Carlo pricing engine: the host side above the C ABI (include/mcg.h).

Mirrors the reference's Python facade `rust_pricing.PricingPlan`
(crates/pricing-python/src/lib.rs:347-388): `PricingPlan.compile(request)`
then `.evaluate()`.  Pricing always runs on the GPU through libmcg.so.
"""
from . import _abi  # noqa: F401
from .desc import LocalVarianceSpec, PlanSpec, ProductSpec  # noqa: F401

__all__ = ["PlanSpec", "ProductSpec", "LocalVarianceSpec"]

"""The reference's Python facade over this engine: `PricingRequest.from_json`,
`PricingPlan.compile(request, *, worker_threads, reduction_block_size=None)`,
`PricingPlan.evaluate()` -> `PricingResult` with `to_json()`
(crates/pricing-python/src/lib.rs:277-330,347-400), and
`PricingPlan.evaluate_width_ladder()` (crates/pricing/src/engine/risk/pricing.rs:329).

A compiled plan owns its engine plan (mcg_plan_create once, mcg_plan_evaluate
per call); an American request keeps its plan and LSM configuration and is
trained and valued by mcg_lsm_price on every evaluation.  `worker_threads`
is accepted for the reference's signature: the GPU does not use host threads.
"""
from __future__ import annotations

import json
from typing import Optional

from . import wire


class ValidationError(ValueError):
    """A request that does not compile (the reference's validation exception)."""


class PricingError(RuntimeError):
    """An evaluation that failed on the engine (the reference's pricing exception)."""


class PricingRequest:
    def __init__(self, document: dict):
        self.document = document

    @staticmethod
    def from_json(text: str) -> "PricingRequest":
        try:
            doc = json.loads(text)
        except json.JSONDecodeError as exc:
            raise ValidationError(str(exc)) from exc
        if not isinstance(doc, dict):
            raise ValidationError("a pricing request is a JSON object")
        return PricingRequest(doc)

    def to_json(self) -> str:
        return json.dumps(self.document, sort_keys=True)

    def fingerprint(self) -> str:
        return wire.request_fingerprint(self.document)


class PricingResult:
    def __init__(self, document: dict):
        self.document = document

    @property
    def value(self) -> dict:
        return self.document["value"]

    @property
    def risks(self) -> dict:
        return self.document["risks"]

    def to_json(self) -> str:
        return json.dumps(self.document, sort_keys=True)


class PricingPlan:
    def __init__(self, request: PricingRequest, compiled: wire.CompiledRequest, reduction_block_size: int):
        self.request = request
        self.compiled = compiled
        self.reduction_block_size = reduction_block_size
        self._plan = None

    @staticmethod
    def compile(request: PricingRequest, *, worker_threads: int,
                reduction_block_size: Optional[int] = None) -> "PricingPlan":
        if worker_threads < 1:
            raise ValidationError("worker_threads must be positive")
        block = 4096 if reduction_block_size is None else int(reduction_block_size)
        if block < 1:
            raise ValidationError("reduction_block_size must be positive")
        doc = request.document
        if (doc.get("risk") or {}).get("payoff_smoothing_width_ladder"):
            # the ladder is evaluated by evaluate_width_ladder; the plan itself
            # prices the primary request
            doc = wire.json_copy(doc)
            wire.width_ladder(doc)
            del doc["risk"]["payoff_smoothing_width_ladder"]
        try:
            compiled = wire.compile_request(doc, reduction_block_size=block)
        except wire.WireError as exc:
            raise ValidationError(str(exc)) from exc
        return PricingPlan(request, compiled, block)

    def evaluate(self) -> PricingResult:
        from . import _native as N
        c = self.compiled
        try:
            if c.lsm is not None:
                r = N.lsm_price(c.plan, c.lsm).result
                doc = wire.result_document(c, r.price, r.delta, r.gamma, r.vega, r.sampling_variance,
                                           r.estimator_variance, r.valuation_paths, request=self.request.document)
                return PricingResult(doc)
            if self._plan is None:
                self._plan = N.Plan(c.plan)
            buf = self._plan.evaluate()
        except N.EngineError as exc:
            raise PricingError(str(exc)) from exc
        p, r = buf.products[0], buf.result
        kt = None
        if c.vega_kt is not None:
            kt = wire._vega_kt_report(c, [e.value for e in buf.node_estimates], r.evaluated_paths)
        return PricingResult(wire.result_document(c, p.price, p.delta, p.gamma, p.vega, p.sampling_variance,
                                                  p.estimator_variance, r.evaluated_paths, kt,
                                                  request=self.request.document))

    def evaluate_width_ladder(self) -> dict:
        try:
            return wire.evaluate_width_ladder(self.request.document,
                                              reduction_block_size=self.reduction_block_size)
        except wire.WireError as exc:
            raise ValidationError(str(exc)) from exc

    def request_fingerprint(self) -> str:
        return wire.request_fingerprint(self.request.document)

    def close(self) -> None:
        if self._plan is not None:
            self._plan.close()
            self._plan = None

"""Replay requests of the reference's fixtures as v3 documents, and the checks
of a `pricing_result` document against a fixture's expected values.

tests/golden/replay_path_dependence.json holds the verbatim requests of
fixtures/replay/path_dependence-{windows-x86_64,macos-aarch64}.json (digital,
discrete and continuous barrier, arithmetic Asian with a known fixing, fixed
lookback with a historical extremum; Black--Scholes, pseudo-MC and RQMC,
exact and compact-C2 smoothed, price-only and full risk) with both platforms'
results.
"""
import json
import os
import struct

import helpers as H

ESTIMATE_KEYS = ("value", "standard_error", "confidence_lower", "confidence_upper")
PLATFORMS = ("windows-x86_64", "macos-aarch64")


def bits(x: float) -> str:
    return struct.pack(">d", x).hex()


def path_dependence_cases():
    return json.load(open(os.path.join(H.GOLDEN, "replay_path_dependence.json")))["cases"]


def _rel(a: float, b: float) -> float:
    return abs(a - b) / max(abs(b), 1e-300)


def estimate_errors(got: dict, want: dict) -> tuple:
    """Largest relative differences of (value and bounds, standard error).
    The bounds are value -/+ 1.96 standard errors, so they are scaled by the
    larger of themselves and the standard error."""
    assert got["effective_sampling_units"] == want["effective_sampling_units"]
    se = want["standard_error"]
    value = max(abs(got[k] - want[k]) / max(abs(want[k]), se, 1e-300)
                for k in ("value", "confidence_lower", "confidence_upper"))
    return value, _rel(got["standard_error"], se) if se else abs(got["standard_error"])


def document_errors(doc: dict, expected: dict) -> tuple:
    """Largest relative differences of a result document's value and risk
    estimates (raw and market-scaled) from one platform's expected values."""
    worst = estimate_errors(doc["value"], expected["value"])
    assert set(doc["risks"]) == set(expected["risks"]), (set(doc["risks"]), set(expected["risks"]))
    for name, want in expected["risks"].items():
        got = doc["risks"][name]
        assert got["raw_unit"]["type"] == want["raw_unit"]
        assert got["market_scaled_unit"]["type"] == want["market_scaled_unit"]
        for e in (estimate_errors(got["raw"], want["raw"]), estimate_errors(got["market_scaled"], want["market_scaled"])):
            worst = (max(worst[0], e[0]), max(worst[1], e[1]))
    return worst


def assert_matches_fixture(doc: dict, case: dict, rel: float, price_bits: bool, se_rel: float | None = None):
    """Every value and bound within `rel` and every standard error within
    `se_rel` (default `rel`) of the nearer platform; with `price_bits`, the
    price and the sampling variance equal one platform's to the last bit (the
    reference's own platforms differ in the last bits of some risks)."""
    se_rel = rel if se_rel is None else se_rel
    errors = {p: document_errors(doc, case["expected"][p]) for p in PLATFORMS}
    best = min(errors, key=lambda p: errors[p][0])
    assert errors[best][0] <= rel and errors[best][1] <= se_rel, (case["name"], errors)
    if price_bits:
        mc = doc["monte_carlo"]
        assert any(doc["value"]["value"] == case["expected"][p]["value"]["value"]
                   and bits(mc["sampling_variance"]) == case["expected"][p]["sampling_variance_bits"]
                   for p in PLATFORMS), (case["name"], doc["value"], bits(mc["sampling_variance"]))
    assert int(doc["monte_carlo"]["evaluated_paths"]) == case["expected"][best]["evaluated_paths"]
    assert doc["monte_carlo"]["independent_sampling_units"] == case["expected"][best]["independent_sampling_units"]

"""The v3 wire format: request documents compiled to plans, and result documents.

* Every replay request of the reference's fixtures (European BS, local
  volatility with VegaKT, early exercise, path-dependent products) compiles to
  the plan the hand-mapped tests use: the oracle gives the same bits on both.
* The path-dependence requests, compiled by the wire module and run on the
  oracle, reproduce fixtures/replay/path_dependence-*.json through the result
  document: value and sampling variance to the last bit on one platform, every
  raw and market-scaled risk estimate within 1e-12 relative.
* Seasoned products: known Asian fixings, a lookback's historical extremum and
  valuation-date fixing, a barrier's historical hit and an unmonitored expiry
  become the plan's seasoned state and monitoring flags.
* Requests off the engine's path raise UnsupportedRequest; malformed ones WireError.
"""
import copy
import math
import struct

import pytest

import helpers as H
import lsm_cases as LC
import lv_cases as LV
import wire_cases as WC
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import wire
from test_oracle_fixtures import replay_cases, replay_spec


def bits(x: float) -> str:
    return struct.pack(">d", x).hex()


def oracle_document(req, threads=4):
    buf = H.oracle_evaluate(req.plan, threads=threads)
    p, r = buf.products[0], buf.result
    return wire.result_document(req, p.price, p.delta, p.gamma, p.vega, p.sampling_variance,
                                p.estimator_variance, r.evaluated_paths), buf


def same_estimates(a, b):
    for name in ("price", "delta", "gamma", "vega", "bump_delta", "bump_gamma", "bump_vega"):
        x, y = getattr(a, name), getattr(b, name)
        assert (bits(x.value), bits(x.standard_error)) == (bits(y.value), bits(y.standard_error)), name
    assert bits(a.sampling_variance) == bits(b.sampling_variance)


@pytest.mark.parametrize("case", WC.path_dependence_cases(), ids=lambda c: c["name"])
def test_path_dependence_replay_through_the_wire(case):
    req = wire.compile_request(case["request"], reduction_block_size=case["reduction_block_size"])
    doc, _ = oracle_document(req)
    WC.assert_matches_fixture(doc, case, rel=1e-12, price_bits=True)


@pytest.mark.parametrize("case", replay_cases(), ids=lambda c: c["name"])
def test_european_replay_request_compiles_to_the_replay_plan(case):
    req = wire.compile_request(case["request"], reduction_block_size=case["reduction_block_size"])
    a = H.oracle_evaluate(req.plan, threads=4).products[0]
    b = H.oracle_evaluate(replay_spec(case), threads=4).products[0]
    same_estimates(a, b)
    e = case["expected"]
    doc = wire.result_document(req, a.price, a.delta, a.gamma, a.vega)
    assert doc["value"]["value"] == e["price"]
    assert doc["risks"]["vega"]["raw"]["value"] == e["vega"]
    assert doc["risks"]["vega"]["market_scaled"]["value"] == e["vega"] * 0.01


@pytest.mark.parametrize("case", LV.cases(), ids=lambda c: c["name"])
def test_local_vol_replay_request_compiles_to_the_replay_plan(case):
    req = wire.compile_request(case["request"], reduction_block_size=case["reduction_block_size"])
    hand = LV.plan(case)
    assert req.plan.model == A.MODEL_LOCAL_VOLATILITY
    assert list(req.plan.local_variance.values) == list(hand.local_variance.values)
    assert req.plan.observation_times == hand.observation_times
    assert req.plan.request_local_vega_nodes == ("vega_kt" in case)
    req.plan.request_local_vega_nodes = False
    a = H.oracle_evaluate(req.plan, threads=4).products[0]
    b = H.oracle_evaluate(hand, threads=4).products[0]
    same_estimates(a, b)
    if "vega_kt" in case:
        # The basis forwards the wire module computes equal the tests' own.
        basis = LV.vega_kt_basis(case)
        maturities = req.vega_kt["reporting_iv_basis"]["maturity_nodes"]
        fwd = [req.plan.spot * math.exp(
            wire.log_discount(req.plan.dividend_times, req.plan.dividend_factors, t)
            - wire.log_discount(req.plan.discount_times, req.plan.discount_factors, t)) for t in maturities]
        assert fwd == list(basis.arrays[3])


@pytest.mark.parametrize("case", LC.cases(), ids=lambda c: c["name"])
def test_early_exercise_replay_request_compiles_to_the_replay_plan(case):
    req = wire.compile_request(case["request"], reduction_block_size=case["reduction_block_size"])
    spec, lsm = LC.plan(case)
    assert req.lsm is not None
    assert req.plan.observation_times == spec.observation_times
    got = H.oracle_lsm(req.plan, req.lsm, threads=3).result
    want = H.oracle_lsm(spec, lsm, threads=3).result
    assert bits(got.price.value) == bits(want.price.value)
    assert bits(got.sampling_variance) == bits(want.sampling_variance)
    assert got.price.value == case["expected"]["value"]["value"]


# ------------------------------------------------------------ seasoned state

def _case(name):
    return copy.deepcopy(next(c for c in WC.path_dependence_cases() if c["name"] == name)["request"])


def test_asian_known_fixings_are_the_seasoned_sum():
    doc = _case("arithmetic_asian_full_risk")
    obs = doc["product"]["observations"]
    req = wire.compile_request(doc)
    p = req.plan.products[0]
    assert p.kind == A.PRODUCT_ASIAN
    assert p.initial_state == 0.0 + 98.0 * 0.2
    assert p.weights == [0.3, 0.5]
    assert req.observation_dates == [o["date"] for o in obs[1:]]
    # A known fixing after the valuation date is rejected (request.rs:136).
    bad = copy.deepcopy(doc)
    bad["product"]["observations"][1]["value"] = {"type": "known", "fixing": 100.0}
    with pytest.raises(wire.WireError):
        wire.compile_request(bad)
    bad = copy.deepcopy(doc)
    bad["product"]["observations"][0]["value"] = {"type": "unknown"}
    with pytest.raises(wire.WireError):
        wire.compile_request(bad)


def test_lookback_history_and_valuation_date_fixing():
    doc = _case("fixed_lookback_full_risk")
    req = wire.compile_request(doc)
    assert req.plan.products[0].initial_state == 105.0
    doc["product"]["monitoring_dates"] = ["2026-06-04", "2026-09-04", "2027-03-05", "2027-09-04"]
    doc["product"]["valuation_date_fixing"] = 107.5
    req = wire.compile_request(doc)
    assert req.plan.products[0].initial_state == 107.5  # Maximum(105, 107.5)
    assert len(req.plan.observation_times) == 2
    doc["product"]["side"] = {"type": "put"}
    assert wire.compile_request(doc).plan.products[0].initial_state == 105.0  # Minimum
    # Without the fixing, the valuation-date monitoring is a time-zero observation
    # (Black-Scholes only: a zero-length step that still takes its normal).
    del doc["product"]["valuation_date_fixing"]
    req = wire.compile_request(doc)
    assert req.plan.observation_times[0] == 0.0 and len(req.plan.observation_times) == 3
    lv = copy.deepcopy(doc)
    lv["model"] = {"type": "local_volatility", "local_variance_grid": {
        "time_nodes": [0.0, 1.0], "log_forward_moneyness_nodes": [-1.0, 1.0], "shape": [2, 2],
        "values": [0.04] * 4, "floor": 1e-8, "cap": 4.0}}
    with pytest.raises(wire.UnsupportedRequest):
        wire.compile_request(lv)
    doc["product"].pop("historical_extremum")
    with pytest.raises(wire.WireError):
        wire.compile_request(doc)


def test_barrier_history_and_unmonitored_expiry():
    doc = _case("discrete_barrier_smoothed_full_risk")
    doc["product"]["monitoring_dates"] = ["2026-06-04", "2027-03-05"]
    doc["product"]["historical_hit"] = False
    req = wire.compile_request(doc)
    p = req.plan.products[0]
    assert p.initial_state == 0.0
    assert p.weights == [1.0, 0.0]  # the expiry observes the payoff but not the barrier
    assert len(req.plan.observation_times) == 2
    doc["product"]["historical_hit"] = True
    assert wire.compile_request(doc).plan.products[0].initial_state == 1.0
    del doc["product"]["historical_hit"]
    with pytest.raises(wire.WireError):
        wire.compile_request(doc)


def test_oracle_honours_seasoned_state_and_flags():
    """A barrier hit before valuation is knocked out for good; an unmonitored
    observation leaves a barrier alone; a lookback whose historical extremum
    is out of reach pays it."""
    doc = _case("discrete_barrier_smoothed_full_risk")
    doc["product"]["monitoring_dates"] = ["2026-06-04", "2027-03-05", "2027-09-04"]
    doc["product"]["historical_hit"] = True
    doc["risk"] = {"delta": False, "vega": False, "smile_dynamics": {"type": "sticky_log_moneyness"}}
    req = wire.compile_request(doc, reduction_block_size=256)
    out, _ = oracle_document(req)
    df = req.plan.discount_factors[-1]
    assert out["value"]["value"] == pytest.approx(2.0 * df, rel=1e-15)  # the rebate on every path
    assert out["value"]["standard_error"] == 0.0
    doc = _case("fixed_lookback_full_risk")
    doc["product"]["historical_extremum"] = 1e6
    doc["risk"] = {"delta": True, "vega": True, "smile_dynamics": {"type": "sticky_log_moneyness"}}
    req = wire.compile_request(doc, reduction_block_size=256)
    out, _ = oracle_document(req)
    assert out["value"]["value"] == pytest.approx((1e6 - 100.0) * df, rel=1e-14)
    assert out["risks"]["delta"]["raw"]["value"] == 0.0
    assert out["risks"]["vega"]["raw"]["value"] == 0.0


# ----------------------------------------------------------------- errors

@pytest.mark.parametrize("edit, error", [
    (lambda d: d.update(document_kind="pricing_result"), wire.WireError),
    (lambda d: d.update(schema_version=4), wire.UnsupportedRequest),
    (lambda d: d["market"].update(discrete_dividends=[{"event_id": 1, "ex_time": 0.5,
                                                        "quote": {"type": "proportional", "beta": 1.0}}]),
     wire.WireError),
    (lambda d: d["market"].update(discrete_dividends=[{"event_id": 1, "ex_time": 0.5,
                                                        "quote": {"type": "stock", "amount": 1.0}}]),
     wire.WireError),
    (lambda d: d.update(model={"type": "bass_local_volatility", "parameters": {}}), wire.UnsupportedRequest),
    (lambda d: d["risk"].update(payoff_smoothing_width_ladder=[1.0, 2.0]), wire.UnsupportedRequest),  # ladder entry
    (lambda d: d["product"].update(expiry="2026-09-04", payment_date="2026-09-04"), wire.UnsupportedRequest),  # t = 0 only
    (lambda d: d["product"].update(type="graph"), wire.UnsupportedRequest),
    (lambda d: d.pop("engine"), wire.WireError),
    (lambda d: d.update(lsm={}), wire.WireError),
    (lambda d: d["engine"].update(type="quantum"), wire.WireError),
])
def test_rejected_requests(edit, error):
    doc = _case("digital_exact_price_only")
    edit(doc)
    with pytest.raises(error):
        wire.compile_request(doc)


def test_width_ladder_on_the_oracle():
    """PricingPlan::evaluate_width_ladder: the primary (its own smoothing) and
    one result per half-width in ladder order, each identical to pricing that
    request alone (same seeds: the same random coordinates), with the raw
    differences of adjacent entries."""
    doc = _case("digital_smoothed_full_risk")
    doc["risk"]["payoff_smoothing_width_ladder"] = [4.0, 2.0, 1.0]

    def price(d):
        out, _ = oracle_document(wire.compile_request(d, reduction_block_size=256))
        return out

    ladder = wire.evaluate_width_ladder(doc, price=price)
    plain = copy.deepcopy(doc)
    del plain["risk"]["payoff_smoothing_width_ladder"]
    assert ladder["primary"] == price(plain)
    assert [e["half_width"] for e in ladder["entries"]] == [4.0, 2.0, 1.0]
    assert ladder["entries"][0]["adjacent_difference"] is None
    for prev, cur in zip(ladder["entries"], ladder["entries"][1:]):
        alone = copy.deepcopy(plain)
        alone["risk"]["payoff_smoothing"] = {"type": "compact_c2", "half_width": cur["half_width"]}
        assert cur["result"] == price(alone)
        d = cur["adjacent_difference"]
        assert d["price"] == cur["result"]["value"]["value"] - prev["result"]["value"]["value"]
        assert d["vega"] == cur["result"]["risks"]["vega"]["raw"]["value"] - prev["result"]["risks"]["vega"]["raw"]["value"]
    # the widths smooth the digital differently
    assert ladder["entries"][0]["result"]["value"]["value"] != ladder["entries"][-1]["result"]["value"]["value"]


@pytest.mark.parametrize("ladder", [[], [1.0, 1.0], [1.0, 2.0, 1.5], [-1.0]])
def test_width_ladder_validation(ladder):
    doc = _case("digital_smoothed_full_risk")
    doc["risk"]["payoff_smoothing_width_ladder"] = ladder
    with pytest.raises(wire.WireError):
        wire.width_ladder(doc)


def test_market_scaling_of_risks():
    """report.rs:255-300: Delta x S/100, Gamma x (S/100)^2, Vega / 100, with the
    confidence bounds of the scaled standard error."""
    case = next(c for c in WC.path_dependence_cases() if c["name"] == "arithmetic_asian_full_risk")
    e = case["expected"]["windows-x86_64"]
    req = wire.compile_request(case["request"])

    class Est:
        def __init__(self, d):
            self.__dict__.update(d)

    doc = wire.result_document(req, Est(e["value"]), *(Est(e["risks"][k]["raw"]) for k in ("delta", "gamma", "vega")))
    for k in ("delta", "gamma", "vega"):
        assert doc["risks"][k]["market_scaled"]["value"] == e["risks"][k]["market_scaled"]["value"]
        assert doc["risks"][k]["market_scaled"]["standard_error"] == e["risks"][k]["market_scaled"]["standard_error"]
        assert doc["risks"][k]["market_scaled"]["confidence_lower"] == e["risks"][k]["market_scaled"]["confidence_lower"]
    assert doc["value"]["estimator"] == {"type": "pseudo_monte_carlo"}


def test_request_fingerprints_match_the_reference():
    """fingerprint_request of every replay request equals the fixture's
    request_fingerprint (BLAKE3 over the canonical encoding)."""
    import json as _json
    from rust_pricing_b200.blake3 import blake3
    assert blake3(b"").hex() == "af1349b9f5f9a1a6a0404dea36dcc9499bcb25c9adc112b7cc9a93cae41f3262"
    assert blake3(b"abc").hex() == "6437b3ac38465133ffb63b75273a8db548c558465d79db03fd359c6cd5bd9d85"
    for case in WC.path_dependence_cases():
        assert wire.request_fingerprint(case["request"]) == case["expected"]["windows-x86_64"]["request_fingerprint"]
    # an integer written for a float field canonicalises to the same request
    doc = copy.deepcopy(WC.path_dependence_cases()[0]["request"])
    want = wire.request_fingerprint(doc)
    doc["product"]["strike"] = 100
    assert wire.request_fingerprint(doc) == want
    assert _json.loads(_json.dumps(doc))  # plain JSON


def test_facade_compile_and_validation():
    from rust_pricing_b200 import PricingPlan, PricingRequest, ValidationError
    case = WC.path_dependence_cases()[4]
    req = PricingRequest.from_json(__import__("json").dumps(case["request"]))
    plan = PricingPlan.compile(req, worker_threads=2, reduction_block_size=256)
    assert plan.compiled.plan.reduction_block_size == 256
    assert plan.request_fingerprint() == case["expected"]["windows-x86_64"]["request_fingerprint"]
    with pytest.raises(ValidationError):
        PricingRequest.from_json("[1, 2")
    bad = copy.deepcopy(case["request"])
    bad["market"]["discrete_dividends"] = [{"event_id": 1, "ex_time": 0.5, "quote": {"type": "fixed_cash", "amount": -1.0}}]
    with pytest.raises(ValidationError):
        PricingPlan.compile(PricingRequest(bad), worker_threads=1)


def test_time_zero_observation_on_the_oracle():
    """A lookback monitored from the valuation date (no fixing): the first
    observation is the spot at time zero, a zero-length step that still takes
    its normal, as the reference's path generator does; the oracle prices it
    with finite estimates (the engine's parity is in the GPU tests)."""
    doc = _case("fixed_lookback_full_risk")
    doc["product"]["monitoring_dates"] = ["2026-09-04", "2027-03-05", "2027-09-04"]
    del doc["product"]["historical_extremum"]
    out, buf = oracle_document(wire.compile_request(doc, reduction_block_size=256))
    assert math.isfinite(out["value"]["value"]) and out["value"]["value"] > 0.0
    assert math.isfinite(out["risks"]["vega"]["raw"]["value"])


def test_documents_follow_the_v3_format_goldens():
    """fixtures/v3/*.golden.json: the golden requests compile (European and
    American), and a result document built from the engine's estimates has the
    golden result's sections and field names (value estimate, diagnostics,
    replay with migration)."""
    import json as _json
    import os as _os
    g = _json.load(open(_os.path.join(H.GOLDEN, "wire_v3_documents.json")))
    req = wire.compile_request(g["pricing_request"])
    assert req.product_type == "european_vanilla" and req.plan.sampling_units == 1024 and req.plan.antithetic
    am = wire.compile_request(g["pricing_request_american"])
    assert am.lsm is not None
    out, _ = oracle_document(req)
    out["replay"] = wire.replay_block(g["pricing_request"])
    golden = g["pricing_result"]
    for section in ("document_kind", "schema_version", "value", "risks", "diagnostics", "replay"):
        assert section in out
    assert set(out["value"]) == set(golden["value"])
    assert set(out["replay"]) == set(golden["replay"])
    assert set(out["replay"]["migration"]) == set(golden["replay"]["migration"])
    assert set(out["diagnostics"]) == set(golden["diagnostics"])
    for k, v in g["pricing_result_american"].get("risks", {}).items():
        assert set(v) == {"raw", "market_scaled", "raw_unit", "market_scaled_unit"}


@pytest.mark.parametrize("case", [c for c in LV.cases() if "vega_kt" in c], ids=lambda c: c["name"])
def test_replicable_vega_kt_is_not_reported_by_node_allocation(case):
    """A European under local volatility whose expiry is a reporting maturity:
    the reference reports its VegaKT by terminal replication
    (crates/pricing/src/engine/risk/vegakt_terminal_replication.rs:10-40), so
    the wire layer refuses rather than return the node allocation; with payoff
    smoothing the reference keeps node allocation, and so does the wire layer."""
    req = wire.compile_request(case["request"], reduction_block_size=case["reduction_block_size"])
    assert req.vega_kt["policy"] == wire.TERMINAL_REPLICATION
    with pytest.raises(wire.UnsupportedRequest, match="terminal-replication"):
        wire.price_request(case["request"], reduction_block_size=case["reduction_block_size"])
    smoothed = copy.deepcopy(case["request"])
    smoothed["risk"]["payoff_smoothing"] = {"type": "compact_c2", "half_width": 0.5}
    assert wire.compile_request(smoothed).vega_kt["policy"] == wire.NODE_ALLOCATION
    off_basis = copy.deepcopy(case["request"])
    basis = off_basis["model"]["reporting_iv_basis"]
    basis["maturity_nodes"] = [t for t in basis["maturity_nodes"] if t != 1.0] + [1.5]
    assert wire.compile_request(off_basis).vega_kt["policy"] == wire.NODE_ALLOCATION


def test_discrete_dividends_compile_to_the_plan_schedule():
    """market.discrete_dividends (all three quote types) become the plan's
    escrowed affine schedule; combinations the engine leaves out raise."""
    doc = _case("digital_exact_price_only")
    doc["market"]["discrete_dividends"] = [
        {"event_id": 1, "ex_time": 0.25, "quote": {"type": "fixed_cash", "amount": 1.5}},
        {"event_id": 2, "ex_time": 0.5, "quote": {"type": "proportional", "beta": 0.02}},
        {"event_id": 3, "ex_time": 0.75, "quote": {"type": "fixed_cash_and_proportional", "fixed_cash": 1.0,
                                                  "beta": 0.01}}]
    req = wire.compile_request(doc)
    assert list(req.plan.dividends) == [(0.25, 1.5, 0.0), (0.5, 0.0, 0.02), (0.75, 1.0, 0.01)]
    H.oracle_evaluate(req.plan, threads=2)  # the oracle prices it
    cont = _case("continuous_barrier_smoothed_full_risk") if any(
        c["name"] == "continuous_barrier_smoothed_full_risk" for c in WC.path_dependence_cases()) else None
    if cont is not None:
        cont["market"]["discrete_dividends"] = doc["market"]["discrete_dividends"]
        with pytest.raises(wire.UnsupportedRequest):
            wire.compile_request(cont)


# ----------------------------------------------------------------- schema migrations

def _migration_goldens():
    import json as _json
    import os as _os
    return (_json.load(open(_os.path.join(H.GOLDEN, "wire_migration.json"))),
            _json.load(open(_os.path.join(H.GOLDEN, "wire_v3_documents.json")))["pricing_request"])


@pytest.mark.parametrize("version", [1, 2])
def test_older_schema_documents_migrate_forward(version):
    """crates/pricing/src/wire/tests.rs:423-450: the v1 (and v2) request goldens
    migrate to the v3 golden request, with the migration ids of each step, a
    pre-migration fingerprint (the source document at its own version) that
    differs from the post-migration one, and the post-migration fingerprint
    equal to the v3 golden's; the migrated request compiles to the v3 plan and
    the result's replay block records the provenance."""
    old, v3 = _migration_goldens()
    doc = old[f"v{version}"]
    assert doc["schema_version"] == version
    migrated, prov = wire.migrate_request(copy.deepcopy(doc))
    assert migrated == v3
    assert prov["original_schema_version"] == version and prov["current_schema_version"] == 3
    want_ids = ["pricing_request/v1-to-v2", "pricing_request/v2-to-v3"][version - 1:]
    assert prov["migration_ids"] == want_ids
    assert prov["pre_migration_fingerprint"] != prov["post_migration_fingerprint"]
    assert prov["post_migration_fingerprint"] == wire.request_fingerprint(v3)
    a, b = wire.compile_request(copy.deepcopy(doc)), wire.compile_request(copy.deepcopy(v3))
    same_estimates(H.oracle_evaluate(a.plan, threads=4).products[0], H.oracle_evaluate(b.plan, threads=4).products[0])
    replay = wire.replay_block(doc)
    assert replay["migration"] == prov and replay["request_fingerprint"] == prov["post_migration_fingerprint"]
    assert wire.replay_block(v3)["migration"]["migration_ids"] == []


@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("edit, error", [
    (lambda d: d["product"].update(valuation_date_fixing=100.0), wire.UnsupportedRequest),
    (lambda d: d.update(model={"type": "bass_local_volatility", "parameters": {}}), wire.UnsupportedRequest),
    (lambda d: d["product"].update(type="graph"), wire.UnsupportedRequest),
    (lambda d: d.update(lsm={}), wire.WireError),
])
def test_older_schemas_refuse_what_they_do_not_have(version, edit, error):
    old, _ = _migration_goldens()
    doc = copy.deepcopy(old[f"v{version}"])
    edit(doc)
    with pytest.raises(error):
        wire.migrate_request(doc)


def test_version_one_has_no_width_ladder():
    old, _ = _migration_goldens()
    doc = copy.deepcopy(old["v1"])
    doc["risk"]["payoff_smoothing_width_ladder"] = [0.5, 1.0]
    with pytest.raises(wire.WireError):
        wire.migrate_request(doc)
    doc["schema_version"] = 2
    migrated, _ = wire.migrate_request(doc)
    assert migrated["risk"]["payoff_smoothing_width_ladder"] == [0.5, 1.0]

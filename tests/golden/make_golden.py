"""Extracts golden vectors from the reference's fixtures into tests/golden/.

Run where a checkout of the reference exists, with REFERENCE_ROOT set to its
root (REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py; GPU
machines have no checkout).  The extracted JSON files are committed; the tests
only read them.

* replay_european_bs.json  -- fixtures/replay/european_bs-windows-x86_64.json:
  request parameters and result values of the pseudo and RQMC full-risk cases.

Every replay case also keeps its verbatim v3 request document ("request"),
which the wire-format tests compile.
* bs_analytical.json       -- fixtures/acceptance/european_bs_analytical.csv.
* path_dependence.json     -- fixtures/path-dependence/reference-cases-v0.1.json
  (smoothing, extrema, exact and smoothed bridge cases; decimal strings).
* replay_local_vol.json    -- fixtures/replay/local_volatility-{windows-x86_64,macos-aarch64}.json:
  the 3 x 5 local-variance grid requests (pseudo and RQMC, price-only and
  Delta/Gamma/Vega) with both platforms' values, standard errors and
  variance bits.
* surfaces.json            -- fixtures/local-vol/reference-cases-v0.1.json: the standard SSVI
  (power-law and Heston-like phi), eSSVI interpolation and constant-volatility
  Dupire cases (70-digit decimal values).
* replay_path_dependence.json -- fixtures/replay/path_dependence-{windows-x86_64,macos-aarch64}.json:
  the digital, discrete and continuous barrier, arithmetic Asian and fixed
  lookback requests (verbatim v3 request documents, Black--Scholes, pseudo and
  RQMC, exact and compact-C2 smoothed, price-only and full risk) with both
  platforms' estimates, variance bits and bump-and-revalue validation bits.
* lv_step_adjoints.json     -- fixtures/local-vol/step-adjoints-v0.1.json: one Log-Euler path per
  case (given nodes, forwards, 3 x 3 grid, shocks) with a quadratic payoff, its
  states and 100-digit bump references of the grid-value derivatives.
* lv_direct_variance.json   -- fixtures/local-vol/direct-variance-v0.1.json: continuous barriers
  (up/down, out/in, partial monitoring, touched) on one Log-Euler path with node
  variances, and 100-digit bump references of the grid-value derivatives.
* wire_v3_documents.json    -- fixtures/v3/*.golden.json: the format goldens of a v3 request and
  result (European and American).
* wire_migration.json      -- fixtures/v1/pricing_request.golden.json and
  fixtures/v2/pricing_request.golden.json: the request documents the schema
  migrations carry to v3 (fixtures/v3/pricing_request.golden.json).
* early_exercise_cases.json -- fixtures/early-exercise/reference-cases-v0.1.json: the
  decision, monomial-basis, feature-scaling and CPQR cases (decimal strings).
* early_exercise.json      -- fixtures/replay/early_exercise-windows-x86_64.json:
  the American put requests (pseudo and RQMC, training and valuation engines,
  LSM configuration) with the fitted decision models, exercise counts,
  valuation stopping indices, in-sample value, price and fixed-policy risks.
"""
import csv
import json
import os
import sys

REF = os.environ.get("REFERENCE_ROOT", "")
if __name__ == "__main__" and not REF:
    sys.exit("set REFERENCE_ROOT to the reference checkout's root")
OUT = os.path.dirname(os.path.abspath(__file__))


def replay():
    src = os.path.join(REF, "fixtures/replay/european_bs-windows-x86_64.json")
    d = json.load(open(src))
    cases = []
    for c in d["cases"]:
        req, res = c["request"], c["result"]
        eng = req["engine"]
        case = {
            "name": c["name"],
            "request": req,
            "engine": eng["type"],
            "master_seed": eng.get("master_seed", eng.get("master_scramble_seed")),
            "sampling_units": eng.get("independent_sampling_units", eng.get("points_per_scramble")),
            "scramble_count": eng.get("scramble_count"),
            "antithetic": eng["variance_reduction"]["antithetic"],
            "brownian_bridge": eng["variance_reduction"]["brownian_bridge"],
            "reduction_block_size": c["execution"]["monte_carlo"]["reduction_block_size"],
            "spot": req["market"]["spot"],
            "discount_curve": req["market"]["discount_curve"],
            "dividend_curve": req["market"]["dividend_curve"],
            "volatility": req["model"]["volatility"],
            "strike": req["product"]["strike"],
            "valuation_date": req["valuation_date"],
            "expiry": req["product"]["expiry"],
            "gamma_bump_relative": req["risk"]["gamma"]["bump"]["value"],
            "expected": {
                "price": res["value"]["value"],
                "price_standard_error": res["value"]["standard_error"],
                "delta": res["risks"]["delta"]["raw"]["value"],
                "delta_standard_error": res["risks"]["delta"]["raw"]["standard_error"],
                "gamma": res["risks"]["gamma"]["raw"]["value"],
                "gamma_standard_error": res["risks"]["gamma"]["raw"]["standard_error"],
                "vega": res["risks"]["vega"]["raw"]["value"],
                "vega_standard_error": res["risks"]["vega"]["raw"]["standard_error"],
                "sampling_variance_bits": c["execution"]["sampling_variance_bits"],
                "estimator_variance_bits": c["execution"]["estimator_variance_bits"],
                "bump_delta_value_bits": c["execution"]["risk_validation"]["delta"]["bump_and_revalue"]["value_bits"],
                "bump_gamma_value_bits": c["execution"]["risk_validation"]["gamma"]["bump_and_revalue"]["value_bits"],
                "bump_vega_value_bits": c["execution"]["risk_validation"]["vega"]["bump_and_revalue"]["value_bits"],
            },
        }
        cases.append(case)
    json.dump({"source": "fixtures/replay/european_bs-windows-x86_64.json", "cases": cases},
              open(os.path.join(OUT, "replay_european_bs.json"), "w"), indent=1)


def _estimate(e):
    return {k: e[k] for k in ("value", "standard_error", "confidence_lower", "confidence_upper",
                              "effective_sampling_units")}


def local_volatility():
    platforms = {p: json.load(open(os.path.join(REF, f"fixtures/replay/local_volatility-{p}.json")))
                 for p in ("windows-x86_64", "macos-aarch64")}
    cases = []
    for i, c in enumerate(platforms["windows-x86_64"]["cases"]):
        req = c["request"]
        grid = req["model"]["local_variance_grid"]
        case = {
            "name": c["name"],
            "request": req,
            **_engine(req["engine"]),
            "reduction_block_size": c["execution"]["monte_carlo"]["reduction_block_size"],
            "spot": req["market"]["spot"],
            "discount_curve": req["market"]["discount_curve"],
            "dividend_curve": req["market"]["dividend_curve"],
            "local_variance_grid": {k: grid[k] for k in ("time_nodes", "log_forward_moneyness_nodes", "values",
                                                         "floor", "cap")},
            "valuation_date": req["valuation_date"],
            "product": {k: req["product"][k] for k in ("expiry", "notional", "strike")},
            "side": req["product"]["side"]["type"],
            "risk": {k: req["risk"][k] for k in ("delta", "gamma", "vega") if k in req["risk"]},
            "expected": {},
        }
        if "vega_kt" in req["risk"]:
            case["vega_kt"] = {"config": req["risk"]["vega_kt"],
                               "reporting_iv_basis": req["model"]["reporting_iv_basis"]}
        for name, d in platforms.items():
            pc = d["cases"][i]
            assert pc["name"] == c["name"]
            res = pc["result"]
            case["expected"][name] = {
                "value": _estimate(res["value"]),
                "sampling_variance_bits": pc["execution"]["sampling_variance_bits"],
                "estimator_variance_bits": pc["execution"]["estimator_variance_bits"],
                "evaluated_paths": int(pc["execution"]["evaluated_paths"]),
                "risks": {k: _estimate(res["risks"][k]["raw"]) for k in ("delta", "gamma", "vega")
                          if k in res["risks"]},
            }
        cases.append(case)
    # The node-allocation audit: the diagnostic local-node allocation's VegaKT
    # values for the two full-risk cases (the "current" side of each difference).
    audit = json.load(open(os.path.join(REF, "fixtures/replay/local-vol-node-allocation-change-audit-v1.json")))
    allocation = {}
    for path, _, current in audit["differences"]:
        parts = path.strip("/").split("/")
        idx = int(parts[1])
        key = "/".join(parts[5:])
        if "covariance" in key or key.startswith("estimates") or key in ("policy_label", "truncation_order"):
            continue
        allocation.setdefault(cases[idx]["name"], {})[key] = current
    for c in cases:
        if c["name"] in allocation:
            c["node_allocation"] = allocation[c["name"]]
    json.dump({"source": "fixtures/replay/local_volatility-{windows-x86_64,macos-aarch64}.json; node allocation: "
                         "fixtures/replay/local-vol-node-allocation-change-audit-v1.json (macos-aarch64)",
               "cases": cases},
              open(os.path.join(OUT, "replay_local_vol.json"), "w"), indent=1)


def path_dependence_replay():
    platforms = {p: json.load(open(os.path.join(REF, f"fixtures/replay/path_dependence-{p}.json")))
                 for p in ("windows-x86_64", "macos-aarch64")}
    cases = []
    for i, c in enumerate(platforms["windows-x86_64"]["cases"]):
        case = {
            "name": c["name"],
            "request": c["request"],
            "reduction_block_size": c["execution"]["monte_carlo"]["reduction_block_size"],
            "expected": {},
        }
        for name, d in platforms.items():
            pc = d["cases"][i]
            assert pc["name"] == c["name"] and pc["request"] == c["request"]
            res, ex = pc["result"], pc["execution"]
            case["expected"][name] = {
                "value": _estimate(res["value"]),
                "risks": {k: {"raw": _estimate(r["raw"]), "market_scaled": _estimate(r["market_scaled"]),
                              "raw_unit": r["raw_unit"]["type"],
                              "market_scaled_unit": r["market_scaled_unit"]["type"]}
                          for k, r in res["risks"].items()},
                "sampling_variance_bits": ex["sampling_variance_bits"],
                "estimator_variance_bits": ex["estimator_variance_bits"],
                "evaluated_paths": int(ex["evaluated_paths"]),
                "independent_sampling_units": ex["independent_sampling_units"],
                "risk_methods": ex["risk_methods"],
                "request_fingerprint": res["replay"]["request_fingerprint"],
                "bump_value_bits": {k: v["bump_and_revalue"]["value_bits"]
                                    for k, v in (ex.get("risk_validation") or {}).items() if v},
            }
        cases.append(case)
    json.dump({"source": "fixtures/replay/path_dependence-{windows-x86_64,macos-aarch64}.json", "cases": cases},
              open(os.path.join(OUT, "replay_path_dependence.json"), "w"), indent=1)


def step_adjoints():
    src = os.path.join(REF, "fixtures/local-vol/step-adjoints-v0.1.json")
    d = json.load(open(src))
    d["source"] = "fixtures/local-vol/step-adjoints-v0.1.json"
    json.dump(d, open(os.path.join(OUT, "lv_step_adjoints.json"), "w"), indent=1)


def direct_variance():
    src = os.path.join(REF, "fixtures/local-vol/direct-variance-v0.1.json")
    d = json.load(open(src))
    keep = {k: d[k] for k in ("reference", "relative_tolerance", "absolute_tolerance", "cases")}
    keep["source"] = "fixtures/local-vol/direct-variance-v0.1.json"
    json.dump(keep, open(os.path.join(OUT, "lv_direct_variance.json"), "w"), indent=1)


def wire_documents():
    out = {}
    for name in ("pricing_request", "pricing_request_american", "pricing_result", "pricing_result_american"):
        out[name] = json.load(open(os.path.join(REF, f"fixtures/v3/{name}.golden.json")))
    out["source"] = "fixtures/v3/*.golden.json"
    json.dump(out, open(os.path.join(OUT, "wire_v3_documents.json"), "w"), indent=1)


def wire_migration():
    out = {f"v{v}": json.load(open(os.path.join(REF, f"fixtures/v{v}/pricing_request.golden.json"))) for v in (1, 2)}
    out["source"] = "fixtures/v1/pricing_request.golden.json, fixtures/v2/pricing_request.golden.json"
    json.dump(out, open(os.path.join(OUT, "wire_migration.json"), "w"), indent=1)


def early_exercise_cases():
    src = os.path.join(REF, "fixtures/early-exercise/reference-cases-v0.1.json")
    d = json.load(open(src))
    keep = {k: d[k] for k in ("decision_cases", "basis_cases", "scaling_cases", "qr_cases")}
    keep["source"] = "fixtures/early-exercise/reference-cases-v0.1.json"
    json.dump(keep, open(os.path.join(OUT, "early_exercise_cases.json"), "w"), indent=1)


def surfaces():
    src = os.path.join(REF, "fixtures/local-vol/reference-cases-v0.1.json")
    d = json.load(open(src))
    keep = {k: d[k] for k in ("standard_ssvi", "essvi_interpolation", "constant_vol_dupire")}
    keep["source"] = "fixtures/local-vol/reference-cases-v0.1.json"
    json.dump(keep, open(os.path.join(OUT, "surfaces.json"), "w"), indent=1)


def analytical():
    src = os.path.join(REF, "fixtures/acceptance/european_bs_analytical.csv")
    rows = list(csv.DictReader(open(src)))
    json.dump({"source": "fixtures/acceptance/european_bs_analytical.csv", "rows": rows},
              open(os.path.join(OUT, "bs_analytical.json"), "w"), indent=1)


def path_dependence():
    src = os.path.join(REF, "fixtures/path-dependence/reference-cases-v0.1.json")
    d = json.load(open(src))
    keep = {k: d[k] for k in ("smoothing_cases", "extrema_cases", "bridge_cases", "smoothed_bridge_cases")}
    keep["source"] = "fixtures/path-dependence/reference-cases-v0.1.json"
    json.dump(keep, open(os.path.join(OUT, "path_dependence.json"), "w"), indent=1)


def _engine(e):
    rqmc = e["type"] == "randomized_quasi_monte_carlo"
    return {
        "engine": "rqmc" if rqmc else "pseudo",
        "master_seed": e["master_scramble_seed"] if rqmc else e["master_seed"],
        "sampling_units": e["points_per_scramble"] if rqmc else e["independent_sampling_units"],
        "scramble_count": e.get("scramble_count"),
        "antithetic": e["variance_reduction"]["antithetic"],
        "brownian_bridge": e["variance_reduction"]["brownian_bridge"],
    }


def early_exercise():
    src = os.path.join(REF, "fixtures/replay/early_exercise-windows-x86_64.json")
    d = json.load(open(src))
    cases = []
    for c in d["cases"]:
        req, res = c["request"], c["result"]
        ee = res["monte_carlo"]["early_exercise"]
        lsm = req["lsm"]
        case = {
            "name": c["name"],
            "request": req,
            "valuation": _engine(req["engine"]),
            "training": _engine(lsm["training_engine"]),
            "reduction_block_size": c["execution"]["monte_carlo"]["reduction_block_size"],
            "lsm": {
                "feature_count": lsm["basis"]["feature_count"],
                "max_degree": lsm["basis"]["max_degree"],
                "cpqr_abs_tolerance": lsm["cpqr"]["abs_rank_tolerance"],
                "cpqr_rel_tolerance": lsm["cpqr"]["rel_rank_tolerance"],
                "itm_abs_tolerance": lsm["itm_abs_tolerance"],
                "max_matrix_elements": lsm["max_matrix_elements"],
                "state_variables": [v["type"] for v in lsm["state_variables"]],
            },
            "spot": req["market"]["spot"],
            "discount_curve": req["market"]["discount_curve"],
            "dividend_curve": req["market"]["dividend_curve"],
            "volatility": req["model"]["volatility"],
            "valuation_date": req["valuation_date"],
            "product": {k: req["product"][k] for k in ("exercise_dates", "expiry", "notional", "strike")},
            "side": req["product"]["side"]["type"],
            "risk": req["risk"],
            "expected": {
                "value": res["value"],
                "sampling_variance": res["monte_carlo"]["sampling_variance"],
                "estimator_variance": res["monte_carlo"]["estimator_variance"],
                "sampling_variance_bits": c["execution"]["sampling_variance_bits"],
                "estimator_variance_bits": c["execution"]["estimator_variance_bits"],
                "evaluated_paths": int(c["execution"]["evaluated_paths"]),
                "independent_sampling_units": c["execution"]["independent_sampling_units"],
                "decision_models": ee["decision_models"],
                "regression_diagnostics": ee["regression_diagnostics"],
                "exercise_counts": ee["exercise_counts"],
                "exercise_probabilities": ee["exercise_probabilities"],
                "stopping_indices": ee["stopping_indices"],
                "in_sample_value": ee["in_sample_value"],
                "training_trajectories": ee["training_trajectories"],
                "valuation_trajectories": ee["valuation_trajectories"],
                "risks": res["risks"],
            },
        }
        cases.append(case)
    json.dump({"source": "fixtures/replay/early_exercise-windows-x86_64.json", "cases": cases},
              open(os.path.join(OUT, "early_exercise.json"), "w"), indent=1)


if __name__ == "__main__":
    if not os.path.isdir(REF):
        sys.exit(f"reference checkout not found at {REF}")
    replay()
    analytical()
    path_dependence()
    early_exercise()
    local_volatility()
    path_dependence_replay()
    early_exercise_cases()
    step_adjoints()
    direct_variance()
    wire_documents()
    wire_migration()
    surfaces()
    print("golden fixtures written to", OUT)

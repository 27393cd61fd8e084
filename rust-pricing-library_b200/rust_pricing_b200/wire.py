"""Pricing requests and results in the reference's v3 wire format.

`compile_request` turns a `pricing_request` document
(schemas/v3/pricing_request.schema.json, parsed by crates/pricing/src/wire.rs
and validated by crates/pricing/src/api/request.rs:60-230) into the engine's
plan the way SimulationPlan::compile does
(crates/pricing/src/engine/compile/simulation.rs:93-330):

* times are ACT/365F year fractions from the valuation date
  (DayCountConvention::year_fraction, crates/pricing/src/core/date.rs:225-231);
* the plan observes every distinct simulated date of the payoff graph once, in
  date order (CompiledPayoff::terminal_observations, payoff/tape.rs:229-247);
* the discount factor is taken at the payment date;
* dates before the valuation date enter as the graph's literals: the known
  Asian fixings, the lookback's historical extremum and valuation-date
  fixing, and the barrier's historical hit (payoff/compile.rs:159-474), which
  the plan carries as a product's seasoned state.

`price_request` evaluates the compiled plan on the GPU through the C ABI and
`result_document` writes the `pricing_result` value and risk estimates in the
reference's layout, with its market scaling (1 % spot Delta and Gamma, one
volatility point Vega) and 95 % normal confidence bounds
(crates/pricing/src/engine/risk/report.rs:255-300,454-489), and the replay
block with the request's BLAKE3 fingerprint over its canonical encoding
(crates/pricing/src/wire.rs:4144-4212).

`evaluate_width_ladder` evaluates a request's compact-C2 half-width ladder
(PricingPlan::evaluate_width_ladder) on the same random coordinates.

Requests outside the engine's hot path raise `UnsupportedRequest`: discrete
dividends, the Bass local-volatility model, simulated observations on the
valuation date outside multi-date Black--Scholes paths, and the
American/LSM state variables other than spot.
"""
from __future__ import annotations

import datetime as _dt
import math
from dataclasses import dataclass, field
from typing import Optional

from . import _abi as A
from .desc import LocalVarianceSpec, LsmSpec, PlanSpec, ProductSpec

NORMAL_95 = 1.959_963_984_540_054  # crates/pricing/src/engine/plan/simulation.rs:24
SCHEMA_VERSION = 3


class WireError(ValueError):
    """A request document that does not follow the v3 schema."""


class UnsupportedRequest(WireError):
    """A valid request that this engine does not price."""


def parse_date(text: str) -> _dt.date:
    try:
        return _dt.date.fromisoformat(text)
    except (TypeError, ValueError) as exc:
        raise WireError(f"invalid date {text!r}") from exc


def year_fraction(start: _dt.date, end: _dt.date) -> float:
    """ACT/365F: whole days over 365 (crates/pricing/src/core/date.rs:225-231)."""
    return float((end - start).days) / 365.0


def _get(obj: dict, key: str, where: str):
    if not isinstance(obj, dict) or key not in obj:
        raise WireError(f"{where}: missing field {key!r}")
    return obj[key]


def _side(product: dict) -> int:
    side = _get(_get(product, "side", "product"), "type", "product.side")
    if side not in ("call", "put"):
        raise WireError(f"product.side: unknown side {side!r}")
    return A.CALL if side == "call" else A.PUT


def _positive(value, where: str) -> float:
    v = float(value)
    if not (v > 0.0 and math.isfinite(v)):
        raise WireError(f"{where} must be positive and finite")
    return v


@dataclass
class CompiledRequest:
    """A request compiled to the engine's plan, with what the result needs."""

    plan: PlanSpec
    lsm: Optional[LsmSpec]
    product_type: str
    estimator: str
    independent_units: int
    spot: float
    request_delta: bool
    request_gamma: bool
    request_vega: bool
    smile_dynamics: str
    vega_kt: Optional[dict] = None
    observation_dates: list = field(default_factory=list)


# --------------------------------------------------------------- dividends

def _dividends(events: list) -> list:
    """market.discrete_dividends (schemas/v3 dividend_event / dividend_quote):
    (ex_time, fixed cash, proportional fraction) per event, as the plan's
    escrowed affine dividend schedule (DividendQuote, crates/pricing/src/market/dividend.rs:9-55)."""
    out = []
    for i, e in enumerate(events):
        where = f"market.discrete_dividends[{i}]"
        t = float(_get(e, "ex_time", where))
        q = _get(e, "quote", where)
        kind = _get(q, "type", where + ".quote")
        if kind == "fixed_cash":
            cash, beta = float(_get(q, "amount", where + ".quote")), 0.0
        elif kind == "proportional":
            cash, beta = 0.0, float(_get(q, "beta", where + ".quote"))
        elif kind == "fixed_cash_and_proportional":
            cash, beta = float(_get(q, "fixed_cash", where + ".quote")), float(_get(q, "beta", where + ".quote"))
        else:
            raise WireError(f"{where}.quote: unknown type {kind!r}")
        if not (math.isfinite(t) and t >= 0.0) or not (math.isfinite(cash) and cash >= 0.0) or \
                not (math.isfinite(beta) and 0.0 <= beta < 1.0):
            raise WireError(f"{where}: ex_time and cash must be finite and >= 0, beta in [0, 1)")
        if out and not t > out[-1][0]:
            raise WireError("market.discrete_dividends must be ordered by strictly increasing ex_time")
        out.append((t, cash, beta))
    return out


# ------------------------------------------------------------------ engine

def _engine(engine: dict, where: str) -> dict:
    kind = _get(engine, "type", where)
    vr = _get(engine, "variance_reduction", where)
    common = dict(antithetic=bool(_get(vr, "antithetic", where)),
                  brownian_bridge=bool(_get(vr, "brownian_bridge", where)))
    if kind == "pseudo_monte_carlo":
        units = int(_get(engine, "independent_sampling_units", where))
        if units < 1:
            raise WireError(f"{where}.independent_sampling_units must be positive")
        return dict(engine=A.ENGINE_PSEUDO, master_seed=int(_get(engine, "master_seed", where)),
                    sampling_units=units, scramble_count=0, **common)
    if kind == "randomized_quasi_monte_carlo":
        points = int(_get(engine, "points_per_scramble", where))
        if points < 1 or points & (points - 1):
            raise WireError(f"{where}.points_per_scramble must be a power of two")
        return dict(engine=A.ENGINE_RQMC, master_seed=int(_get(engine, "master_scramble_seed", where)),
                    sampling_units=points, scramble_count=int(_get(engine, "scramble_count", where)), **common)
    raise WireError(f"{where}: unknown engine type {kind!r}")


# ----------------------------------------------------------------- product

@dataclass
class _Product:
    spec: ProductSpec
    dates: list          # simulated observation dates (sorted, unique, after valuation)
    expiry: _dt.date
    payment: _dt.date


def _simulated(dates, valuation, what: str):
    """The distinct simulated dates in order.  A date equal to the valuation
    date is a time-zero observation: a zero-length step that still takes its
    normal in the reference's path generator; compile_request admits it for
    Black--Scholes paths only."""
    return sorted(set(dates))


def _european(p: dict, valuation) -> _Product:
    expiry = parse_date(_get(p, "expiry", "product"))
    spec = ProductSpec(kind=A.PRODUCT_EUROPEAN, side=_side(p), strike=_positive(p["strike"], "product.strike"),
                       notional=_positive(_get(p, "notional", "product"), "product.notional"))
    return _Product(spec, _simulated([expiry], valuation, "the expiry"), expiry, expiry)


def _american(p: dict, valuation) -> _Product:
    expiry = parse_date(_get(p, "expiry", "product"))
    dates = [parse_date(d) for d in _get(p, "exercise_dates", "product")]
    if any(d < valuation for d in dates):
        raise WireError("american exercise dates before the valuation date (AmericanPastExerciseUnsupported)")
    spec = ProductSpec(kind=A.PRODUCT_AMERICAN, side=_side(p), strike=_positive(p["strike"], "product.strike"),
                       notional=_positive(_get(p, "notional", "product"), "product.notional"))
    return _Product(spec, _simulated(dates, valuation, "an exercise date"), expiry, expiry)


def _digital(p: dict, valuation) -> _Product:
    expiry = parse_date(_get(p, "expiry", "product"))
    payment = parse_date(p["payment_date"]) if "payment_date" in p else expiry
    if payment < expiry:
        raise WireError("digital payment date before expiry")
    kind = _get(_get(p, "payout_kind", "product"), "type", "product.payout_kind")
    if kind not in ("cash", "asset"):
        raise WireError(f"product.payout_kind: unknown kind {kind!r}")
    spec = ProductSpec(kind=A.PRODUCT_DIGITAL, side=_side(p), strike=_positive(p["strike"], "product.strike"),
                       payout=_positive(_get(p, "payout", "product"), "product.payout"),
                       digital_payout=A.DIGITAL_CASH if kind == "cash" else A.DIGITAL_ASSET)
    return _Product(spec, _simulated([expiry], valuation, "the expiry"), expiry, payment)


def _barrier(p: dict, valuation) -> _Product:
    expiry = parse_date(_get(p, "expiry", "product"))
    payment = parse_date(_get(p, "payment_date", "product"))
    monitoring = [parse_date(d) for d in _get(p, "monitoring_dates", "product")]
    if not monitoring or any(a >= b for a, b in zip(monitoring, monitoring[1:])) or monitoring[-1] > expiry:
        raise WireError("barrier monitoring dates must be increasing and end on or before expiry")
    continuous = _get(_get(p, "monitoring", "product"), "type", "product.monitoring") == "continuous"
    direction = _get(_get(p, "direction", "product"), "type", "product.direction")
    style = _get(_get(p, "style", "product"), "type", "product.style")
    past = [d for d in monitoring if d < valuation]
    history = p.get("historical_hit")
    if bool(past) != (history is not None):
        raise WireError("barrier history must be given exactly when monitoring dates precede valuation")
    live = [d for d in monitoring if d >= valuation]
    spec = ProductSpec(kind=A.PRODUCT_CONTINUOUS_BARRIER if continuous else A.PRODUCT_DISCRETE_BARRIER,
                       side=_side(p), strike=_positive(p["strike"], "product.strike"),
                       notional=_positive(_get(p, "notional", "product"), "product.notional"),
                       barrier=_positive(_get(p, "barrier", "product"), "product.barrier"),
                       barrier_direction=A.BARRIER_UP if direction == "up" else A.BARRIER_DOWN,
                       barrier_style=A.KNOCK_OUT if style == "knock_out" else A.KNOCK_IN,
                       rebate=float(p["rebate"]) if p.get("rebate") is not None else None)
    if continuous:
        # The bridge runs from the valuation date through every plan interval;
        # the reference's window ends at the last monitoring date
        # (compile/simulation.rs:215-256).
        if monitoring[-1] != expiry:
            raise UnsupportedRequest("continuous barrier monitored to a date before expiry")
        if history:
            raise UnsupportedRequest("continuous barrier already hit before the valuation date")
        # Time-zero points are dropped for a continuous barrier (simulation.rs:224-225).
        dates = sorted(set([d for d in live if d > valuation] + [expiry]))
        return _Product(spec, _simulated(dates, valuation, "the expiry"), expiry, payment)
    dates = _simulated(sorted(set(live + [expiry])), valuation, "a barrier monitoring date")
    monitored = set(live)
    if any(d not in monitored for d in dates):
        spec.weights = [1.0 if d in monitored else 0.0 for d in dates]
    if history is not None:
        spec.initial_state = 1.0 if history else 0.0
    return _Product(spec, dates, expiry, payment)


def _asian(p: dict, valuation) -> _Product:
    payment = parse_date(_get(p, "payment_date", "product"))
    observations = _get(p, "observations", "product")
    if not observations:
        raise WireError("asian observations must not be empty")
    dates = [parse_date(_get(o, "date", "observation")) for o in observations]
    if any(a >= b for a, b in zip(dates, dates[1:])):
        raise WireError("asian observation dates must be strictly increasing")
    known_sum, weights, sim = 0.0, [], []
    seen_unknown = False
    for o, d in zip(observations, dates):
        value = _get(o, "value", "observation")
        w = float(_get(o, "weight", "observation"))
        kind = _get(value, "type", "observation.value")
        if kind == "known":
            if d > valuation:
                raise WireError("asian observation after the valuation date cannot carry a known fixing")
            # Literal fixings in observation order (compile.rs:162-176); the
            # dates increase, so every known fixing precedes the simulated ones.
            known_sum = known_sum + float(_get(value, "fixing", "observation.value")) * w
        elif kind == "unknown":
            if d < valuation:
                raise WireError("asian observation before the valuation date requires a known fixing")
            seen_unknown = True
            sim.append(d)
            weights.append(w)
        else:
            raise WireError(f"observation.value: unknown type {kind!r}")
    total = math.fsum(float(o["weight"]) for o in observations)
    if not (abs(total - 1.0) <= max(1e-12, 1e-12 * len(observations))):
        # ArithmeticAsianSpec::new (crates/pricing/src/product/spec.rs:653-663)
        raise WireError("asian observation weights must sum to one")
    if not seen_unknown:
        raise UnsupportedRequest("asian with every fixing known has no simulated observation")
    spec = ProductSpec(kind=A.PRODUCT_ASIAN, side=_side(p), strike=_positive(p["strike"], "product.strike"),
                       notional=_positive(_get(p, "notional", "product"), "product.notional"), weights=weights)
    if len(sim) != len(observations):
        spec.initial_state = known_sum
    return _Product(spec, _simulated(sim, valuation, "an asian observation"), dates[-1], payment)


def _lookback(p: dict, valuation) -> _Product:
    payment = parse_date(_get(p, "payment_date", "product"))
    monitoring = [parse_date(d) for d in _get(p, "monitoring_dates", "product")]
    if not monitoring or any(a >= b for a, b in zip(monitoring, monitoring[1:])):
        raise WireError("lookback monitoring dates must be strictly increasing")
    call = _side(p) == A.CALL
    extremum = p.get("historical_extremum")
    fixing = p.get("valuation_date_fixing")
    has_past = any(d < valuation for d in monitoring)
    if has_past != (extremum is not None):
        raise WireError("lookback historical extremum must be given exactly when monitoring dates precede valuation")
    if fixing is not None and valuation not in monitoring:
        raise WireError("lookback valuation-date fixing requires a monitoring date equal to the valuation date")
    # The literal head of the running extremum (compile.rs:426-452): the
    # historical extremum, then the valuation-date fixing under Maximum /
    # Minimum (ties keep the left operand).
    state = None
    if extremum is not None:
        state = _positive(extremum, "product.historical_extremum")
    if fixing is not None:
        f = _positive(fixing, "product.valuation_date_fixing")
        if state is None:
            state = f
        elif call:
            state = state if state >= f else f
        else:
            state = state if state <= f else f
    live = [d for d in monitoring if d > valuation or (d == valuation and fixing is None)]
    if not live:
        raise UnsupportedRequest("lookback with every monitoring date fixed has no simulated observation")
    spec = ProductSpec(kind=A.PRODUCT_LOOKBACK, side=A.CALL if call else A.PUT,
                       strike=_positive(p["strike"], "product.strike"),
                       notional=_positive(_get(p, "notional", "product"), "product.notional"),
                       initial_state=state)
    return _Product(spec, _simulated(live, valuation, "a lookback monitoring date"), monitoring[-1], payment)


_PRODUCTS = {
    "european_vanilla": _european,
    "american_vanilla": _american,
    "digital": _digital,
    "barrier": _barrier,
    "arithmetic_asian": _asian,
    "fixed_lookback": _lookback,
}


# ------------------------------------------------------------ curves, model

def _curve(c: dict, where: str):
    times = [float(t) for t in _get(c, "times", where)]
    factors = [float(f) for f in _get(c, "discount_factors", where)]
    if len(times) != len(factors) or len(times) < 1:
        raise WireError(f"{where}: times and discount_factors differ in length")
    return times, factors


def log_discount(times, factors, t: float) -> float:
    """Log-linear discount curve: ln DF at a pillar, linear in ln DF between
    pillars and along the last segment beyond them (the curve the engine's
    plan compile uses, crates/pricing/src/market/curve.rs)."""
    logs = [math.log(f) for f in factors]
    for i, ti in enumerate(times):
        if ti == t:
            return logs[i]
    right = next((i for i, ti in enumerate(times) if ti > t), len(times) - 1)
    left = right - 1
    w = (t - times[left]) / (times[right] - times[left])
    return logs[left] + w * (logs[right] - logs[left])


def _model(doc: dict, plan_kw: dict, expiry_time: float, warnings: list):
    model = _get(doc, "model", "request")
    kind = _get(model, "type", "model")
    if kind in ("black_scholes", "black_76"):
        # Both integrate the forward with one volatility in the simulation
        # plan (compile/simulation.rs:280-288).
        vol = float(_get(model, "volatility", "model"))
        if not (vol >= 0.0 and math.isfinite(vol)):
            raise WireError("model.volatility must be finite and non-negative")
        plan_kw.update(model=A.MODEL_BLACK_SCHOLES, volatility=vol)
        return None
    if kind == "local_volatility":
        g = _get(model, "local_variance_grid", "model")
        tn = [float(t) for t in _get(g, "time_nodes", "local_variance_grid")]
        xn = [float(x) for x in _get(g, "log_forward_moneyness_nodes", "local_variance_grid")]
        shape = list(_get(g, "shape", "local_variance_grid"))
        values = [float(v) for v in _get(g, "values", "local_variance_grid")]
        if shape != [len(tn), len(xn)] or len(values) != len(tn) * len(xn):
            raise WireError("local_variance_grid: shape does not match the nodes and values")
        plan_kw.update(model=A.MODEL_LOCAL_VOLATILITY, volatility=0.0,
                       local_variance=LocalVarianceSpec(tn, xn, values, float(g["floor"]), float(g["cap"])))
        return model.get("reporting_iv_basis")
    if kind == "bass_local_volatility":
        raise UnsupportedRequest("the Bass local-volatility model is not on this engine's path")
    raise WireError(f"model: unknown type {kind!r}")


# ----------------------------------------------------------------- VegaKT policy

# The reference's two VegaKT methods for a local-volatility request: the exact
# market-IV risk of a statically replicable terminal payoff
# (crates/pricing/src/engine/risk/vegakt_terminal_replication.rs:7) and the
# allocation of the path simulation's local-vega node sensitivities to the
# reporting buckets (crates/pricing/src/engine/risk/local_vol_allocation.rs:108-163).
TERMINAL_REPLICATION = "terminal_payoff_replication_iv_v1"
NODE_ALLOCATION = "local_vol_node_allocation_diagnostic_v1"


def _terminal_replication_applies(ptype: str, times: list, plan_kw: dict, basis: dict) -> bool:
    """Whether the reference prices this request's VegaKT by terminal
    replication instead of node allocation
    (compile_terminal_replication_vega_kt and compile_terminal_vega_kt,
    crates/pricing/src/engine/risk/vegakt_terminal_replication.rs:10-40,
    crates/pricing/src/engine/risk/vegakt_terminal_pricing.rs:21-71): no early
    exercise, continuous barrier or payoff smoothing, identity dividend
    coordinates, the expiry among the reporting basis's maturities, and a
    payoff that is piecewise affine in the terminal spot alone
    (try_terminal_payoff_gamma_measure, crates/pricing/src/engine/risk/vegakt_terminal.rs:200-330:
    literals, the expiry's spot, sums, differences, minima, maxima and
    constant scalings).  Of this engine's products that is the European
    vanilla and an Asian or fixed lookback whose only simulated observation is
    the expiry; digitals (an indicator) and barriers (hit state) are not.
    A grid whose every time row is flat in log-moneyness is counted as
    replicable too: the reference then checks the grid's cumulative variance
    against the basis's implied volatilities and may route the request to its
    terminal pathwise method, neither of which is node allocation."""
    if ptype == "european_vanilla":
        terminal = True
    elif ptype in ("arithmetic_asian", "fixed_lookback"):
        terminal = len(times) == 1
    else:
        terminal = False
    if not terminal or plan_kw.get("smoothing_half_width", 0.0) > 0.0:
        return False
    maturities = [float(t) for t in basis.get("maturity_nodes", [])]
    return times[-1] in maturities


# ----------------------------------------------------------------- compile

def compile_request(doc: dict, *, reduction_block_size: int = 4096) -> CompiledRequest:
    """The engine plan of one v3 `pricing_request` document.

    `reduction_block_size` is the reference's ExecutionPolicy block size
    (crates/pricing/src/engine/mc/execution.rs), not part of the request."""
    if _get(doc, "document_kind", "request") != "pricing_request":
        raise WireError("document_kind must be 'pricing_request'")
    if _get(doc, "schema_version", "request") != SCHEMA_VERSION:
        doc, _ = migrate_request(doc)
    valuation = parse_date(_get(doc, "valuation_date", "request"))
    product_doc = _get(doc, "product", "request")
    ptype = _get(product_doc, "type", "product")
    if ptype not in _PRODUCTS:
        raise UnsupportedRequest(f"product type {ptype!r}")
    product = _PRODUCTS[ptype](product_doc, valuation)
    if product.expiry < valuation:
        raise WireError("expiry before the valuation date")
    has_lsm = "lsm" in doc
    if (ptype == "american_vanilla") != has_lsm:
        raise WireError("lsm configuration is required for, and only for, american_vanilla")

    market = _get(doc, "market", "request")
    if _get(market, "type", "market") != "equity":
        raise WireError("market.type must be 'equity'")
    dividends = _dividends(market.get("discrete_dividends") or [])
    spot = _positive(_get(market, "spot", "market"), "market.spot")
    dt, dfs = _curve(_get(market, "discount_curve", "market"), "market.discount_curve")
    qt, qfs = _curve(_get(market, "dividend_curve", "market"), "market.dividend_curve")

    engine = _engine(_get(doc, "engine", "request"), "engine")
    times = [year_fraction(valuation, d) for d in product.dates]
    payment_time = year_fraction(valuation, product.payment)
    plan_kw = dict(observation_times=times, products=[product.spec], spot=spot,
                   discount_times=dt, discount_factors=dfs, dividend_times=qt, dividend_factors=qfs,
                   reduction_block_size=reduction_block_size, payment_time=payment_time, dividends=dividends,
                   **engine)
    warnings: list = []
    basis = _model(doc, plan_kw, times[-1], warnings)
    if times[0] == 0.0 and (plan_kw["model"] != A.MODEL_BLACK_SCHOLES or ptype == "american_vanilla"
                            or len(times) == 1):
        raise UnsupportedRequest("an observation on the valuation date is simulated at time zero only on "
                                 "multi-date Black-Scholes paths")

    risk = _get(doc, "risk", "request")
    for key in ("delta", "vega", "smile_dynamics"):
        _get(risk, key, "risk")
    if risk.get("payoff_smoothing_width_ladder"):
        raise UnsupportedRequest("a width-ladder request is evaluated by evaluate_width_ladder")
    req_delta, req_vega = bool(risk["delta"]), bool(risk["vega"])
    gamma = risk.get("gamma")
    plan_kw.update(request_delta=req_delta, request_vega=req_vega, request_gamma=gamma is not None)
    if gamma is not None:
        bump = _get(gamma, "bump", "risk.gamma")
        kind = _get(bump, "type", "risk.gamma.bump")
        if kind not in ("relative", "absolute"):
            raise WireError(f"risk.gamma.bump: unknown type {kind!r}")
        plan_kw.update(gamma_bump_relative=kind == "relative",
                       gamma_bump=_positive(_get(bump, "value", "risk.gamma.bump"), "risk.gamma.bump.value"))
    smoothing = risk.get("payoff_smoothing")
    if smoothing is not None:
        if _get(smoothing, "type", "risk.payoff_smoothing") != "compact_c2":
            raise WireError("risk.payoff_smoothing: unknown kernel")
        plan_kw["smoothing_half_width"] = _positive(_get(smoothing, "half_width", "risk.payoff_smoothing"),
                                                    "risk.payoff_smoothing.half_width")
    if "checkpoint_interval" in risk:
        plan_kw["checkpoint_interval"] = int(risk["checkpoint_interval"])
    vega_kt = None
    if risk.get("vega_kt") is not None:
        if plan_kw.get("model") != A.MODEL_LOCAL_VOLATILITY or basis is None:
            raise WireError("risk.vega_kt needs a local-volatility model with a reporting_iv_basis")
        plan_kw["request_local_vega_nodes"] = True
        replicable = _terminal_replication_applies(ptype, times, plan_kw, basis)
        vega_kt = {"config": risk["vega_kt"], "reporting_iv_basis": basis,
                   "policy": TERMINAL_REPLICATION if replicable else NODE_ALLOCATION}

    if dividends:
        if ptype == "american_vanilla" or product.spec.kind == A.PRODUCT_CONTINUOUS_BARRIER:
            raise UnsupportedRequest("discrete dividends with early exercise or a continuous barrier")
        if plan_kw.get("model") == A.MODEL_LOCAL_VOLATILITY and (req_vega or vega_kt is not None):
            raise UnsupportedRequest("local-volatility Vega and VegaKT with discrete dividends")
    plan = PlanSpec(**plan_kw)
    if plan.engine == A.ENGINE_RQMC and plan.scramble_count < 1:
        raise WireError("engine.scramble_count must be positive")
    lsm = None
    if has_lsm:
        lsm = _lsm(doc["lsm"], plan)
    units = plan.scramble_count if plan.engine == A.ENGINE_RQMC else plan.sampling_units
    return CompiledRequest(plan=plan, lsm=lsm, product_type=ptype,
                           estimator="randomized_quasi_monte_carlo" if plan.engine == A.ENGINE_RQMC
                           else "pseudo_monte_carlo",
                           independent_units=units, spot=spot, request_delta=req_delta,
                           request_gamma=gamma is not None, request_vega=req_vega,
                           smile_dynamics=_get(risk["smile_dynamics"], "type", "risk.smile_dynamics"),
                           vega_kt=vega_kt, observation_dates=[d.isoformat() for d in product.dates])


def _lsm(cfg: dict, plan: PlanSpec) -> LsmSpec:
    """LsmConfig (crates/pricing/src/engine/mc/lsm.rs:328-495) of a spot state."""
    states = [_get(s, "type", "lsm.state_variables") for s in _get(cfg, "state_variables", "lsm")]
    if states != ["spot"]:
        raise UnsupportedRequest("LSM state variables other than one spot")
    basis = _get(cfg, "basis", "lsm")
    if int(_get(basis, "feature_count", "lsm.basis")) != 1:
        raise UnsupportedRequest("LSM bases of more than one feature")
    training = _engine(_get(cfg, "training_engine", "lsm"), "lsm.training_engine")
    if training["engine"] != plan.engine:
        raise UnsupportedRequest("an LSM training engine of another kind than the valuation engine")
    cpqr = _get(cfg, "cpqr", "lsm")
    return LsmSpec(training_seed=training["master_seed"], training_units=training["sampling_units"],
                   training_scramble_count=training["scramble_count"], training_antithetic=training["antithetic"],
                   training_brownian_bridge=training["brownian_bridge"],
                   max_degree=int(_get(basis, "max_degree", "lsm.basis")),
                   itm_abs_tolerance=float(_get(cfg, "itm_abs_tolerance", "lsm")),
                   cpqr_abs_tolerance=float(_get(cpqr, "abs_rank_tolerance", "lsm.cpqr")),
                   cpqr_rel_tolerance=float(_get(cpqr, "rel_rank_tolerance", "lsm.cpqr")),
                   max_matrix_elements=int(_get(cfg, "max_matrix_elements", "lsm")))


# ------------------------------------------------------------ fingerprint

# Request fields the schema types as integers; every other number is an f64.
_INTEGER_FIELDS = frozenset((
    "schema_version", "underlying_id", "currency_id", "curve_id", "event_id", "master_seed",
    "master_scramble_seed", "independent_sampling_units", "points_per_scramble", "scramble_count",
    "feature_count", "max_degree", "max_matrix_elements", "checkpoint_interval", "aad_tile_capacity", "shape"))


def _canonical(value, key=None):
    """The request as the reference re-serialises it (serde_json::Value):
    object keys sorted, integer-typed fields as integers, other numbers as f64."""
    if isinstance(value, dict):
        return {k: _canonical(v, k) for k, v in value.items()}
    if isinstance(value, list):
        return [_canonical(v, key) for v in value]
    if isinstance(value, bool) or value is None or isinstance(value, str):
        return value
    if isinstance(value, (int, float)):
        return int(value) if key in _INTEGER_FIELDS else float(value)
    raise WireError(f"unsupported JSON value {value!r}")


def _encode(value, out: bytearray) -> None:
    """encode_value (crates/pricing/src/wire.rs:4165-4212): tag, big-endian
    u64 payload length, payload; u64/i64/f64 numbers big-endian, strings as
    UTF-8, arrays and objects with a u64 count (object entries in key order)."""
    import struct
    if value is None:
        tag, payload = 0, b""
    elif isinstance(value, bool):
        tag, payload = 1, bytes([int(value)])
    elif isinstance(value, int):
        tag, payload = (2, struct.pack(">Q", value)) if value >= 0 else (3, struct.pack(">q", value))
    elif isinstance(value, float):
        if not math.isfinite(value):
            raise WireError("non-finite JSON number")
        tag, payload = 4, struct.pack(">d", value)
    elif isinstance(value, str):
        tag, payload = 5, value.encode("utf-8")
    elif isinstance(value, list):
        body = bytearray(struct.pack(">Q", len(value)))
        for v in value:
            _encode(v, body)
        tag, payload = 6, bytes(body)
    else:
        body = bytearray(struct.pack(">Q", len(value)))
        for k in sorted(value):
            _encode(k, body)
            _encode(value[k], body)
        tag, payload = 7, bytes(body)
    out.append(tag)
    out += struct.pack(">Q", len(payload))
    out += payload


def _fingerprint_value(value, schema_version: int) -> str:
    """fingerprint_request_value (wire.rs:4158-4163): BLAKE3 of
    "pricing/request\0", the schema version as a big-endian u32 and the
    encoding of the value."""
    import struct
    from .blake3 import blake3
    body = bytearray(b"pricing/request\0" + struct.pack(">I", schema_version))
    _encode(value, body)
    return "blake3-256:" + blake3(bytes(body)).hex()


def request_fingerprint(doc: dict) -> str:
    """fingerprint_request (wire.rs:4144-4163): the fingerprint of the v3
    request as the reference re-serialises it (the canonical encoding)."""
    return _fingerprint_value(_canonical(doc), SCHEMA_VERSION)


MIGRATION_REQUEST_V1_TO_V2 = "pricing_request/v1-to-v2"
MIGRATION_REQUEST_V2_TO_V3 = "pricing_request/v2-to-v3"


def migrate_request(doc: dict) -> tuple[dict, dict]:
    """request_from_document's schema migration (crates/pricing/src/wire.rs:4015-4076,
    RequestV1 -> RequestV2 -> RequestV3 at :1090-1137): a version-1 or -2
    `pricing_request` carried to version 3 (v1 -> v2: the risk block gains no
    smoothing-width ladder; v2 -> v3: no LSM block), and the migration
    provenance the result's replay block records: the source and current
    versions, the migration ids, the fingerprint of the source document as
    parsed at its own version and that of the migrated request.  Features the
    older schemas do not have are refused, as the reference refuses them:
    graph products, Bass local volatility, a lookback's valuation-date fixing,
    an LSM block, and (version 1) a smoothing-width ladder."""
    import copy
    version = _get(doc, "schema_version", "request")
    if version == SCHEMA_VERSION:
        fp = request_fingerprint(doc)
        return doc, {"original_schema_version": SCHEMA_VERSION, "current_schema_version": SCHEMA_VERSION,
                     "migration_ids": [], "pre_migration_fingerprint": fp, "post_migration_fingerprint": fp}
    if version not in (1, 2) or isinstance(version, bool):
        raise UnsupportedRequest(f"schema_version {version!r} (this engine reads versions 1 to 3)")
    product, model = doc.get("product") or {}, doc.get("model") or {}
    if product.get("type") == "graph":
        raise UnsupportedRequest("graph products require pricing_specification v2")
    if model.get("type") == "bass_local_volatility":
        raise UnsupportedRequest(f"Bass local volatility is not in schema version {version}")
    if "valuation_date_fixing" in product:
        raise UnsupportedRequest(f"Lookback valuation-date fixing is not in schema version {version}")
    if "lsm" in doc:
        raise WireError(f"unknown field `lsm` in a schema-version-{version} request")
    if version == 1 and "payoff_smoothing_width_ladder" in (doc.get("risk") or {}):
        raise WireError("unknown field `payoff_smoothing_width_ladder` in a schema-version-1 risk block")
    pre = _fingerprint_value(doc, version)
    current = copy.deepcopy(doc)
    current["schema_version"] = SCHEMA_VERSION
    post = request_fingerprint(current)
    ids = [MIGRATION_REQUEST_V1_TO_V2, MIGRATION_REQUEST_V2_TO_V3] if version == 1 else [MIGRATION_REQUEST_V2_TO_V3]
    return current, {"original_schema_version": version, "current_schema_version": SCHEMA_VERSION,
                     "migration_ids": ids, "pre_migration_fingerprint": pre, "post_migration_fingerprint": post}


def replay_block(doc: dict) -> dict:
    """The result's replay section: this engine's version and platform, the
    (migrated) request's fingerprint and the migration provenance."""
    import platform
    from . import __version__
    _, migration = migrate_request(doc)
    return {"library_version": __version__, "platform": f"{platform.system().lower()}-{platform.machine()}-b200",
            "request_fingerprint": migration["post_migration_fingerprint"], "schema_version": SCHEMA_VERSION,
            "migration": migration}


# ------------------------------------------------------------------ result

def _estimate(e, estimator: str, scale: float = 1.0) -> dict:
    """An Estimate of the result document.  The market-scaled estimate of a
    risk is estimate_from_statistics with `scale` (report.rs:454-473):
    value * scale and standard error * |scale|, with the 95 % bounds
    recomputed from them."""
    value = e.value * scale
    se = e.standard_error * abs(scale)
    half = NORMAL_95 * se
    if scale == 1.0:
        lower, upper = e.confidence_lower, e.confidence_upper
    else:
        lower, upper = value - half, value + half
    return {"value": value, "standard_error": se, "confidence_lower": lower, "confidence_upper": upper,
            "estimator": {"type": estimator}, "effective_sampling_units": int(e.effective_sampling_units)}


def _risk(e, estimator: str, scale: float, raw_unit: str, scaled_unit: str) -> dict:
    return {"raw": _estimate(e, estimator), "market_scaled": _estimate(e, estimator, scale),
            "raw_unit": {"type": raw_unit}, "market_scaled_unit": {"type": scaled_unit}}


def result_document(req: CompiledRequest, price, delta=None, gamma=None, vega=None,
                    sampling_variance: Optional[float] = None, estimator_variance: Optional[float] = None,
                    evaluated_paths: Optional[int] = None, vega_kt: Optional[dict] = None,
                    warnings: Optional[list] = None, request: Optional[dict] = None) -> dict:
    """A `pricing_result` document (schemas/v3/pricing_result.schema.json) of
    the engine's estimates: value, risks with raw and market-scaled values
    (report.rs:255-300), diagnostics and the Monte Carlo variances."""
    est = req.estimator
    risks: dict = {}
    s = req.spot * 0.01
    if req.request_delta and delta is not None:
        risks["delta"] = _risk(delta, est, s, "delta_raw", "delta_one_percent_spot")
    if req.request_gamma and gamma is not None:
        risks["gamma"] = _risk(gamma, est, s * s, "gamma_raw", "gamma_one_percent_spot_squared")
    if req.request_vega and vega is not None:
        risks["vega"] = _risk(vega, est, 0.01, "vega_raw", "vega_one_vol_point")
    if vega_kt is not None:
        risks["vega_kt"] = vega_kt
    doc = {"document_kind": "pricing_result", "schema_version": SCHEMA_VERSION,
           "value": _estimate(price, est), "risks": risks,
           "diagnostics": {"warnings": list(warnings or [])}}
    if sampling_variance is not None:
        doc["monte_carlo"] = {"sampling_variance": sampling_variance, "estimator_variance": estimator_variance,
                              "independent_sampling_units": req.independent_units,
                              "evaluated_paths": str(evaluated_paths)}
    if request is not None:
        doc["replay"] = replay_block(request)
    return doc


def _vega_kt_report(req: CompiledRequest, node_means, evaluated_paths: int) -> dict:
    """VegaKT raw buckets and projection of the local-vega node sensitivities
    (engine/risk/vegakt.rs:856, risk/local_vol_allocation.rs:108-163)."""
    from ._native import VegaKtBasisSpec, vega_kt_project
    plan, kt = req.plan, req.vega_kt
    basis = kt["reporting_iv_basis"]
    maturities = [float(t) for t in basis["maturity_nodes"]]
    forwards = [plan.spot * math.exp(log_discount(plan.dividend_times, plan.dividend_factors, t)
                                     - log_discount(plan.discount_times, plan.discount_factors, t))
                for t in maturities]
    spec = VegaKtBasisSpec(maturities, basis["log_forward_moneyness_nodes"], basis["implied_volatilities"],
                           forwards, float(kt["config"]["relative_density_threshold"]))
    g = plan.local_variance
    out, buckets = vega_kt_project(g.time_nodes, g.log_moneyness_nodes, node_means, evaluated_paths, spec)
    xs = list(basis["log_forward_moneyness_nodes"])
    vols = list(basis["implied_volatilities"])
    coordinates = [{"maturity": t, "log_moneyness": x, "implied_volatility": vols[i * len(xs) + j]}
                   for i, t in enumerate(maturities) for j, x in enumerate(xs)]
    return {"policy_label": NODE_ALLOCATION,
            "coordinates": coordinates, "raw_buckets": [float(b) for b in buckets],
            "projection": {"scalar_vega": out.scalar_vega, "signed_residual": out.signed_residual,
                           "pre_projection": out.pre_projection,
                           "reporting_stats": {"left_edge_count": int(out.left_edge_count),
                                               "right_edge_count": int(out.right_edge_count),
                                               "left_edge_sensitivity": out.left_edge_sensitivity,
                                               "right_edge_sensitivity": out.right_edge_sensitivity}},
            "residual_diagnostics": {"initial_time": out.initial_time,
                                     "excluded_probability_mass": out.density_excluded}}


def width_ladder(doc: dict) -> list:
    """The request's compact-C2 half-width ladder (PayoffSmoothingWidthLadder::new,
    crates/pricing/src/risk/request.rs:24-52): non-empty, positive, strictly
    monotone (two entries: distinct)."""
    ladder = [float(w) for w in _get(doc, "risk", "request").get("payoff_smoothing_width_ladder") or []]
    if not ladder:
        raise WireError("risk.payoff_smoothing_width_ladder is empty")
    for w in ladder:
        _positive(w, "risk.payoff_smoothing_width_ladder")
    if len(ladder) > 2:
        ascending = ladder[1] > ladder[0]
        if not all((b > a) if ascending else (b < a) for a, b in zip(ladder, ladder[1:])):
            raise WireError("risk.payoff_smoothing_width_ladder must be strictly monotone")
    elif len(ladder) == 2 and ladder[0] == ladder[1]:
        raise WireError("risk.payoff_smoothing_width_ladder must be strictly monotone")
    return ladder


def evaluate_width_ladder(doc: dict, *, reduction_block_size: int = 4096, price=None) -> dict:
    """PricingPlan::evaluate_width_ladder (crates/pricing/src/engine/risk/pricing.rs:53-84,329-393):
    the primary request (its own smoothing, the ladder removed) and the same
    request at every half-width of the ladder, all on the same engine seeds and
    therefore the same random coordinates; each entry carries its raw
    difference from the previous entry (price, Delta, Gamma, Vega).  `price`
    evaluates one request document (default: price_request on the GPU)."""
    price = price or (lambda d: price_request(d, reduction_block_size=reduction_block_size))
    ladder = width_ladder(doc)
    base = json_copy(doc)
    base["risk"].pop("payoff_smoothing_width_ladder", None)
    primary = price(base)
    entries = []
    for half_width in ladder:
        request = json_copy(base)
        request["risk"]["payoff_smoothing"] = {"type": "compact_c2", "half_width": half_width}
        result = price(request)
        difference = None
        if entries:
            prev = entries[-1]["result"]
            difference = {"price": result["value"]["value"] - prev["value"]["value"]}
            for k in ("delta", "gamma", "vega"):
                cur, old = result["risks"].get(k), prev["risks"].get(k)
                difference[k] = cur["raw"]["value"] - old["raw"]["value"] if cur and old else None
        entries.append({"half_width": half_width, "result": result, "adjacent_difference": difference})
    return {"primary": primary, "entries": entries}


def json_copy(doc):
    import copy
    return copy.deepcopy(doc)


def price_request(doc: dict, *, reduction_block_size: int = 4096, stream: int = 0,
                  node_allocation_diagnostic: bool = False) -> dict:
    """Price one v3 request on the GPU and return its `pricing_result` document.

    A local-volatility request whose VegaKT the reference computes by terminal
    replication (see _terminal_replication_applies) raises UnsupportedRequest:
    that market-IV method is not built here, and node allocation would give a
    different VegaKT document.  `node_allocation_diagnostic=True` asks for the
    node allocation anyway; the VegaKT document then names its method in
    `policy_label`."""
    from . import _native as N
    req = compile_request(doc, reduction_block_size=reduction_block_size)
    if req.vega_kt is not None and req.vega_kt["policy"] == TERMINAL_REPLICATION and not node_allocation_diagnostic:
        raise UnsupportedRequest("VegaKT of a statically replicable terminal payoff: the reference reports its "
                                 "terminal-replication market-IV risk (terminal_payoff_replication_iv_v1), which "
                                 "this engine does not compute; pass node_allocation_diagnostic=True for the "
                                 "local-vega node allocation")
    if req.lsm is not None:
        buf = N.lsm_price(req.plan, req.lsm, stream=stream)
        r = buf.result
        return result_document(req, r.price, r.delta, r.gamma, r.vega, r.sampling_variance,
                               r.estimator_variance, r.valuation_paths, request=doc)
    with N.Plan(req.plan) as plan:
        buf = plan.evaluate(stream)
    p = buf.products[0]
    r = buf.result
    kt = None
    if req.vega_kt is not None:
        kt = _vega_kt_report(req, [e.value for e in buf.node_estimates], r.evaluated_paths)
    return result_document(req, p.price, p.delta, p.gamma, p.vega, p.sampling_variance, p.estimator_variance,
                           r.evaluated_paths, kt, request=doc)

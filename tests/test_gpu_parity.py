"""Engine vs oracle parity on identical draws (small sizes), plus the
reference's own replay values and the analytic benchmark.

Tolerances are in gpu_common: 1e-12 of the component's scale for estimates,
1e-8 for CRN bump-validation components (they divide last-ulp libm
differences by the bump).
"""
import json
import os
import math

import pytest

import helpers as H
import lv_cases as L
import gpu_common as G
from bs_closed_form import black_scholes
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W
from rust_pricing_b200.desc import PlanSpec, ProductSpec
from test_oracle_fixtures import replay_cases, replay_spec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", replay_cases(), ids=lambda c: c["name"])
def test_replay_against_reference_values(engine, case):
    spec = replay_spec(case)
    buf = G.run_engine(spec)
    p, e = buf.products[0], case["expected"]
    for est, key in ((p.price, "price"), (p.delta, "delta"), (p.gamma, "gamma"), (p.vega, "vega")):
        assert abs(est.value - e[key]) <= 1e-12 * abs(e[key]), key
        assert abs(est.standard_error - e[key + "_standard_error"]) <= 1e-9 * e[key + "_standard_error"]
    G.assert_parity(spec, engine_buf=buf)


@pytest.mark.parametrize("case", L.cases(), ids=lambda c: c["name"])
def test_local_vol_replay_against_reference_values(engine, case):
    """The 3 x 5 local-variance grid requests of the reference's replay fixture
    (pseudo 8192 antithetic units; RQMC 512 x 8, bridge): price, CRN Delta and
    Gamma, reverse-sweep Vega within 1e-12 of the reference's values."""
    spec = L.plan(case)
    buf = G.run_engine(spec)
    p = buf.products[0]
    e = case["expected"]["windows-x86_64"]
    ests = [("price", p.price, e["value"])] + [(k, getattr(p, k), v) for k, v in e["risks"].items()]
    for name, est, want in ests:
        assert abs(est.value - want["value"]) <= G.DIRECT_TOL * max(abs(want["value"]), want["standard_error"]), name
        assert abs(est.standard_error - want["standard_error"]) <= 1e-9 * want["standard_error"], name
    G.assert_parity(spec, engine_buf=buf)


@pytest.mark.parametrize("case", [c for c in L.cases() if "node_allocation" in c], ids=lambda c: c["name"])
def test_local_vol_vega_kt_node_allocation(engine, case):
    """The engine's local-vega node sensitivities of the LV replay risk cases,
    allocated to the reporting-IV buckets by mcg_vega_kt_project, against the
    reference's node-allocation audit values (1e-12: the node sums are reduced
    on the device in another order)."""
    spec = L.plan(case)
    spec.request_local_vega_nodes = True
    buf = G.run_engine(spec)
    means = [e.value for e in buf.node_estimates]
    g = case["local_variance_grid"]
    out, buckets = N.vega_kt_project(g["time_nodes"], g["log_forward_moneyness_nodes"], means,
                                     buf.result.evaluated_paths, L.vega_kt_basis(case))
    L.check_node_allocation(out, buckets, case["node_allocation"], 1e-12)


@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
@pytest.mark.parametrize("antithetic", [False, True])
def test_european_risk_parity(engine, engine_kind, antithetic):
    spec = W.european_bs(paths=1 << 13 if engine_kind == A.ENGINE_RQMC else 20001, engine=engine_kind,
                         antithetic=antithetic, scrambles=8)
    G.assert_parity(spec)


def test_digital_and_put_parity(engine):
    for product in (ProductSpec(kind=A.PRODUCT_DIGITAL, side=A.PUT, payout=2.0),
                    ProductSpec(kind=A.PRODUCT_DIGITAL, digital_payout=A.DIGITAL_ASSET),
                    ProductSpec(kind=A.PRODUCT_EUROPEAN, side=A.PUT, strike=90.0)):
        spec = W.european_bs(paths=10007)
        spec.products = [product]
        G.assert_parity(spec)
        spec.smoothing_half_width = 0.5
        G.assert_parity(spec)


def _bs_multi(engine_kind, smoothing, antithetic):
    times = W.daily_times(52)
    prods = [ProductSpec(kind=A.PRODUCT_ASIAN, weights=[1 / 52] * 52),
             ProductSpec(kind=A.PRODUCT_LOOKBACK, side=A.PUT),
             ProductSpec(kind=A.PRODUCT_CONTINUOUS_BARRIER, barrier=85.0, rebate=1.0),
             ProductSpec(kind=A.PRODUCT_DISCRETE_BARRIER, barrier=120.0, barrier_direction=A.BARRIER_UP,
                         barrier_style=A.KNOCK_IN)]
    return PlanSpec(observation_times=times, products=prods, engine=engine_kind,
                    sampling_units=512 if engine_kind == A.ENGINE_RQMC else 4099, scramble_count=8,
                    antithetic=antithetic, smoothing_half_width=smoothing, **W.flat_curves())


@pytest.mark.parametrize("engine_kind", [A.ENGINE_PSEUDO, A.ENGINE_RQMC])
@pytest.mark.parametrize("smoothing", [0.0, 0.5])
def test_black_scholes_path_products(engine, engine_kind, smoothing):
    G.assert_parity(_bs_multi(engine_kind, smoothing, antithetic=engine_kind == A.ENGINE_PSEUDO))


@pytest.fixture(scope="module")
def grid(engine):
    return G.gpu_grid


def test_local_vol_rqmc_bridge(engine, grid):
    G.assert_parity(W.local_vol_rqmc(grid, points=1 << 10, scrambles=4))


@pytest.mark.parametrize("bridge", [False, True])
def test_local_vol_pseudo(engine, grid, bridge):
    G.assert_parity(W.local_vol_rqmc(grid, points=1500, engine=A.ENGINE_PSEUDO, bridge=bridge))


@pytest.mark.parametrize("smoothing", [0.0, 0.5])
@pytest.mark.parametrize("antithetic", [False, True])
def test_local_vol_continuous_barrier_crn_greeks(engine, grid, smoothing, antithetic):
    spec = W.local_vol_adjoint(grid, paths=1024, smoothing=smoothing)
    spec.antithetic = antithetic
    G.assert_parity(spec)


def test_local_vol_short_grid_with_substeps(engine, grid):
    """Observations coarser than the surface rows: the time grid substeps."""
    surface = W.SsviSurface(steps=40, expiries=20)
    spec = W.local_vol_rqmc(grid, points=256, scrambles=2, steps=40, surface=surface)
    spec.observation_times = [surface.time_nodes[-1] * i / 8 for i in range(1, 9)]
    spec.products = [ProductSpec(kind=A.PRODUCT_EUROPEAN), ProductSpec(kind=A.PRODUCT_LOOKBACK)]
    G.assert_parity(spec)


def test_european_statistical_acceptance_full_size(engine):
    """2^20 paths: estimates within 4 SE of the closed form (the reference's acceptance check)."""
    spec = W.european_bs(paths=1 << 20)
    p = G.run_engine(spec).products[0]
    cf = black_scholes(True, 100.0, 100.0, 1.0, W.RATE, W.DIVIDEND, 0.2)
    for est, key in ((p.price, "price"), (p.delta, "delta"), (p.vega, "vega"), (p.gamma, "gamma")):
        assert abs(est.value - cf[key]) <= 4.0 * est.standard_error, key


def test_evaluation_is_deterministic(engine, grid):
    spec = W.local_vol_rqmc(grid, points=1 << 12, scrambles=4)
    a, b = G.run_engine(spec), G.run_engine(spec)
    for k in range(2):
        for c in range(A.PATHWISE_COMPONENTS):
            x, y = a.products[k].components[c], b.products[k].components[c]
            assert (x.sum, x.correction, x.count, x.mean, x.second_moment) == \
                   (y.sum, y.correction, y.count, y.mean, y.second_moment)

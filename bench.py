#!/usr/bin/env python
"""Benchmark of the B200 Monte Carlo engine on the local-volatility RQMC workload.

Workload (one "step" = one evaluation of the whole workload):
  SSVI surface (theta = 0.04 t, rho = -0.4, eta = 1, gamma = 0.5) -> Dupire
  local-variance grid 31 x 100, 252 daily Log-Euler steps, T = 1, 2^20 Sobol
  points x 16 scrambles with a Brownian-bridge plan, an arithmetic-average Asian
  call K = 100 and a discrete down-and-out call (B = 80, daily, rebate 1) priced
  on the same draws.  2^24 paths x 252 steps = 4.23e9 path-steps per step.
  Synthetic market (S = 100, r = 3%, q = 1%); FP64 arithmetic.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Weak scaling: rank r evaluates scrambles [16 r, 16 r + 16) of one plan, so each
GPU's work is fixed; after the timed region each rank's price statistics are
gathered to rank 0 and merged (rust_pricing_b200/shards.py).
`--impl reference` times the CPU restatement of the reference's executor (the
oracle) on this host's cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "rust-pricing-library_b200")
sys.path.insert(0, PKG)

METRIC = "path-steps/s on 1 B200; time to 1bp price err: batched/adjoint/learned vs plain"
UNIT = "path-steps/s"
POINTS, SCRAMBLES, STEPS = 1 << 20, 16, 252
# Algorithmic FP64 operations per path-step of this workload (each IEEE result
# counts once; div, sqrt, log and exp count as one operation each):
#   AS241 central branch 33 (+ 15% tails x 31) + midpoint map 2 + bridge node 5
#   + increment 2 + Log-Euler step 27 (f/F, ln, clamp, x weight 3, bilinear 12,
#   sqrt, exponent 5, exp, ratio and state products 2) + Asian 2 + barrier 4.
FLOPS_PER_PATH_STEP = 33 + 0.15 * 31 + 2 + 5 + 2 + 27 + 2 + 4
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--points", type=int, default=POINTS)
    ap.add_argument("--scrambles", type=int, default=SCRAMBLES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--precision", choices=["f64", "f32"], default="f64",
                    help="path arithmetic of the timed workload (f32: FP32 path bulk)")
    ap.add_argument("--path-risk-units", type=int, default=1 << 20,
                    help="pseudo paths of the BS path-risk secondary measurement")
    ap.add_argument("--dual-units", type=int, default=1 << 14,
                    help="antithetic outer units of the Andersen-Broadie secondary measurement")
    ap.add_argument("--secondary", default="all",
                    help="comma list of secondary measurements: european, early_exercise, book, f32, "
                         "adjoint, path_risk, dual; all; none")
    ap.add_argument("--adjoint-paths", type=int, default=1 << 20)
    ap.add_argument("--lsm-units", type=int, default=1 << 20)
    ap.add_argument("--book-trades", type=int, default=4096)
    ap.add_argument("--book-units", type=int, default=1 << 16)
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def workload(points, scrambles, builder, scramble_begin=0, precision="f64"):
    from rust_pricing_b200 import _abi as A
    from rust_pricing_b200 import workloads as W
    spec = W.local_vol_rqmc(builder, points=points, scrambles=scrambles)
    spec.scramble_begin = scramble_begin
    spec.precision = A.PRECISION_F32_BULK if precision == "f32" else A.PRECISION_F64
    return spec


def gpu_grid(surface, floor, cap):
    import numpy as np
    from rust_pricing_b200 import _native as N
    tt, tv, slope, rho, eta, gamma, tn, xn = surface.grid_args()
    arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (tt, tv, tn, xn)]
    out = np.zeros(len(tn) * len(xn))
    rep = C.c_uint32()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    N.check(N.library().mcg_ssvi_local_variance_grid(
        dp(arr[0]), dp(arr[1]), len(tt), slope, rho, eta, gamma, dp(arr[2]), len(tn), dp(arr[3]),
        len(xn), floor, cap, dp(out), C.byref(rep)))
    return out.reshape(len(tn), len(xn))


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return {}


def cpu_baseline(points: int, scrambles: int, threads: int, grid_builder=None):
    """The oracle (CPU restatement of the reference executor) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers as H
    from rust_pricing_b200 import workloads as W
    if grid_builder is None:
        import gpu_common as G
        grid_builder = G.oracle_grid
    spec = W.local_vol_rqmc(grid_builder, points=points, scrambles=scrambles)
    spec.reduction_block_size = 256
    t0 = time.perf_counter()
    H.oracle_evaluate(spec, threads)
    dt = time.perf_counter() - t0
    path_steps = points * scrambles * STEPS
    return path_steps / dt, dt, path_steps


def time_to_bp(ms: float, se: float, price: float) -> float:
    """Device time to a 1 bp standard error (SE <= 1e-4 |price|), scaling the
    measured time by the variance ratio."""
    target = 1e-4 * abs(price)
    return ms * (se / target) ** 2 if target > 0 else float("inf")


def book_secondary(trades: int, units: int):
    """The batched-book configuration: `trades` seeded single-product trades
    (maturities U(0.1, 3) y with daily steps, strikes U(70, 130), 40/25/20/15 %
    European/Asian/continuous down-and-out/lookback, half Black--Scholes, half
    local volatility on their own SSVI grids), `units` pseudo paths each, in
    one persistent launch replayed from a CUDA graph, against pricing the same
    trades one plan per call."""
    from rust_pricing_b200 import _native as N, workloads as W
    t0 = time.perf_counter()
    specs = W.batched_book(gpu_grid, trades=trades, units=units)
    t1 = time.perf_counter()
    book = N.Book(specs, autotune=True, use_graph=True)
    t2 = time.perf_counter()
    book.evaluate()
    prices, rep = book.evaluate()
    book.close()
    out = {"workload": f"{trades} trades x {units} pseudo paths (seed {W.BOOK_SEED}), one persistent launch",
           "device_ms": rep.device_ms, "path_steps": rep.path_steps,
           "path_steps_per_s": rep.path_steps / (rep.device_ms * 1e-3), "work_items": rep.items,
           "tiles_per_item": rep.tiles_per_item, "ctas_per_sm": rep.ctas_per_sm, "graph": bool(rep.graph),
           "autotune_s": rep.autotune_ms * 1e-3, "create_s": t2 - t1, "generate_s": t1 - t0}
    # plain: the same trades, one plan and one evaluation each, device time
    # (path kernel + reduction of each call, CUDA events) against the book's
    plans = [N.Plan(sp) for sp in specs]
    for p in plans[:4]:
        p.evaluate()
    dev_plain, t3 = 0.0, time.perf_counter()
    for p in plans:
        dev_plain += p.evaluate().result.device_ms
    wall_plain = time.perf_counter() - t3
    for p in plans:
        p.close()
    out["plain_one_plan_per_call"] = {"trades": len(specs), "device_ms": dev_plain, "wall_ms": wall_plain * 1e3,
                                      "path_steps_per_s": rep.path_steps / (dev_plain * 1e-3)}
    out["batched_over_plain_device_time"] = dev_plain / rep.device_ms
    return out


def time_to_pct(ms: float, se: float, value: float) -> float:
    """Device time to a 1 % standard error of a Greek (SE <= 0.01 |value|)."""
    target = 1e-2 * abs(value)
    return ms * (se / target) ** 2 if target > 0 else float("inf")


def adjoint_secondary(paths: int = 1 << 20):
    """The adjoint configuration: a continuous down-and-out call (B = 80,
    rebate 1) under the SSVI local-variance grid, compact-C2 smoothing 0.5,
    `paths` pseudo paths x 252 daily steps.
      adjoint: one forward pass and one reverse sweep give the price, the
        adjoint Delta, the Vega and all 3100 grid-node sensitivities;
      adjoint_full: CRN Delta/Gamma, adjoint Delta, bumped-adjoint Gamma,
        Vega and the nodes (three spot runtimes forward and reversed);
      plain: the price with CRN Delta/Gamma (the reference's local-volatility
        Delta and Gamma are central bumps); a node sensitivity without the
        adjoint is two bumped revaluations of the price."""
    from rust_pricing_b200 import _native as N, workloads as W
    out = {"workload": f"continuous down-and-out call under SSVI local vol, compact-C2 0.5, {paths} pseudo "
                       "paths x 252 steps"}
    configs = {"adjoint": dict(delta=False, vega=True), "adjoint_full": dict(delta=True, vega=True),
               "plain": dict(delta=True, vega=False), "price_only": dict(delta=False, vega=False)}
    runs = {}
    for name, c in configs.items():
        spec = W.local_vol_adjoint(gpu_grid, paths=paths, risk=c["delta"])
        spec.request_vega = spec.request_local_vega_nodes = c["vega"]
        with N.Plan(spec) as plan:
            plan.evaluate()
            runs[name] = plan.evaluate()
    for name in ("adjoint", "adjoint_full"):
        r = runs[name]
        p, ms = r.products[0], r.result.device_ms
        out[name] = {"device_ms": ms, "price": p.price.value, "adjoint_delta": p.adjoint_delta.value,
                     "adjoint_delta_se": p.adjoint_delta.standard_error, "vega": p.vega.value,
                     "vega_se": p.vega.standard_error,
                     "ms_to_1pct_delta": time_to_pct(ms, p.adjoint_delta.standard_error, p.adjoint_delta.value),
                     "ms_to_1pct_vega": time_to_pct(ms, p.vega.standard_error, p.vega.value),
                     "node_sensitivities": len(r.node_estimates) if r.node_estimates is not None else 0}
    pl, po = runs["plain"], runs["price_only"]
    pp, ms_p, ms_0 = pl.products[0], pl.result.device_ms, po.result.device_ms
    out["plain"] = {"device_ms": ms_p, "price": pp.price.value, "crn_delta": pp.delta.value,
                    "crn_delta_se": pp.delta.standard_error,
                    "ms_to_1pct_delta": time_to_pct(ms_p, pp.delta.standard_error, pp.delta.value),
                    "price_only_ms": ms_0, "ms_for_3000_node_sensitivities_by_bumping": 2 * 3000 * ms_0}
    out["plain_over_adjoint_time_to_1pct_delta"] = out["plain"]["ms_to_1pct_delta"] / out["adjoint"]["ms_to_1pct_delta"]
    out["plain_over_adjoint_node_sensitivities"] = (out["plain"]["ms_for_3000_node_sensitivities_by_bumping"] /
                                                    out["adjoint"]["device_ms"])
    return out


def path_risk_secondary(units: int = 1 << 20, cpu_units: int = 1 << 14):
    """Black--Scholes pathwise risk of path-dependent products (the reference's
    pathwise_values over pathwise_aad): an arithmetic Asian call on 252 daily
    fixings and a continuous down-and-out call (B = 80, rebate 1, compact-C2
    0.5), S = K = 100, r = 3 %, q = 1 %, sigma = 0.2, T = 1, `units` pseudo
    paths, Delta / Gamma (1 % relative bump) / Vega with the CRN validation
    bumps: 7 evaluations of every path.  The oracle on the host's cores
    prices `cpu_units` paths of the same plan for comparison."""
    from rust_pricing_b200 import _abi as A, _native as N
    from rust_pricing_b200.desc import PlanSpec, ProductSpec
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers as H
    times = [(i + 1) / STEPS for i in range(STEPS)]
    products = {
        "asian_call": ProductSpec(kind=A.PRODUCT_ASIAN, strike=100.0, weights=[1.0 / STEPS] * STEPS),
        "continuous_down_and_out": ProductSpec(kind=A.PRODUCT_CONTINUOUS_BARRIER, strike=100.0, barrier=80.0,
                                               barrier_direction=A.BARRIER_DOWN, barrier_style=A.KNOCK_OUT,
                                               rebate=1.0),
    }
    out = {"workload": f"BS path risk, {units} pseudo paths x {STEPS} observations, Delta/Gamma/Vega + CRN "
                       "validation bumps (7 evaluations per path)"}
    for name, prod in products.items():
        spec = PlanSpec(observation_times=times, products=[prod], sampling_units=units, master_seed=20260904,
                        request_delta=True, request_gamma=True, request_vega=True, gamma_bump=0.01,
                        smoothing_half_width=0.5 if prod.kind == A.PRODUCT_CONTINUOUS_BARRIER else 0.0)
        with N.Plan(spec) as plan:
            plan.evaluate()
            r = min((plan.evaluate() for _ in range(3)), key=lambda b: b.result.device_ms)
        p, ms = r.products[0], r.result.device_ms
        evaluations = units * STEPS * 7
        spec.sampling_units = cpu_units
        t0 = time.perf_counter()
        H.oracle_evaluate(spec, threads=os.cpu_count() or 1)
        cpu_s = time.perf_counter() - t0
        out[name] = {"device_ms": ms, "path_step_evaluations_per_s": evaluations / (ms * 1e-3),
                     "price": p.price.value, "delta": p.delta.value, "delta_se": p.delta.standard_error,
                     "gamma": p.gamma.value, "vega": p.vega.value, "vega_se": p.vega.standard_error,
                     "ms_to_1pct_delta": time_to_pct(ms, p.delta.standard_error, p.delta.value),
                     "kernel_launches": r.result.kernel_launches,
                     "cpu_oracle_path_step_evaluations_per_s": cpu_units * STEPS * 7 / cpu_s,
                     "cpu_threads": os.cpu_count() or 1}
    return out


def european_secondary(paths: int = 1 << 20, cpu_units: int = 1 << 24):
    """The plain European configuration: a Black--Scholes call S = K = 100,
    r = 3 %, q = 1 %, sigma = 20 %, T = 1, one exact lognormal step, `paths`
    pseudo paths (seed 0x0123456789abcdef), FP64, price with pathwise Delta and
    Vega and Gamma by a 1 % relative bump (which also fills the CRN validation
    components: 7 evaluations of every path), checked against the closed form.  The
    oracle on the host's cores prices `cpu_units` paths of the same plan."""
    from rust_pricing_b200 import _native as N, workloads as W
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers as H
    from bs_closed_form import black_scholes
    spec = W.european_bs(paths=paths)
    with N.Plan(spec) as plan:
        plan.evaluate()
        runs = [plan.evaluate() for _ in range(5)]
    r = min(runs, key=lambda b: b.result.device_ms)
    p, ms = r.products[0], r.result.device_ms
    cf = black_scholes(True, 100.0, 100.0, 1.0, W.RATE, W.DIVIDEND, 0.2)
    spec.sampling_units = cpu_units
    threads = os.cpu_count() or 1
    H.oracle_evaluate(spec, threads)
    t0 = time.perf_counter()
    H.oracle_evaluate(spec, threads)
    cpu_s = time.perf_counter() - t0
    out = {"workload": f"European BS call, {paths} pseudo paths, 1 exact step, FP64, price + pathwise Delta/Vega "
                       "+ 1 % relative Gamma bump (7 path evaluations per unit); checked against the closed form",
           "device_ms": ms, "path_steps_per_s": paths / (ms * 1e-3),
           "path_evaluations_per_s": 7 * paths / (ms * 1e-3), "kernel_launches": r.result.kernel_launches,
           "ms_to_1bp_standard_error": time_to_bp(ms, p.price.standard_error, p.price.value),
           "ms_to_1pct_delta": time_to_pct(ms, p.delta.standard_error, p.delta.value),
           "ms_to_1pct_vega": time_to_pct(ms, p.vega.standard_error, p.vega.value),
           "cpu_oracle_path_steps_per_s": cpu_units / cpu_s, "cpu_threads": threads,
           "cpu_sample": f"{cpu_units} paths, full risk ({cpu_s:.2f} s)"}
    for key, est in (("price", p.price), ("delta", p.delta), ("vega", p.vega), ("gamma", p.gamma)):
        out[key] = {"value": est.value, "standard_error": est.standard_error, "closed_form": cf[key],
                    "error_in_standard_errors": (est.value - cf[key]) / est.standard_error}
    out["gpu_over_cpu_oracle"] = out["path_steps_per_s"] / out["cpu_oracle_path_steps_per_s"]
    return out


def dual_secondary(units: int = 1 << 14, cpu_units: int = 2048):
    """Andersen--Broadie upper bound of the early-exercise configuration's
    American put (S = K = 100, r = 5 %, sigma = 25 %, T = 1, 50 exercise
    dates; cubic policy on 2^16 antithetic training units): `units` antithetic
    outer paths, 256 inner paths where the policy continues and 129 where it
    exercises, from every non-terminal date.  The oracle on the host's cores
    runs `cpu_units` outer units of the same plan for comparison."""
    from rust_pricing_b200 import _native as N, workloads as W
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers as H
    from bermudan_tree import bermudan_equally_spaced
    spec, lsm = W.american_bs(dates=50, units=units, training_units=1 << 16, antithetic=True)
    n2, n3, seed = 256, 129, 0x1234
    N.lsm_dual(spec, lsm, n2, n3, seed)
    r = min((N.lsm_dual(spec, lsm, n2, n3, seed) for _ in range(2)), key=lambda x: x.device_ms)
    tree = bermudan_equally_spaced(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 50, steps=5000)
    spec.sampling_units = cpu_units
    t0 = time.perf_counter()
    c = H.oracle_lsm_dual(spec, lsm, n2, n3, seed, threads=os.cpu_count() or 1)
    cpu_s = time.perf_counter() - t0
    return {"workload": f"Andersen-Broadie dual, American put, 50 dates, {units} x 2 outer paths, "
                        f"N2 = {n2}, N3 = {n3} inner paths; checked against a 5000-step Bermudan tree",
            "tree": tree, "device_ms": r.device_ms, "nested_ms": r.nested_ms,
            "lower_bound": r.lower_bound.value, "lower_se": r.lower_bound.standard_error,
            "upper_bound": r.upper_bound.value, "upper_se": r.upper_bound.standard_error,
            "duality_gap": r.duality_gap.value, "gap_se": r.duality_gap.standard_error,
            "inner_paths": r.inner_paths, "inner_paths_per_s": r.inner_paths / (r.nested_ms * 1e-3),
            "kernel_launches": r.kernel_launches,
            "cpu_oracle_inner_paths_per_s": c.inner_paths / cpu_s, "cpu_threads": os.cpu_count() or 1,
            "cpu_sample": f"{cpu_units} outer units, training included ({cpu_s:.1f} s)"}


def multi_asset_secondary(paths: int = 1 << 20, cpu_units: int = 1 << 14):
    """Correlated multi-asset paths: a four-asset basket call (two Black--Scholes
    assets, two local-volatility assets on their own SSVI Dupire grids),
    weights 0.4/0.3/0.2/0.1, strike 100, a correlation change at half a year,
    daily steps over one year, `paths` antithetic pseudo units.  The oracle on
    the host's cores prices `cpu_units` units of the same plan."""
    import math
    from rust_pricing_b200 import _abi as A, _native as N, workloads as W
    from rust_pricing_b200.desc import AssetSpec, MultiAssetSpec
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers as H

    def div(q):
        return dict(dividend_times=(0.0, 2.0), dividend_factors=(1.0, math.exp(-2.0 * q)))

    grids = [W.local_vol_grid(W.SsviSurface(steps=STEPS, expiries=30, rho=rho, eta=eta), gpu_grid)
             for rho, eta in ((-0.4, 1.0), (-0.3, 0.8))]
    assets = [AssetSpec(spot=100.0, volatility=0.2, **div(0.01)),
              AssetSpec(spot=95.0, model=A.MODEL_LOCAL_VOLATILITY, local_variance=grids[0], **div(0.02)),
              AssetSpec(spot=110.0, volatility=0.25, **div(0.0)),
              AssetSpec(spot=90.0, model=A.MODEL_LOCAL_VOLATILITY, local_variance=grids[1], **div(0.015))]
    rho = [[1.0, 0.5, 0.3, 0.1], [0.5, 1.0, 0.4, 0.2], [0.3, 0.4, 1.0, -0.3], [0.1, 0.2, -0.3, 1.0]]
    half = [[1.0 if i == j else 0.5 * rho[i][j] for j in range(4)] for i in range(4)]
    spec = MultiAssetSpec(assets=assets, correlations=[(-1.0 / 365, rho), (0.5, half)], strike=100.0,
                          weights=[0.4, 0.3, 0.2, 0.1], sampling_units=paths, antithetic=True,
                          brownian_bridge=False, maximum_step=1.0 / STEPS, reduction_block_size=4096,
                          discount_times=(0.0, 2.0), discount_factors=(1.0, math.exp(-0.06)))
    N.multi_asset_price(spec)
    r = min((N.multi_asset_price(spec) for _ in range(3)), key=lambda x: x.device_ms)
    asset_steps = paths * 2 * r.time_steps * len(assets)
    spec.sampling_units = cpu_units
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    c = H.oracle_multi(spec, threads)
    cpu_s = time.perf_counter() - t0
    return {"workload": f"4-asset basket call (2 BS + 2 SSVI local vol), correlation change at 0.5 y, "
                        f"{r.time_steps} daily steps, {paths} antithetic pseudo units",
            "device_ms": r.device_ms, "path_asset_steps_per_s": asset_steps / (r.device_ms * 1e-3),
            "price": r.price.value, "standard_error": r.price.standard_error,
            "ms_to_1bp_standard_error": time_to_bp(r.device_ms, r.price.standard_error, r.price.value),
            "kernel_launches": r.kernel_launches,
            "cpu_oracle_path_asset_steps_per_s": cpu_units * 2 * c.time_steps * len(assets) / cpu_s,
            "cpu_threads": threads, "cpu_sample": f"{cpu_units} units ({cpu_s:.1f} s)"}


def f32_secondary(points: int, scrambles: int, prices64):
    """The timed workload with the FP32 path bulk: time and the error of each
    price against the FP64 run's."""
    from rust_pricing_b200 import _native as N
    spec = workload(points, scrambles, gpu_grid, precision="f32")
    with N.Plan(spec) as plan:
        plan.evaluate()
        times, r = [], None
        for _ in range(3):
            r = plan.evaluate()
            times.append(r.result.device_ms)
    p32 = [r.products[k].price.value for k in range(len(spec.products))]
    return {"ms_per_step": min(times), "path_steps_per_s": points * scrambles * STEPS / (min(times) * 1e-3),
            "prices": p32, "relative_error_vs_f64": [(a - b) / b for a, b in zip(p32, prices64)],
            "error_in_standard_errors": None}


def lsm_secondary(units: int = 1 << 20):
    """The early-exercise configuration (American put S=K=100, r=5%, sigma=25%,
    T=1, 50 dates, 2^20 training + 2^20 valuation paths): the reference's
    polynomial policy and the learned continuation, against the 5000-step
    Bermudan binomial tree.  One untimed warm-up, then one timed evaluation each."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from bermudan_tree import bermudan_equally_spaced
    from rust_pricing_b200 import _abi as A, _native as N, workloads as W
    tree = bermudan_equally_spaced(100.0, 100.0, 0.05, 0.0, 0.25, 1.0, 50, steps=5000)
    out = {"workload": f"American put by LSM, 50 dates, {units} + {units} paths, cubic basis; checked against a 5000-step "
                       "Bermudan binomial tree", "tree": tree}
    for name, kind in (("plain", A.CONTINUATION_POLYNOMIAL), ("learned", A.CONTINUATION_MLP)):
        spec, lsm = W.american_bs(dates=50, units=units)
        lsm.continuation = kind
        lsm.mlp_seed = 7
        N.lsm_price(spec, lsm)
        r = N.lsm_price(spec, lsm).result
        # fitting is a fixed cost; only the valuation scales with the paths
        fixed = r.path_kernel_ms + r.regression_ms + r.mlp_ms
        out[name] = {"device_ms": r.device_ms, "fit_ms": fixed, "valuation_ms": r.device_ms - fixed,
                     "price": r.price.value, "standard_error": r.price.standard_error,
                     "error_vs_tree": r.price.value - tree, "policy": "mlp" if r.continuation_used else "polynomial",
                     "path_steps_per_s": 2 * units * 50 / (r.device_ms * 1e-3),
                     "ms_to_1bp_standard_error": fixed + time_to_bp(r.device_ms - fixed, r.price.standard_error,
                                                                    r.price.value),
                     "kernel_launches": r.kernel_launches}
    return out


def sized_cpu_sample(threads: int, grid_builder=None, target_s: float = 15.0):
    """Points per scramble (a power of two, 2 scrambles) for about `target_s`
    seconds of oracle work on this host, from a short calibration run."""
    rate, _, _ = cpu_baseline(1 << 14, 1, threads, grid_builder)
    points, scrambles = 1 << 11, 2
    while points < (1 << 20) and 2 * scrambles * points * STEPS / rate <= target_s:
        points *= 2
    while scrambles < 16 and 2 * scrambles * points * STEPS / rate <= target_s:
        scrambles *= 2
    return points, scrambles


def run_reference(args, rank, world):
    """CPU executor (oracle port) on all host cores; rank 0 only."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup and 1):
        cpu_baseline(1 << 10, 1, threads)
    sample_points, sample_scrambles = sized_cpu_sample(threads)
    times = []
    for _ in range(args.steps):
        value, dt, ps = cpu_baseline(sample_points, sample_scrambles, threads)
        times.append(dt)
    per = statistics.mean(times)
    value = sample_points * sample_scrambles * STEPS / per
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "local-vol RQMC: SSVI->Dupire 31x100 grid, 252 daily steps, 2^20 Sobol points x 16 "
                               "scrambles, Brownian bridge, Asian call + discrete down-and-out on the same draws",
                   "sample": f"{sample_points} points x {sample_scrambles} scrambles per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sample_points} points x {sample_scrambles} scrambles x {STEPS} steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    import numpy as np
    import torch
    from rust_pricing_b200 import _native as N
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    handle = stream.cuda_stream
    spec = workload(args.points, args.scrambles, gpu_grid, scramble_begin=rank * args.scrambles,
                    precision=args.precision)
    plan = N.Plan(spec)
    path_steps_rank = args.points * args.scrambles * STEPS
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        res = plan.evaluate(handle)
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kernel_ms, launches = [], 0
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for k in range(args.steps):
            flush.zero_()
            events[k][0].record(stream)
            buf = plan.evaluate(handle)
            events[k][1].record(stream)
            kernel_ms.append(buf.result.path_kernel_ms)
            launches += buf.result.kernel_launches
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in events]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    # Prices of the whole job: every rank's scramble-shard statistics merged on
    # rank 0 in rank order (one rank: the plan's own estimates).
    if world > 1:
        from rust_pricing_b200 import shards
        merged = shards.gather_prices(buf, len(spec.products), rank, world)
    else:
        merged = [{"value": buf.products[k].price.value, "standard_error": buf.products[k].price.standard_error}
                  for k in range(len(spec.products))]
    ms_per_step = total_ms / args.steps
    value = world * path_steps_rank / (ms_per_step * 1e-3)

    # roofline of the dominant kernel (the path kernel): FP64 operations
    peak = C.c_double()
    N.check(N.library().mcg_measure_fp64_peak(C.c_void_p(handle), C.byref(peak)))
    path_ms = statistics.mean(kernel_ms)
    achieved = FLOPS_PER_PATH_STEP * path_steps_rank / (path_ms * 1e-3) / 1e12
    roofline = {"bound": "fp64" if args.precision == "f64" else "fp64 (FP32 path bulk: the FP64 figure only bounds it)",
                "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value if peak.value else None,
                # DRAM bytes of one path-kernel launch, scaled by CTA count from the ncu capture
                # of the 2^16-point x 16-scramble case (1.342208 MB read + 256 B written over
                # 4096 CTAs of two 128-unit tiles: grid, scramble tables and tile records, in
                # proportion to the CTAs)
                "traffic": (1.337088e6 + 256.0) * (args.points * args.scrambles / 256) / 4096,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the path kernel on the "
                                  "2^16-point x 16-scramble case, scaled by CTA count",
                "peak_source": "measured live: mcg_measure_fp64_peak (DFMA chains, this GPU)",
                "flops_per_path_step": FLOPS_PER_PATH_STEP, "kernel_ms": path_ms}

    # end to end: the C-ABI call with host buffers (plan compile + upload + run + results back)
    e2e_times = []
    desc = spec.desc()
    for _ in range(args.e2e_steps):
        rb = __import__("rust_pricing_b200._abi", fromlist=["_abi"]).ResultBuffers(len(spec.products))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        N.check(N.library().mcg_price(C.byref(desc), C.c_void_p(handle), C.byref(rb.result)), rb.result.error)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = min(e2e_times)
    grid_bytes = spec.grid_value_count() * 8 + (len(spec.local_variance.time_nodes) + len(spec.local_variance.log_moneyness_nodes)) * 8
    h2d = grid_bytes + spec._dimension_hint() * 32 * 4 + len(spec.observation_times) * 8 * 4 + 2 * STEPS * 8 * 12
    d2h = args.scrambles * len(spec.products) * 18 * 40 + 32
    e2e = {"value": world * path_steps_rank / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "seconds_per_step": e2e_s,
           "path": "mcg_price(): plan compile, upload, evaluate, statistics back"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "f64" else "f32 path bulk, f64 payoffs",
        "data": "synthetic",
        "config": {"workload": "local-vol RQMC: SSVI->Dupire 31x100 grid, 252 daily steps, 2^20 Sobol points x 16 "
                               "scrambles, Brownian bridge, Asian call + discrete down-and-out on the same draws",
                   "points_per_scramble": args.points, "scrambles_per_gpu": args.scrambles, "time_steps": STEPS,
                   "path_steps_per_gpu": path_steps_rank, "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"scramble shards x{world}"},
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "prices": [m["value"] for m in merged] if merged else None,
        "price_standard_errors": [m["standard_error"] for m in merged] if merged else None,
        "ms_to_1bp_standard_error": [time_to_bp(ms_per_step, m["standard_error"], m["value"])
                                     for m in merged] if merged else None,
    }
    wanted = {"european", "early_exercise", "book", "f32", "adjoint", "path_risk", "dual",
              "multi_asset"} if args.secondary == "all" else (
        set() if args.secondary == "none" else set(args.secondary.split(",")))
    if rank == 0 and world == 1 and wanted:
        sec = {}
        if "european" in wanted:
            sec["european"] = european_secondary()
        if "early_exercise" in wanted:
            sec["early_exercise"] = lsm_secondary(args.lsm_units)
        if "f32" in wanted and args.precision == "f64":
            f32 = f32_secondary(args.points, args.scrambles, line["prices"])
            f32["error_in_standard_errors"] = [e * p / se for e, p, se in zip(
                f32["relative_error_vs_f64"], line["prices"], line["price_standard_errors"])]
            sec["f32_bulk"] = f32
        if "book" in wanted:
            sec["batched_book"] = book_secondary(args.book_trades, args.book_units)
        if "adjoint" in wanted:
            sec["adjoint"] = adjoint_secondary(args.adjoint_paths)
        if "path_risk" in wanted:
            sec["bs_path_risk"] = path_risk_secondary(args.path_risk_units)
        if "dual" in wanted:
            sec["dual_upper_bound"] = dual_secondary(args.dual_units)
        if "multi_asset" in wanted:
            sec["multi_asset"] = multi_asset_secondary()
        line["secondary"] = sec
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample_points, sample_scrambles = sized_cpu_sample(threads, grid_builder=gpu_grid)
        value_cpu, dt, ps = cpu_baseline(sample_points, sample_scrambles, threads, grid_builder=gpu_grid)
        line["cpu_baseline"] = {"value": value_cpu, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{sample_points} points x {sample_scrambles} scrambles x {STEPS} steps "
                                          f"({ps:.3g} path-steps, {dt:.1f} s)"}
    plan.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

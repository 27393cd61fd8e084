"""Implied-variance surfaces of the reference's equation fixture
(tests/golden/surfaces.json, from fixtures/local-vol/reference-cases-v0.1.json)
and of the reference's own unit tests, as SurfaceSpecs."""
import ctypes as C
import json
import os

import numpy as np

import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200.desc import SurfaceSpec  # noqa: F401  (re-exported for tests)


def golden():
    return json.load(open(os.path.join(H.GOLDEN, "surfaces.json")))


def ssvi_case_surface(case: dict) -> tuple[SurfaceSpec, float, float]:
    """A standard-SSVI case gives theta and its time derivative at one time:
    a two-knot theta curve through (1, theta) with slope theta_t reproduces
    both at t = 1 (a PCHIP with two knots is the line through them)."""
    i = case["inputs"]
    theta, theta_t = float(i["theta"]), float(i["theta_t"])
    common = dict(theta_times=[1.0, 2.0], theta_values=[theta, theta + theta_t], terminal_theta_slope=theta_t,
                  rho=float(i["rho"]))
    if "lambda" in i:
        s = SurfaceSpec(kind=A.SURFACE_SSVI_HESTON_LIKE, lam=float(i["lambda"]), **common)
    else:
        s = SurfaceSpec(kind=A.SURFACE_SSVI_POWER_LAW, eta=float(i["eta"]), gamma=float(i["gamma"]), **common)
    return s, 1.0, float(i["k"])


def essvi_case_surface(case: dict) -> tuple[SurfaceSpec, float, float]:
    i = case["inputs"]
    s = SurfaceSpec(kind=A.SURFACE_ESSVI, slice_times=[float(i["t0"]), float(i["t1"])],
                    slice_thetas=[float(i["theta0"]), float(i["theta1"])],
                    slice_psis=[float(i["psi0"]), float(i["psi1"])],
                    slice_rho_psis=[float(i["rho_psi0"]), float(i["rho_psi1"])], terminal_theta_slope=0.02)
    return s, float(i["t"]), float(i["k"])


def unit_test_essvi() -> SurfaceSpec:
    """valid_surface() of crates/pricing/src/market/essvi.rs tests."""
    return SurfaceSpec(kind=A.SURFACE_ESSVI, slice_times=[1.0, 2.0], slice_thetas=[0.04, 0.09],
                       slice_psis=[0.2, 0.25], slice_rho_psis=[-0.08, -0.05], terminal_theta_slope=0.02)


def oracle_total_variance(surface: SurfaceSpec, t: float, k: float) -> np.ndarray:
    out = np.zeros(4)
    d = surface.desc()
    rc = H.oracle().oracle_surface_total_variance(C.byref(d), t, k, H.dptr(out))
    assert rc == 0
    return out


def oracle_grid(surface: SurfaceSpec, tn, xn, floor=1e-8, cap=4.0):
    tn, xn = (np.ascontiguousarray(a, dtype=np.float64) for a in (tn, xn))
    out = np.zeros(len(tn) * len(xn))
    d = surface.desc()
    repairs = H.oracle().oracle_surface_grid(C.byref(d), H.dptr(tn), len(tn), H.dptr(xn), len(xn), floor, cap,
                                             H.dptr(out))
    return out.reshape(len(tn), len(xn)), repairs


def grid_surfaces():
    """Surfaces of every kind over the C2 grid shape (30 expiries, 100 nodes)."""
    from rust_pricing_b200 import workloads as W
    base = W.SsviSurface()
    heston = SurfaceSpec(kind=A.SURFACE_SSVI_HESTON_LIKE, theta_times=base.theta_times,
                         theta_values=base.theta_values, terminal_theta_slope=base.terminal_slope, rho=-0.4,
                         lam=2.0)
    power = SurfaceSpec(kind=A.SURFACE_SSVI_POWER_LAW, theta_times=base.theta_times, theta_values=base.theta_values,
                        terminal_theta_slope=base.terminal_slope, rho=-0.4, eta=1.0, gamma=0.5)
    times = [0.25, 0.5, 1.0, 1.5]
    thetas = [0.01, 0.02, 0.04, 0.06]
    psis = [0.1, 0.14, 0.2, 0.24]
    essvi = SurfaceSpec(kind=A.SURFACE_ESSVI, slice_times=times, slice_thetas=thetas, slice_psis=psis,
                        slice_rho_psis=[-0.3 * p for p in psis], terminal_theta_slope=0.04)
    return {"power": power, "heston": heston, "essvi": essvi}, base.time_nodes, base.log_moneyness_nodes

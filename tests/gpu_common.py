"""Helpers of the GPU parity tests: run a plan on the engine and on the oracle."""
import ctypes as C

import numpy as np

import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import workloads as W

# Tolerances, relative to the component's scale (|total| or its spread):
#   direct estimates (price, AAD Delta/Vega, bumped-AAD Gamma, CRN LV Greeks): 1e-12,
#   the CRN validation bumps and their differences divide last-ulp libm
#   differences by the bump size (1e-4 for volatility), so they get 1e-8.
DIRECT_TOL = 1e-12
BUMP_TOL = 1e-8
BUMP_COMPONENTS = {A.BUMP_DELTA, A.DELTA_DIFFERENCE, A.BUMP_VEGA, A.VEGA_DIFFERENCE,
                   A.BUMP_GAMMA, A.GAMMA_DIFFERENCE}


def gpu_grid(surface, floor, cap):
    tt, tv, slope, rho, eta, gamma, tn, xn = surface.grid_args()
    tt, tv, tn, xn = (np.ascontiguousarray(a, dtype=np.float64) for a in (tt, tv, tn, xn))
    out = np.zeros(len(tn) * len(xn))
    rep = C.c_uint32()
    N.check(N.library().mcg_ssvi_local_variance_grid(
        H.dptr(tt), H.dptr(tv), len(tt), slope, rho, eta, gamma, H.dptr(tn), len(tn), H.dptr(xn),
        len(xn), floor, cap, H.dptr(out), C.byref(rep)))
    return out.reshape(len(tn), len(xn))


def oracle_grid(surface, floor, cap):
    tt, tv, slope, rho, eta, gamma, tn, xn = surface.grid_args()
    tt, tv, tn, xn = (np.ascontiguousarray(a, dtype=np.float64) for a in (tt, tv, tn, xn))
    out = np.zeros(len(tn) * len(xn))
    assert H.oracle().oracle_ssvi_grid(H.dptr(tt), H.dptr(tv), len(tt), slope, rho, eta, gamma,
                                       H.dptr(tn), len(tn), H.dptr(xn), len(xn), floor, cap, H.dptr(out)) >= 0
    return out.reshape(len(tn), len(xn))


def run_engine(spec):
    with N.Plan(spec) as plan:
        return plan.evaluate()


# A bump-minus-primary difference inherits the error of its bump component,
# which can be far larger than the (cancelling) difference itself.
DIFFERENCE_OF = {A.DELTA_DIFFERENCE: A.BUMP_DELTA, A.VEGA_DIFFERENCE: A.BUMP_VEGA,
                 A.GAMMA_DIFFERENCE: A.BUMP_GAMMA}


def _scale(stat):
    total = stat.sum + stat.correction
    return max(abs(total), (max(stat.second_moment, 0.0) * max(stat.count, 1)) ** 0.5)


def component_errors(spec, engine_buf, oracle_buf):
    """Scaled difference per product and component."""
    worst = []
    for k in range(len(spec.products)):
        comps = oracle_buf.products[k].components
        for c in range(A.PATHWISE_COMPONENTS):
            a = comps[c]
            b = engine_buf.products[k].components[c]
            at, bt = a.sum + a.correction, b.sum + b.correction
            scale = _scale(a)
            if c in DIFFERENCE_OF:
                scale = max(scale, _scale(comps[DIFFERENCE_OF[c]]))
            worst.append((abs(at - bt) / max(scale, 1e-300), k, c, at, bt))
    return worst


def assert_parity(spec, engine_buf=None, oracle_buf=None, threads=8):
    engine_buf = engine_buf or run_engine(spec)
    oracle_buf = oracle_buf or H.oracle_evaluate(spec, threads)
    for err, k, c, at, bt in component_errors(spec, engine_buf, oracle_buf):
        tol = BUMP_TOL if c in BUMP_COMPONENTS else DIRECT_TOL
        assert err <= tol, f"product {k} component {c}: oracle {at!r} engine {bt!r} (scaled error {err:.2e})"
    for k in range(len(spec.products)):
        a, b = oracle_buf.products[k], engine_buf.products[k]
        assert abs(a.price.value - b.price.value) <= DIRECT_TOL * max(abs(a.price.value), a.price.standard_error)
        assert abs(a.price.standard_error - b.price.standard_error) <= 1e-10 * max(a.price.standard_error, 1e-300)
        assert a.price.effective_sampling_units == b.price.effective_sampling_units
    return engine_buf, oracle_buf

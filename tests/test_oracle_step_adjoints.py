"""The oracle's local-volatility reverse sweep against the reference's
step-adjoint fixture (fixtures/local-vol/step-adjoints-v0.1.json, equation (10)
of SSRN 4107770: 100-digit Decimal path prices with five-point bumps of each
grid value; tests/golden/lv_step_adjoints.json).  One Log-Euler path per case
on the fixture's nodes, forwards, 3 x 3 variance grid and shocks, paying
sum_k q_k S_k^2 + c S_2 S_5; its states and the grid-value adjoints of the
oracle's reverse sweep (lv_reverse, the one the engine's adjoint kernel is
checked against) agree with the references within the fixture's relative
tolerance 1e-9 (interior, flat, and both clamped ends of the grid)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import helpers as H

FIXTURE = json.load(open(os.path.join(H.GOLDEN, "lv_step_adjoints.json")))


def _lib():
    lib = H.oracle()
    dp = C.POINTER(C.c_double)
    lib.oracle_lv_step_adjoints.argtypes = [dp, C.c_uint32, dp, dp, C.c_uint32, dp, C.c_uint32, dp, C.c_double,
                                            dp, dp, dp, dp]
    lib.oracle_lv_step_adjoints.restype = C.c_int
    return lib


@pytest.mark.parametrize("case", FIXTURE["cases"], ids=lambda c: c["id"])
def test_step_adjoints_match_the_decimal_references(case):
    arr = lambda k: np.ascontiguousarray(case[k], dtype=np.float64)
    times, fwd, gt, gx, gv, shocks = (arr(k) for k in ("simulation_times", "forwards", "grid_times", "nodes",
                                                        "variances", "shocks"))
    q = np.asarray(case["quadratic_weights"], dtype=np.float64)
    e = case["expected"]
    s = np.asarray(e["states"], dtype=np.float64)
    # dPayoff/dS_k of sum q_k S_k^2 + c S_2 S_5 at the path's states
    seeds = 2.0 * q * s
    seeds[2] += case["cross_weight"] * s[-1]
    seeds[-1] += case["cross_weight"] * s[2]
    seeds = np.ascontiguousarray(seeds)
    states, adj = np.zeros(len(times)), np.zeros(len(gv))
    rc = _lib().oracle_lv_step_adjoints(H.dptr(times), len(times), H.dptr(fwd), H.dptr(gt), len(gt), H.dptr(gx),
                                        len(gx), H.dptr(gv), case["initial"], H.dptr(shocks), H.dptr(seeds),
                                        H.dptr(states), H.dptr(adj))
    assert rc == 0
    rel = FIXTURE["relative_tolerance"]
    np.testing.assert_allclose(states, e["states"], rtol=1e-13)
    for got, want in zip(adj, e["grid_variance"]):
        assert abs(got - want) <= rel * abs(want) or (want == 0.0 and got == 0.0), (got, want)


DIRECT = json.load(open(os.path.join(H.GOLDEN, "lv_direct_variance.json")))


@pytest.mark.parametrize("case", DIRECT["cases"], ids=lambda c: c["id"])
def test_barrier_direct_variance_adjoints(case):
    """fixtures/local-vol/direct-variance-v0.1.json: an exact continuous
    barrier over the first `monitor_end` intervals of one Log-Euler path, with
    node variances at the path's states, paying a rebate or q S_T^2; the
    oracle's price and the grid-value adjoints of its reverse sweep (bridge
    state seeds plus direct variance seeds at the nodes) within 1e-9 of the
    100-digit references."""
    lib = H.oracle()
    dp = C.POINTER(C.c_double)
    lib.oracle_lv_barrier_adjoints.argtypes = [dp, C.c_uint32, dp, dp, C.c_uint32, dp, C.c_uint32, dp, C.c_double,
                                               dp, C.c_double, C.c_int, C.c_int, C.c_uint32, C.c_double,
                                               C.c_double, C.c_double, dp, dp]
    lib.oracle_lv_barrier_adjoints.restype = C.c_int
    arr = lambda k: np.ascontiguousarray(case[k], dtype=np.float64)
    times, fwd, gt, gx, gv, shocks = (arr(k) for k in ("times", "forwards", "grid_times", "nodes", "variances",
                                                        "shocks"))
    price = C.c_double()
    adj = np.zeros(len(gv))
    rc = lib.oracle_lv_barrier_adjoints(H.dptr(times), len(times), H.dptr(fwd), H.dptr(gt), len(gt), H.dptr(gx),
                                        len(gx), H.dptr(gv), case["initial"], H.dptr(shocks), case["barrier"],
                                        int(case["direction"] == "up"), int(case["style"] == "out"),
                                        case["monitor_end"], case["quadratic"], case["rebate"], case["discount"],
                                        C.byref(price), H.dptr(adj))
    assert rc == 0
    rel = DIRECT["relative_tolerance"]
    e = case["expected"]
    assert abs(price.value - e["price"]) <= rel * abs(e["price"])
    for got, want in zip(adj, e["grid_variance"]):
        assert abs(got - want) <= rel * abs(want) + 1e-12, (got, want)

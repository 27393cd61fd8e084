"""The oracle's regression pieces against the reference's early-exercise
reference cases (fixtures/early-exercise/reference-cases-v0.1.json, 80-digit
decimal expectations; tests/golden/early_exercise_cases.json):

* FeatureScaling::fit: mean, population variance and scale within 2 ulps of
  the decimal values, the zero-scale threshold 64 eps max(1, max |v|) exactly,
  the inactive flag;
* fit_cpqr: pivot order (largest remaining norm first, ties to the smaller
  original column), rank under the absolute and relative tolerances,
  coefficients in the original column order and the residual sum of squares;
* the decision rules the engine applies: exercise only when the immediate
  value is strictly above the continuation, ITM only strictly above the
  tolerance; and the one-feature monomial basis order.
"""
import ctypes as C
import json
import os
from decimal import Decimal

import numpy as np
import pytest

import helpers as H

CASES = json.load(open(os.path.join(H.GOLDEN, "early_exercise_cases.json")))


def _lib():
    lib = H.oracle()
    dp, u32p = C.POINTER(C.c_double), C.POINTER(C.c_uint32)
    lib.oracle_lsm_scaling.argtypes = [dp, C.c_uint64, dp]
    lib.oracle_lsm_scaling.restype = C.c_int
    lib.oracle_lsm_cpqr.argtypes = [dp, C.c_uint64, C.c_uint32, dp, C.c_double, C.c_double, u32p, u32p, dp, dp]
    lib.oracle_lsm_cpqr.restype = C.c_int
    return lib


def close(got: float, want: str, ulps: float = 2.0) -> bool:
    w = float(Decimal(want))
    return abs(got - w) <= ulps * np.spacing(max(abs(w), 1e-300))


@pytest.mark.parametrize("case", CASES["scaling_cases"], ids=lambda c: c["id"])
def test_feature_scaling(case):
    values = np.array([float(Decimal(v)) for v in case["values"]])
    out = np.zeros(4)
    inactive = _lib().oracle_lsm_scaling(H.dptr(values), len(values), H.dptr(out))
    e = case["expected"]
    assert bool(inactive) == e["inactive"]
    assert close(out[0], e["mean"]) or abs(out[0] - float(Decimal(e["mean"]))) < 1e-15
    assert close(out[1], e["population_variance"])
    assert close(out[2], e["scale"])
    assert out[3] == float(Decimal(e["zero_scale_threshold"]))


@pytest.mark.parametrize("case", CASES["qr_cases"], ids=lambda c: c["id"])
def test_cpqr(case):
    m = np.array([[float(Decimal(v)) for v in row] for row in case["matrix"]])
    y = np.array([float(Decimal(v)) for v in case["target"]])
    rows, cols = m.shape
    pivot = np.zeros(cols, dtype=np.uint32)
    coef = np.zeros(cols)
    rank = C.c_uint32()
    rss = C.c_double()
    flat = np.ascontiguousarray(m.ravel())
    rc = _lib().oracle_lsm_cpqr(H.dptr(flat), rows, cols, H.dptr(y), float(Decimal(case["abs_rank_tol"])),
                                float(Decimal(case["rel_rank_tol"])), H.uptr(pivot), C.byref(rank), H.dptr(coef),
                                C.byref(rss))
    assert rc == 0
    e = case["expected"]
    assert list(pivot) == e["pivot_order"]
    assert rank.value == e["rank"]
    for got, want in zip(coef, e["coefficients"]):
        assert abs(got - float(Decimal(want))) <= 4e-15 * max(1.0, abs(float(Decimal(want))))
    assert abs(rss.value - float(Decimal(e["residual_sum_squares"]))) <= 1e-14


@pytest.mark.parametrize("case", CASES["decision_cases"], ids=lambda c: c["id"])
def test_decision_rules(case):
    # ExerciseDecisionModel::should_exercise and the ITM filter: strict comparisons.
    imm, other = float(Decimal(case["immediate_value"])), float(Decimal(case["comparison_value"]))
    assert (imm > other) == case["expected"]


def test_one_feature_basis_order():
    case = next(c for c in CASES["basis_cases"] if c["feature_count"] == 1)
    # the engine's basis for one spot feature: monomials of increasing degree
    assert case["expected_exponents"] == [[d] for d in range(case["max_degree"] + 1)]

"""Shared test helpers: paths, the oracle loader and descriptor utilities.

The oracle (oracle/_build/liboracle.so) is the reference restatement; the engine under test is
loaded through rust_pricing_b200._native.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rust-pricing-library_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

from rust_pricing_b200 import _abi as A  # noqa: E402

ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")

_oracle = None


def oracle():
    """Load (building if needed) the CPU oracle library."""
    global _oracle
    if _oracle is not None:
        return _oracle
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    lib = C.CDLL(ORACLE_SO)
    u32, u64, dbl = C.c_uint32, C.c_uint64, C.c_double
    lib.oracle_philox_block.argtypes = [u64, C.POINTER(u32), C.POINTER(u32)]
    lib.oracle_philox_word.argtypes = [u64, u64, u32, u32]
    lib.oracle_philox_word.restype = u32
    lib.oracle_open_unit_interval.argtypes = [u32]
    lib.oracle_open_unit_interval.restype = dbl
    lib.oracle_inverse_normal.argtypes = [dbl]
    lib.oracle_inverse_normal.restype = dbl
    lib.oracle_philox_normal.argtypes = [u64, u64, u32, u32]
    lib.oracle_philox_normal.restype = dbl
    lib.oracle_sobol_word.argtypes = [C.POINTER(u32), u32]
    lib.oracle_sobol_word.restype = u32
    lib.oracle_scramble.argtypes = [u64, u32, u32, C.POINTER(u32), C.POINTER(u32)]
    lib.oracle_rqmc_word.argtypes = [C.POINTER(u32), u64, u32, u32, u32]
    lib.oracle_rqmc_word.restype = u32
    dp = C.POINTER(dbl)
    lib.oracle_bridge_compile.argtypes = [dp, u32, C.POINTER(u32), C.POINTER(u32), dp, dp, dp]
    lib.oracle_bridge_compile.restype = C.c_int
    lib.oracle_bridge_apply.argtypes = [dp, u32, dp, dp]
    lib.oracle_bridge_reverse.argtypes = [dp, u32, dp, dp]
    lib.oracle_evaluate.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(A.Result), C.c_int]
    lib.oracle_evaluate.restype = C.c_int
    lib.oracle_unit_shocks.argtypes = [C.POINTER(A.PlanDesc), u32, u64, dp]
    lib.oracle_unit_values.argtypes = [C.POINTER(A.PlanDesc), u32, u64, dp]
    lib.oracle_time_grid.argtypes = [C.POINTER(A.PlanDesc), dp, u32, C.POINTER(u32)]
    lib.oracle_last_error.restype = C.c_char_p
    lib.oracle_ssvi_grid.argtypes = [dp, dp, u32, dbl, dbl, dbl, dbl, dp, u32, dp, u32, dbl, dbl, dp]
    lib.oracle_ssvi_grid.restype = C.c_int
    lib.oracle_surface_grid.argtypes = [C.POINTER(A.SurfaceDesc), dp, u32, dp, u32, dbl, dbl, dp]
    lib.oracle_surface_grid.restype = C.c_int
    lib.oracle_surface_total_variance.argtypes = [C.POINTER(A.SurfaceDesc), dbl, dbl, dp]
    lib.oracle_surface_total_variance.restype = C.c_int
    lib.oracle_vega_kt_project.argtypes = [dp, u32, dp, u32, dp, u64, C.POINTER(A.VegaKtBasis),
                                           C.POINTER(A.VegaKtProjection)]
    lib.oracle_vega_kt_project.restype = C.c_int
    lib.oracle_piecewise_sinh_nodes.argtypes = [dbl, dbl, u32, u32, dbl, dbl, dp]
    lib.oracle_piecewise_sinh_nodes.restype = C.c_int
    lib.oracle_smoothing.argtypes = [dbl, dbl, dp]
    lib.oracle_smooth_extrema.argtypes = [dbl, dbl, dbl, dp]
    lib.oracle_exact_bridge.argtypes = [C.c_int, dbl, dbl, dbl, dbl, dp]
    lib.oracle_exact_bridge.restype = C.c_int
    lib.oracle_smoothed_bridge.argtypes = [C.c_int, dbl, dbl, dbl, dbl, dbl, dp]
    lib.oracle_smoothed_bridge.restype = C.c_int
    lib.oracle_barrier_path.argtypes = [C.c_int, dbl, dbl, dp, dp, dp, u32, dp, dp]
    lib.oracle_barrier_path.restype = C.c_int
    lib.oracle_interval_adjoint.argtypes = [C.c_int, dbl, dbl, dbl, dbl, dbl, dbl, dbl, dbl, dp]
    lib.oracle_interval_adjoint.restype = C.c_int
    lib.oracle_lsm_price.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(A.LsmDesc), C.POINTER(A.LsmResult),
                                     C.c_int]
    lib.oracle_lsm_price.restype = C.c_int
    lib.oracle_lsm_last_error.restype = C.c_char_p
    lib.oracle_lsm_spots.argtypes = [C.POINTER(A.PlanDesc), u32, C.c_int, C.POINTER(dbl), u64]
    lib.oracle_lsm_spots.restype = C.c_int64
    lib.oracle_lsm_dual.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(A.LsmDesc), C.POINTER(A.DualDesc),
                                    C.POINTER(A.DualResult), C.c_int]
    lib.oracle_lsm_dual.restype = C.c_int
    lib.oracle_lsm_fit.argtypes = [C.POINTER(dbl), C.POINTER(dbl), C.POINTER(dbl), u64,
                                   C.POINTER(A.LsmDesc), C.POINTER(A.LsmDateModel)]
    lib.oracle_lsm_fit.restype = C.c_int
    lib.oracle_multi_asset_price.argtypes = [C.POINTER(A.MultiAssetDesc), C.POINTER(A.MultiAssetResult), C.c_int]
    lib.oracle_multi_asset_price.restype = C.c_int
    lib.oracle_bump_evaluate.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(A.BumpRequest), C.c_uint32,
                                         C.POINTER(A.BumpEstimate), C.POINTER(A.BumpReport), C.c_int]
    lib.oracle_bump_evaluate.restype = C.c_int
    _oracle = lib
    return lib


def oracle_evaluate(spec, threads: int | None = None):
    """Run the oracle on a PlanSpec; returns the ResultBuffers."""
    lib = oracle()
    nodes = spec.grid_value_count() * len(spec.products) if spec.request_local_vega_nodes else 0
    buf = A.ResultBuffers(len(spec.products), nodes, spec.scramble_count if spec.engine == A.ENGINE_RQMC else 0)
    desc = spec.desc()
    rc = lib.oracle_evaluate(C.byref(desc), C.byref(buf.result), threads or os.cpu_count() or 1)
    if rc != 0:
        raise RuntimeError(f"oracle status {A.STATUS_NAMES.get(rc, rc)}: "
                           f"{lib.oracle_last_error().decode()} error={buf.result.error.code}")
    return buf


def oracle_lsm(spec, lsm, stopping: bool = False, threads: int | None = None):
    """Run the oracle's early-exercise evaluation; returns the LsmBuffers."""
    lib = oracle()
    paths = spec.sampling_units * (spec.scramble_count if spec.engine == A.ENGINE_RQMC else 1)
    paths *= 2 if spec.antithetic else 1
    nodes = spec.grid_value_count() if spec.request_local_vega_nodes else 0
    buf = A.LsmBuffers(len(spec.observation_times), paths if stopping else 0, nodes)
    desc, ldesc = spec.desc(), lsm.desc()
    rc = lib.oracle_lsm_price(C.byref(desc), C.byref(ldesc), C.byref(buf.result),
                              threads or os.cpu_count() or 1)
    if rc != 0:
        raise RuntimeError(f"oracle status {A.STATUS_NAMES.get(rc, rc)}: "
                           f"{lib.oracle_lsm_last_error().decode()} {lib.oracle_last_error().decode()}")
    return buf


def oracle_lsm_dual(spec, lsm, n2: int, n3: int, seed: int, threads: int | None = None):
    """Run the oracle's Andersen--Broadie dual; returns the DualResult."""
    lib = oracle()
    out = A.DualResult()
    desc, ldesc = spec.desc(), lsm.desc()
    dual = A.DualDesc(n2, n3, seed & 0xFFFFFFFFFFFFFFFF)
    rc = lib.oracle_lsm_dual(C.byref(desc), C.byref(ldesc), C.byref(dual), C.byref(out),
                             threads or os.cpu_count() or 1)
    if rc != 0:
        raise RuntimeError(f"oracle status {A.STATUS_NAMES.get(rc, rc)}: {lib.oracle_lsm_last_error().decode()}")
    return out


def dptr(array):
    return array.ctypes.data_as(C.POINTER(C.c_double))


def uptr(array):
    return array.ctypes.data_as(C.POINTER(C.c_uint32))


def oracle_multi(spec, threads: int | None = None):
    """Run the oracle's multi-asset evaluation; returns the MultiAssetResult."""
    out = A.MultiAssetResult()
    desc = spec.desc()
    rc = oracle().oracle_multi_asset_price(C.byref(desc), C.byref(out), threads or os.cpu_count() or 1)
    if rc != 0:
        raise RuntimeError(f"oracle multi-asset status {A.STATUS_NAMES.get(rc, rc)}")
    return out


def bump_requests(requests):
    """[(measure, size, relative)] -> a ctypes array of mcg_bump_request."""
    return (A.BumpRequest * len(requests))(*[A.BumpRequest(m, int(rel), size) for m, size, rel in requests])


def oracle_bump(spec, requests, threads: int | None = None):
    """The oracle's bump-and-revalue: (estimates, report)."""
    req = bump_requests(requests)
    est = (A.BumpEstimate * len(requests))()
    rep = A.BumpReport()
    desc = spec.desc()
    rc = oracle().oracle_bump_evaluate(C.byref(desc), req, len(requests), est, C.byref(rep),
                                       threads or os.cpu_count() or 1)
    if rc != 0:
        raise RuntimeError(f"oracle bump status {A.STATUS_NAMES.get(rc, rc)}")
    return list(est), rep

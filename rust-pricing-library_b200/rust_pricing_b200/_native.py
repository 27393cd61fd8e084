"""Loader of the engine library (libmcg.so, include/mcg.h).

The engine has no CPU fallback: if the library is missing or cannot be loaded,
every entry point raises.  `build()` (rust-pricing-library_b200/build.py)
compiles it in place for sm_100a.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(HERE, "libmcg.so")

EXPORTS = (
    "mcg_abi_version", "mcg_last_error", "mcg_plan_create", "mcg_plan_evaluate", "mcg_price",
    "mcg_plan_destroy", "mcg_plan_shape", "mcg_philox_normals", "mcg_rqmc_words",
    "mcg_ssvi_local_variance_grid", "mcg_measure_fp64_peak", "mcg_price_european_noalloc",
    "mcg_lsm_price", "mcg_mlp_forward", "mcg_mlp_gradient", "mcg_book_create", "mcg_book_evaluate",
    "mcg_book_destroy", "mcg_surface_local_variance_grid", "mcg_surface_total_variance", "mcg_vega_kt_project",
    "mcg_lsm_dual", "mcg_multi_asset_price", "mcg_bump_evaluate",
)

_lib = None


class EngineError(RuntimeError):
    """An mcg_status other than MCG_OK, with the library's message."""

    def __init__(self, status: int, message: str, error: A.ErrorRecord | None = None):
        self.status = status
        self.name = A.STATUS_NAMES.get(status, str(status))
        self.error = error
        detail = ""
        if error is not None and error.code:
            detail = (f" (sampling unit {error.sampling_unit}, step {error.step}, "
                      f"value bits 0x{error.value_bits:016x})")
        super().__init__(f"{self.name}: {message}{detail}")


def library() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY_PATH):
        raise EngineError(14, f"engine library {LIBRARY_PATH} is not built; run build()")
    lib = C.CDLL(LIBRARY_PATH)
    u32, u64, dbl, vp = C.c_uint32, C.c_uint64, C.c_double, C.c_void_p
    lib.mcg_abi_version.restype = u32
    lib.mcg_last_error.restype = C.c_char_p
    lib.mcg_plan_create.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(vp)]
    lib.mcg_plan_create.restype = C.c_int
    lib.mcg_plan_evaluate.argtypes = [vp, vp, C.POINTER(A.Result)]
    lib.mcg_plan_evaluate.restype = C.c_int
    lib.mcg_price.argtypes = [C.POINTER(A.PlanDesc), vp, C.POINTER(A.Result)]
    lib.mcg_price.restype = C.c_int
    lib.mcg_plan_destroy.argtypes = [vp]
    lib.mcg_plan_shape.argtypes = [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]
    lib.mcg_plan_shape.restype = C.c_int
    lib.mcg_philox_normals.argtypes = [u64, u64, u64, u32, u32, C.POINTER(dbl)]
    lib.mcg_philox_normals.restype = C.c_int
    lib.mcg_rqmc_words.argtypes = [C.POINTER(u32), u32, u64, u32, u64, u64, C.POINTER(u32)]
    lib.mcg_rqmc_words.restype = C.c_int
    dp = C.POINTER(dbl)
    lib.mcg_ssvi_local_variance_grid.argtypes = [dp, dp, u32, dbl, dbl, dbl, dbl, dp, u32, dp, u32,
                                                 dbl, dbl, dp, C.POINTER(u32)]
    lib.mcg_ssvi_local_variance_grid.restype = C.c_int
    lib.mcg_surface_local_variance_grid.argtypes = [C.POINTER(A.SurfaceDesc), dp, u32, dp, u32, dbl, dbl, dp,
                                                    C.POINTER(u32)]
    lib.mcg_surface_local_variance_grid.restype = C.c_int
    lib.mcg_surface_total_variance.argtypes = [C.POINTER(A.SurfaceDesc), dp, dp, u32, dp]
    lib.mcg_surface_total_variance.restype = C.c_int
    lib.mcg_vega_kt_project.argtypes = [dp, u32, dp, u32, dp, u64, C.POINTER(A.VegaKtBasis),
                                        C.POINTER(A.VegaKtProjection)]
    lib.mcg_vega_kt_project.restype = C.c_int
    lib.mcg_price_european_noalloc.argtypes = [C.POINTER(A.PlanDesc), vp, C.POINTER(A.Result)]
    lib.mcg_price_european_noalloc.restype = C.c_int
    lib.mcg_measure_fp64_peak.argtypes = [vp, C.POINTER(dbl)]
    lib.mcg_measure_fp64_peak.restype = C.c_int
    lib.mcg_lsm_price.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(A.LsmDesc), vp, C.POINTER(A.LsmResult)]
    lib.mcg_lsm_price.restype = C.c_int
    lib.mcg_lsm_dual.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(A.LsmDesc), C.POINTER(A.DualDesc), vp,
                                 C.POINTER(A.DualResult)]
    lib.mcg_lsm_dual.restype = C.c_int
    fp = C.POINTER(C.c_float)
    lib.mcg_mlp_forward.argtypes = [fp, fp, u32, fp]
    lib.mcg_mlp_forward.restype = C.c_int
    lib.mcg_mlp_gradient.argtypes = [fp, fp, fp, C.POINTER(C.c_uint8), u32, fp, fp]
    lib.mcg_mlp_gradient.restype = C.c_int
    lib.mcg_book_create.argtypes = [C.POINTER(A.PlanDesc), u32, C.POINTER(A.BookOptions), C.POINTER(vp)]
    lib.mcg_book_create.restype = C.c_int
    lib.mcg_book_evaluate.argtypes = [vp, vp, C.POINTER(A.Estimate), C.POINTER(A.BookReport)]
    lib.mcg_book_evaluate.restype = C.c_int
    lib.mcg_book_destroy.argtypes = [vp]
    lib.mcg_multi_asset_price.argtypes = [C.POINTER(A.MultiAssetDesc), vp, C.POINTER(A.MultiAssetResult)]
    lib.mcg_multi_asset_price.restype = C.c_int
    lib.mcg_bump_evaluate.argtypes = [C.POINTER(A.PlanDesc), C.POINTER(A.BumpRequest), u32, vp,
                                      C.POINTER(A.BumpEstimate), C.POINTER(A.BumpReport)]
    lib.mcg_bump_evaluate.restype = C.c_int
    if lib.mcg_abi_version() != A.ABI_VERSION:
        raise EngineError(1, "engine library ABI version mismatch")
    _lib = lib
    return lib


def check(status: int, error: A.ErrorRecord | None = None) -> None:
    if status != 0:
        raise EngineError(status, library().mcg_last_error().decode(), error)


def surface_grid(surface, time_nodes, log_moneyness_nodes, floor: float = 1e-8, cap: float = 4.0):
    """mcg_surface_local_variance_grid: (values[nt, nx], repairs)."""
    import numpy as np
    tn = np.ascontiguousarray(time_nodes, dtype=np.float64)
    xn = np.ascontiguousarray(log_moneyness_nodes, dtype=np.float64)
    out = np.zeros(len(tn) * len(xn))
    rep = C.c_uint32()
    dp = C.POINTER(C.c_double)
    d = surface.desc()
    check(library().mcg_surface_local_variance_grid(C.byref(d), tn.ctypes.data_as(dp), len(tn),
                                                     xn.ctypes.data_as(dp), len(xn), floor, cap,
                                                     out.ctypes.data_as(dp), C.byref(rep)))
    return out.reshape(len(tn), len(xn)), rep.value


def surface_total_variance(surface, times, log_moneyness):
    """mcg_surface_total_variance: (n, 4) array of w, w_k, w_kk, w_t."""
    import numpy as np
    t = np.ascontiguousarray(times, dtype=np.float64)
    k = np.ascontiguousarray(log_moneyness, dtype=np.float64)
    out = np.zeros(4 * len(t))
    dp = C.POINTER(C.c_double)
    d = surface.desc()
    check(library().mcg_surface_total_variance(C.byref(d), t.ctypes.data_as(dp), k.ctypes.data_as(dp), len(t),
                                                out.ctypes.data_as(dp)))
    return out.reshape(len(t), 4)


class VegaKtBasisSpec:
    """A reporting-IV basis (maturities x log-moneyness implied volatilities),
    the forwards at its maturities and the relative density threshold."""

    def __init__(self, maturities, log_moneyness, implied_volatilities, forwards, threshold: float = 1e-8):
        import numpy as np
        self.arrays = [np.ascontiguousarray(a, dtype=np.float64).ravel()
                       for a in (maturities, log_moneyness, implied_volatilities, forwards)]
        self.threshold = threshold

    def desc(self) -> A.VegaKtBasis:
        dp = C.POINTER(C.c_double)
        m, x, iv, f = self.arrays
        return A.VegaKtBasis(m.ctypes.data_as(dp), len(m), x.ctypes.data_as(dp), len(x), iv.ctypes.data_as(dp),
                             f.ctypes.data_as(dp), self.threshold)

    def buckets(self) -> int:
        return len(self.arrays[0]) * len(self.arrays[1])


def vega_kt_project(time_nodes, log_moneyness_nodes, node_sensitivities, evaluated_paths: int,
                    basis: VegaKtBasisSpec):
    """mcg_vega_kt_project (host code): (projection record, raw buckets)."""
    import numpy as np
    tn = np.ascontiguousarray(time_nodes, dtype=np.float64)
    xn = np.ascontiguousarray(log_moneyness_nodes, dtype=np.float64)
    nodes = np.ascontiguousarray(node_sensitivities, dtype=np.float64).ravel()
    out = A.VegaKtProjection()
    buckets = np.zeros(basis.buckets())
    dp = C.POINTER(C.c_double)
    out.bucket_capacity = len(buckets)
    out.raw_buckets = buckets.ctypes.data_as(dp)
    b = basis.desc()
    check(library().mcg_vega_kt_project(tn.ctypes.data_as(dp), len(tn), xn.ctypes.data_as(dp), len(xn),
                                         nodes.ctypes.data_as(dp), evaluated_paths, C.byref(b), C.byref(out)))
    return out, buckets


def lsm_price(spec, lsm, stopping: bool = False, stream: int = 0) -> A.LsmBuffers:
    """mcg_lsm_price: train and value an early-exercise policy on the GPU."""
    paths = spec.sampling_units * (spec.scramble_count if spec.engine == A.ENGINE_RQMC else 1)
    paths *= 2 if spec.antithetic else 1
    nodes = spec.grid_value_count() if spec.request_local_vega_nodes else 0
    buf = A.LsmBuffers(len(spec.observation_times), paths if stopping else 0, nodes)
    desc, ldesc = spec.desc(), lsm.desc()
    status = library().mcg_lsm_price(C.byref(desc), C.byref(ldesc), C.c_void_p(stream), C.byref(buf.result))
    check(status, buf.result.error)
    return buf


def lsm_dual(spec, lsm, continuation_inner_paths: int, exercise_inner_paths: int, inner_seed: int,
             stream: int = 0) -> A.DualResult:
    """mcg_lsm_dual: Andersen--Broadie lower and upper bounds of an
    early-exercise price around the fitted LSM policy, on the GPU."""
    out = A.DualResult()
    desc, ldesc = spec.desc(), lsm.desc()
    dual = A.DualDesc(continuation_inner_paths, exercise_inner_paths, inner_seed & 0xFFFFFFFFFFFFFFFF)
    status = library().mcg_lsm_dual(C.byref(desc), C.byref(ldesc), C.byref(dual), C.c_void_p(stream),
                                    C.byref(out))
    check(status, out.error)
    return out


def multi_asset_price(spec, stream: int = 0) -> A.MultiAssetResult:
    """mcg_multi_asset_price: a basket or worst-of option on correlated
    Black--Scholes / local-volatility assets, on the GPU."""
    out = A.MultiAssetResult()
    desc = spec.desc()
    check(library().mcg_multi_asset_price(C.byref(desc), C.c_void_p(stream), C.byref(out)), out.error)
    return out


def mlp_forward(params, x):
    """mcg_mlp_forward on host arrays: params (MLP_PARAMS,), x (n, 2) -> (n,)."""
    import numpy as np
    p = np.ascontiguousarray(params, dtype=np.float32)
    xs = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(len(xs), dtype=np.float32)
    fp = C.POINTER(C.c_float)
    check(library().mcg_mlp_forward(p.ctypes.data_as(fp), xs.ctypes.data_as(fp), len(xs), out.ctypes.data_as(fp)))
    return out


def mlp_gradient(params, x, y, mask):
    """mcg_mlp_gradient: gradient of sum mask (f(x) - y)^2 and that sum."""
    import numpy as np
    p = np.ascontiguousarray(params, dtype=np.float32)
    xs = np.ascontiguousarray(x, dtype=np.float32)
    ys = np.ascontiguousarray(y, dtype=np.float32)
    ms = np.ascontiguousarray(mask, dtype=np.uint8)
    grad = np.zeros(A.MLP_PARAMS, dtype=np.float32)
    loss = C.c_float()
    fp = C.POINTER(C.c_float)
    check(library().mcg_mlp_gradient(p.ctypes.data_as(fp), xs.ctypes.data_as(fp), ys.ctypes.data_as(fp),
                                      ms.ctypes.data_as(C.POINTER(C.c_uint8)), len(xs), grad.ctypes.data_as(fp),
                                      C.byref(loss)))
    return grad, loss.value


class Plan:
    """An mcg_plan handle: compile once, evaluate many times."""

    def __init__(self, spec):
        self.spec = spec
        self.desc = spec.desc()
        self.handle = C.c_void_p()
        check(library().mcg_plan_create(C.byref(self.desc), C.byref(self.handle)))
        self.nodes = spec.grid_value_count() * len(spec.products) if spec.request_local_vega_nodes else 0

    def evaluate(self, stream: int = 0) -> A.ResultBuffers:
        scrambles = self.spec.scramble_count if self.spec.engine == A.ENGINE_RQMC else 0
        buf = A.ResultBuffers(len(self.spec.products), self.nodes, scrambles)
        status = library().mcg_plan_evaluate(self.handle, C.c_void_p(stream), C.byref(buf.result))
        check(status, buf.result.error)
        return buf

    def shape(self):
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(library().mcg_plan_shape(self.handle, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def close(self) -> None:
        if self.handle:
            library().mcg_plan_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Book:
    """An mcg_book handle: a book of single-product plans priced in one launch."""

    def __init__(self, specs, autotune: bool = True, tiles_per_item: int = 0, ctas_per_sm: int = 0,
                 use_graph: bool = True):
        self.specs = list(specs)
        descs = (A.PlanDesc * len(self.specs))()
        for i, sp in enumerate(self.specs):
            descs[i] = sp.desc()  # each spec keeps its arrays alive
        self._descs = descs
        opts = A.BookOptions(int(autotune), tiles_per_item, ctas_per_sm, int(use_graph))
        self.handle = C.c_void_p()
        check(library().mcg_book_create(descs, len(self.specs), C.byref(opts), C.byref(self.handle)))

    def evaluate(self, stream: int = 0):
        prices = (A.Estimate * len(self.specs))()
        report = A.BookReport()
        status = library().mcg_book_evaluate(self.handle, C.c_void_p(stream), prices, C.byref(report))
        check(status, report.error)
        return prices, report

    def close(self) -> None:
        if self.handle:
            library().mcg_book_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def bump_evaluate(spec, requests, stream: int = 0):
    """mcg_bump_evaluate: bump-and-revalue of a price-only plan on common random
    numbers, every scenario side in one launch.  `requests` are
    (measure, size, relative) triples; returns (estimates, report)."""
    n = len(requests)
    req = (A.BumpRequest * n)(*[A.BumpRequest(m, int(rel), size) for m, size, rel in requests])
    est = (A.BumpEstimate * n)()
    rep = A.BumpReport()
    desc = spec.desc()
    check(library().mcg_bump_evaluate(C.byref(desc), req, n, C.c_void_p(stream), est, C.byref(rep)), rep.error)
    return list(est), rep

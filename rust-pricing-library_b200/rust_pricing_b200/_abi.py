"""ctypes mirror of include/mcg.h (the engine's C ABI).

The structures here must match the header field for field; the layout test in
tests/test_abi.py compares their sizes with the C compiler's.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 3
PATHWISE_COMPONENTS = 18

PRICE, DELTA, VEGA, GAMMA = 0, 1, 2, 3
BUMP_DELTA, DELTA_DIFFERENCE, BUMP_VEGA, VEGA_DIFFERENCE = 4, 5, 6, 7
BUMP_GAMMA, GAMMA_DIFFERENCE = 8, 9
BARRIER_ENDPOINT_HIT, BARRIER_DIVIDEND_JUMP_HIT, BARRIER_BRIDGE_HIT_WEIGHT = 10, 11, 12
BARRIER_INTERVAL_COUNT, BARRIER_FINITE_CORRECTION_COUNT = 13, 14
BARRIER_ZERO_VARIANCE_COUNT, BARRIER_SURVIVAL_UNDERFLOW_COUNT = 15, 16
BARRIER_CERTAIN_SURVIVAL_COUNT = 17

MODEL_BLACK_SCHOLES, MODEL_LOCAL_VOLATILITY = 0, 1
ENGINE_PSEUDO, ENGINE_RQMC = 0, 1
PRECISION_F64, PRECISION_F32_BULK = 0, 1
(PRODUCT_EUROPEAN, PRODUCT_DIGITAL, PRODUCT_ASIAN, PRODUCT_LOOKBACK,
 PRODUCT_DISCRETE_BARRIER, PRODUCT_CONTINUOUS_BARRIER, PRODUCT_AMERICAN) = range(7)
CALL, PUT = 0, 1
BARRIER_UP, BARRIER_DOWN = 0, 1
KNOCK_OUT, KNOCK_IN = 0, 1
DIGITAL_CASH, DIGITAL_ASSET = 0, 1

STATUS_NAMES = {
    0: "ok", 1: "invalid_argument", 2: "unsupported", 3: "cuda", 4: "allocation",
    5: "insufficient_sampling_units", 6: "non_finite_state", 7: "invalid_surface_query",
    8: "sobol_dimension", 9: "brownian_bridge", 10: "barrier_bridge", 11: "market",
    12: "lsm", 13: "timeout", 14: "not_built",
}

_dp = C.POINTER(C.c_double)
_up = C.POINTER(C.c_uint32)


class Dividends(C.Structure):
    _fields_ = [("count", C.c_uint32), ("ex_times", _dp), ("fixed_cash", _dp), ("proportional", _dp)]


class Curve(C.Structure):
    _fields_ = [("pillar_count", C.c_uint32), ("times", _dp), ("discount_factors", _dp)]


SURFACE_SSVI_POWER_LAW, SURFACE_SSVI_HESTON_LIKE, SURFACE_ESSVI = 0, 1, 2


class SurfaceDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("theta_times", _dp), ("theta_values", _dp), ("theta_count", C.c_uint32),
        ("terminal_theta_slope", C.c_double), ("rho", C.c_double), ("eta", C.c_double), ("gamma", C.c_double),
        ("lambda_", C.c_double), ("slice_times", _dp), ("slice_thetas", _dp), ("slice_psis", _dp),
        ("slice_rho_psis", _dp), ("slice_count", C.c_uint32),
    ]


class VegaKtBasis(C.Structure):
    _fields_ = [("maturity_nodes", _dp), ("maturity_count", C.c_uint32), ("log_moneyness_nodes", _dp),
                ("log_moneyness_count", C.c_uint32), ("implied_volatilities", _dp), ("forwards", _dp),
                ("relative_density_threshold", C.c_double)]


class VegaKtProjection(C.Structure):
    _fields_ = [("bucket_capacity", C.c_uint32), ("raw_buckets", _dp), ("scalar_vega", C.c_double),
                ("signed_residual", C.c_double), ("density_excluded", C.c_double), ("pre_projection", C.c_double),
                ("initial_time", C.c_double),
                ("left_edge_sensitivity", C.c_double), ("right_edge_sensitivity", C.c_double),
                ("left_edge_count", C.c_uint64), ("right_edge_count", C.c_uint64)]


class LocalVarianceGrid(C.Structure):
    _fields_ = [
        ("time_count", C.c_uint32), ("log_moneyness_count", C.c_uint32),
        ("time_nodes", _dp), ("log_moneyness_nodes", _dp), ("values", _dp),
        ("floor", C.c_double), ("cap", C.c_double),
    ]


class ProductDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("side", C.c_int32), ("strike", C.c_double), ("notional", C.c_double),
        ("digital_payout", C.c_int32), ("payout", C.c_double),
        ("barrier_direction", C.c_int32), ("barrier_style", C.c_int32), ("has_rebate", C.c_int32),
        ("barrier", C.c_double), ("rebate", C.c_double),
        ("observation_weights", _dp),
        ("has_initial_state", C.c_int32), ("initial_state", C.c_double),
    ]


class PlanDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32), ("model", C.c_int32), ("engine", C.c_int32),
        ("precision", C.c_int32),
        ("master_seed", C.c_uint64), ("sampling_units", C.c_uint64),
        ("scramble_count", C.c_uint32), ("scramble_begin", C.c_uint32), ("antithetic", C.c_int32),
        ("brownian_bridge", C.c_int32),
        ("reduction_block_size", C.c_uint64),
        ("sobol_dimension_count", C.c_uint32), ("sobol_directions", _up),
        ("spot", C.c_double), ("discount_curve", Curve), ("dividend_curve", Curve),
        ("volatility", C.c_double), ("local_variance", LocalVarianceGrid),
        ("observation_count", C.c_uint32), ("observation_times", _dp), ("payment_time", C.c_double),
        ("product_count", C.c_uint32), ("products", C.POINTER(ProductDesc)),
        ("request_delta", C.c_int32), ("request_gamma", C.c_int32), ("request_vega", C.c_int32),
        ("request_local_vega_nodes", C.c_int32), ("gamma_bump_relative", C.c_int32),
        ("gamma_bump", C.c_double), ("smoothing_half_width", C.c_double),
        ("checkpoint_interval", C.c_uint32),
        ("discrete_dividends", Dividends),
    ]


class Statistics(C.Structure):
    _fields_ = [("sum", C.c_double), ("correction", C.c_double), ("count", C.c_uint64),
                ("mean", C.c_double), ("second_moment", C.c_double)]

    def total(self) -> float:
        return self.sum + self.correction


class Estimate(C.Structure):
    _fields_ = [("value", C.c_double), ("standard_error", C.c_double),
                ("confidence_lower", C.c_double), ("confidence_upper", C.c_double),
                ("effective_sampling_units", C.c_uint64)]


class ProductResult(C.Structure):
    _fields_ = [
        ("components", Statistics * PATHWISE_COMPONENTS),
        ("price", Estimate), ("delta", Estimate), ("gamma", Estimate), ("vega", Estimate),
        ("bump_delta", Estimate), ("bump_gamma", Estimate), ("bump_vega", Estimate),
        ("sampling_variance", C.c_double), ("estimator_variance", C.c_double),
        ("adjoint_components", Statistics * 2), ("adjoint_delta", Estimate), ("adjoint_gamma", Estimate),
    ]


class ErrorRecord(C.Structure):
    _fields_ = [("code", C.c_int32), ("step", C.c_uint32), ("sampling_unit", C.c_uint64),
                ("value_bits", C.c_uint64)]


class Result(C.Structure):
    _fields_ = [
        ("product_capacity", C.c_uint32), ("products", C.POINTER(ProductResult)),
        ("node_capacity", C.c_uint32), ("local_vega_nodes", C.POINTER(Statistics)),
        ("local_vega_node_estimates", C.POINTER(Estimate)),
        ("independent_sampling_units", C.c_uint64), ("evaluated_paths", C.c_uint64),
        ("time_steps", C.c_uint32), ("effective_dimension", C.c_uint32),
        ("reduction_records", C.c_uint32), ("kernel_launches", C.c_uint32),
        ("device_ms", C.c_float), ("path_kernel_ms", C.c_float), ("error", ErrorRecord),
        ("replicate_capacity", C.c_uint32), ("replicate_means", _dp),
    ]


# ---- correlated multi-asset paths ----
MAX_ASSETS = 8
MULTI_BASKET, MULTI_WORST_OF = 0, 1


class AssetDesc(C.Structure):
    _fields_ = [
        ("model", C.c_int32), ("spot", C.c_double), ("dividend_curve", Curve), ("volatility", C.c_double),
        ("local_variance", LocalVarianceGrid),
    ]


class MultiAssetDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32), ("asset_count", C.c_uint32), ("assets", C.POINTER(AssetDesc)),
        ("discount_curve", Curve), ("correlation_count", C.c_uint32), ("correlation_times", _dp),
        ("correlations", _dp), ("maximum_step", C.c_double), ("expiry", C.c_double), ("payment_time", C.c_double),
        ("engine", C.c_int32), ("master_seed", C.c_uint64), ("sampling_units", C.c_uint64),
        ("scramble_count", C.c_uint32), ("antithetic", C.c_int32), ("brownian_bridge", C.c_int32),
        ("reduction_block_size", C.c_uint64), ("sobol_dimension_count", C.c_uint32), ("sobol_directions", _up),
        ("product", C.c_int32), ("side", C.c_int32), ("strike", C.c_double), ("notional", C.c_double),
        ("weights", _dp), ("scales", _dp), ("smoothing_half_width", C.c_double),
    ]


class MultiAssetResult(C.Structure):
    _fields_ = [
        ("price_statistics", Statistics), ("price", Estimate), ("sampling_variance", C.c_double),
        ("evaluated_paths", C.c_uint64), ("independent_sampling_units", C.c_uint64),
        ("time_steps", C.c_uint32), ("dimension", C.c_uint32), ("kernel_launches", C.c_uint32),
        ("device_ms", C.c_float), ("error", ErrorRecord),
    ]


# ---- bump-and-revalue on common random numbers ----
BUMP_SPOT_DELTA, BUMP_SPOT_GAMMA, BUMP_VOLATILITY_VEGA = 0, 1, 2


class BumpRequest(C.Structure):
    _fields_ = [("measure", C.c_int32), ("relative", C.c_int32), ("size", C.c_double)]


class BumpEstimate(C.Structure):
    _fields_ = [
        ("measure", C.c_int32), ("scenario", C.c_uint32), ("amount", C.c_double), ("value", C.c_double),
        ("standard_error", C.c_double), ("units", C.c_uint64), ("up_price", C.c_double),
        ("down_price", C.c_double),
    ]


class BumpReport(C.Structure):
    _fields_ = [
        ("scenarios", C.c_uint32), ("sides", C.c_uint32), ("evaluations", C.c_uint64),
        ("base_price", Estimate), ("path_steps", C.c_uint64), ("kernel_launches", C.c_uint32),
        ("device_ms", C.c_float), ("error", ErrorRecord),
    ]


class ResultBuffers:
    """Caller-owned result storage for `products` products and `nodes` node entries."""

    @property
    def node_stats(self):
        return self.node_stats_array

    def __init__(self, products: int, nodes: int = 0, scrambles: int = 0):
        self.products = (ProductResult * max(products, 1))()
        self.node_stats_array = (Statistics * nodes)() if nodes else None
        self.node_estimates = (Estimate * nodes)() if nodes else None
        self.result = Result()
        self.result.product_capacity = products
        self.result.products = C.cast(self.products, C.POINTER(ProductResult))
        self.result.node_capacity = nodes
        if nodes:
            self.result.local_vega_nodes = C.cast(self.node_stats_array, C.POINTER(Statistics))
            self.result.local_vega_node_estimates = C.cast(self.node_estimates, C.POINTER(Estimate))
        # RQMC: each scramble's component means, [scramble][product][component]
        self.replicate_count = scrambles * products * PATHWISE_COMPONENTS
        self.replicate_array = (C.c_double * self.replicate_count)() if scrambles else None
        if scrambles:
            self.result.replicate_capacity = self.replicate_count
            self.result.replicate_means = C.cast(self.replicate_array, _dp)

    def replicate_means(self, product: int, component: int = PRICE) -> list:
        """The scramble means of one product's component, in scramble order."""
        if self.replicate_array is None:
            return []
        n = len(self.products)
        per = n * PATHWISE_COMPONENTS
        scrambles = self.replicate_count // per
        return [self.replicate_array[(s * n + product) * PATHWISE_COMPONENTS + component] for s in range(scrambles)]


# ---- early exercise (Longstaff--Schwartz) ----
LSM_MAX_DEGREE = 7
LSM_MAX_BASIS = LSM_MAX_DEGREE + 1
CONTINUATION_POLYNOMIAL, CONTINUATION_MLP = 0, 1
DOMAIN_VALUATION, DOMAIN_LSM_TRAIN = 0, 1
MLP_HIDDEN = 64
MLP_PARAMS = 64 * 2 + 64 + 64 * 64 + 64 + 64 + 1


class LsmDesc(C.Structure):
    _fields_ = [
        ("max_degree", C.c_uint32), ("itm_abs_tolerance", C.c_double),
        ("cpqr_abs_tolerance", C.c_double), ("cpqr_rel_tolerance", C.c_double),
        ("max_matrix_elements", C.c_uint64),
        ("training_seed", C.c_uint64), ("training_units", C.c_uint64),
        ("training_scramble_count", C.c_uint32), ("training_antithetic", C.c_int32),
        ("training_brownian_bridge", C.c_int32), ("continuation", C.c_int32),
        ("mlp_epochs", C.c_uint32), ("mlp_batch", C.c_uint32), ("mlp_learning_rate", C.c_float),
        ("mlp_seed", C.c_uint64),
    ]


class LsmDateModel(C.Structure):
    _fields_ = [
        ("regression", C.c_int32), ("itm_rows", C.c_uint32), ("candidate_rows", C.c_uint32),
        ("active_columns", C.c_uint32), ("diagonal_count", C.c_uint32), ("rank", C.c_uint32),
        ("feature_inactive", C.c_int32), ("reserved", C.c_uint32),
        ("feature_mean", C.c_double), ("feature_variance", C.c_double),
        ("feature_scale", C.c_double), ("zero_scale_threshold", C.c_double),
        ("pivot_order", C.c_uint32 * LSM_MAX_BASIS), ("diagonal_abs", C.c_double * LSM_MAX_BASIS),
        ("rank_threshold", C.c_double), ("coefficients", C.c_double * LSM_MAX_BASIS),
        ("residual_sum_squares", C.c_double),
    ]


class LsmResult(C.Structure):
    _fields_ = [
        ("date_capacity", C.c_uint32), ("models", C.POINTER(LsmDateModel)),
        ("exercise_counts", C.POINTER(C.c_uint64)),
        ("stopping_capacity", C.c_uint64), ("stopping_indices", C.POINTER(C.c_uint32)),
        ("price_statistics", Statistics), ("price", Estimate),
        ("sampling_variance", C.c_double), ("estimator_variance", C.c_double),
        ("in_sample_value", C.c_double),
        ("training_paths", C.c_uint64), ("valuation_paths", C.c_uint64),
        ("independent_sampling_units", C.c_uint64),
        ("date_count", C.c_uint32), ("kernel_launches", C.c_uint32),
        ("device_ms", C.c_float), ("path_kernel_ms", C.c_float),
        ("regression_ms", C.c_float), ("valuation_ms", C.c_float),
        ("risk_components", Statistics * PATHWISE_COMPONENTS),
        ("delta", Estimate), ("gamma", Estimate), ("vega", Estimate),
        ("bump_delta", Estimate), ("bump_gamma", Estimate), ("bump_vega", Estimate),
        ("continuation_used", C.c_int32), ("mlp_steps", C.c_uint32), ("mlp_ms", C.c_float),
        ("mlp_final_loss", C.c_float), ("polynomial_in_sample", C.c_double), ("mlp_in_sample", C.c_double),
        ("mlp_param_capacity", C.c_uint32), ("mlp_params", C.POINTER(C.c_float)),
        ("node_capacity", C.c_uint32), ("local_vega_nodes", C.POINTER(Statistics)),
                ("local_vega_node_estimates", C.POINTER(Estimate)), ("error", ErrorRecord),
    ]


class DualDesc(C.Structure):
    """mcg_dual_desc: the Andersen--Broadie inner path counts and seed."""
    _fields_ = [("continuation_inner_paths", C.c_uint32), ("exercise_inner_paths", C.c_uint32),
                ("inner_seed", C.c_uint64)]


class DualResult(C.Structure):
    _fields_ = [
        ("components", Statistics * 3),
        ("lower_bound", Estimate), ("upper_bound", Estimate), ("duality_gap", Estimate),
        ("price_confidence_interval_95", C.c_double * 2),
        ("outer_trajectories", C.c_uint64), ("inner_paths", C.c_uint64),
        ("exercise_date_count", C.c_uint32), ("kernel_launches", C.c_uint32),
        ("device_ms", C.c_float), ("nested_ms", C.c_float),
        ("error", ErrorRecord),
    ]


class LsmBuffers:
    """Caller-owned storage for an early-exercise result of `dates` exercise
    dates and, when `stopping` > 0, that many valuation stopping indices."""

    def __init__(self, dates: int, stopping: int = 0, nodes: int = 0):
        self.node_stats = (Statistics * nodes)() if nodes else None
        self.node_estimates = (Estimate * nodes)() if nodes else None
        self.models = (LsmDateModel * max(dates, 1))()
        self.counts = (C.c_uint64 * max(dates, 1))()
        self.stops = (C.c_uint32 * stopping)() if stopping else None
        self.mlp_params = (C.c_float * MLP_PARAMS)()
        self.result = LsmResult()
        self.result.mlp_param_capacity = MLP_PARAMS
        self.result.mlp_params = C.cast(self.mlp_params, C.POINTER(C.c_float))
        self.result.date_capacity = dates
        self.result.models = C.cast(self.models, C.POINTER(LsmDateModel))
        self.result.exercise_counts = C.cast(self.counts, C.POINTER(C.c_uint64))
        self.result.stopping_capacity = stopping
        if stopping:
            self.result.stopping_indices = C.cast(self.stops, C.POINTER(C.c_uint32))
        self.result.node_capacity = nodes
        if nodes:
            self.result.local_vega_nodes = C.cast(self.node_stats, C.POINTER(Statistics))
            self.result.local_vega_node_estimates = C.cast(self.node_estimates, C.POINTER(Estimate))


# ---- batched book ----
class BookOptions(C.Structure):
    _fields_ = [("autotune", C.c_int32), ("tiles_per_item", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("use_graph", C.c_int32)]


class BookReport(C.Structure):
    _fields_ = [("trade_count", C.c_uint32), ("items", C.c_uint32), ("tiles_per_item", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("ctas", C.c_uint32), ("kernel_launches", C.c_uint32),
                ("graph", C.c_int32), ("device_ms", C.c_float), ("autotune_ms", C.c_float),
                ("path_steps", C.c_uint64), ("error", ErrorRecord)]

/*
 * mcg.h -- C ABI of the B200 Monte Carlo pricing engine.
 *
 * The engine replaces the CPU executor seam of msfmfjt/rust-pricing-library:
 *
 *   SimulationPlan::execute            crates/pricing/src/engine/risk/valuation.rs:19-33
 *     -> execute_pseudo / execute_rqmc crates/pricing/src/engine/risk/valuation.rs:126-437
 *     -> execute_local_vol_pseudo/rqmc crates/pricing/src/engine/risk/local_vol.rs:24-420
 *     -> DeterministicExecutor::try_map_reduce_*  crates/pricing/src/engine/mc/execution.rs:361-726
 *
 * A caller compiles a request into an `mcg_plan_desc` (the data the reference
 * keeps in its immutable `SimulationPlan`, crates/pricing/src/engine/plan/simulation.rs:73-119),
 * hands it to `mcg_plan_create`, and evaluates the plan on a CUDA stream.  The
 * result carries, per product, the 18 pathwise components as
 * `DeterministicStatistics` records (crates/pricing/src/engine/mc/execution.rs:140-166)
 * reduced in a fixed order, plus the estimates the reference builds from them
 * (crates/pricing/src/engine/risk/report.rs:454-473).
 *
 * Everything here is plain C11: pointers, sizes and scalars.  Arrays passed in a
 * descriptor are owned by the caller and copied during `mcg_plan_create`.
 * Every entry point returns an `mcg_status`; none of them aborts the process.
 */
#ifndef MCG_H
#define MCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCG_ABI_VERSION 3u

/* Component layout of one sampling unit, crates/pricing/src/engine/plan/simulation.rs:26-62. */
#define MCG_PRICE 0
#define MCG_DELTA 1
#define MCG_VEGA 2
#define MCG_GAMMA 3
#define MCG_BUMP_DELTA 4
#define MCG_DELTA_DIFFERENCE 5
#define MCG_BUMP_VEGA 6
#define MCG_VEGA_DIFFERENCE 7
#define MCG_BUMP_GAMMA 8
#define MCG_GAMMA_DIFFERENCE 9
#define MCG_BARRIER_ENDPOINT_HIT 10
#define MCG_BARRIER_DIVIDEND_JUMP_HIT 11
#define MCG_BARRIER_BRIDGE_HIT_WEIGHT 12
#define MCG_BARRIER_INTERVAL_COUNT 13
#define MCG_BARRIER_FINITE_CORRECTION_COUNT 14
#define MCG_BARRIER_ZERO_VARIANCE_COUNT 15
#define MCG_BARRIER_SURVIVAL_UNDERFLOW_COUNT 16
#define MCG_BARRIER_CERTAIN_SURVIVAL_COUNT 17
#define MCG_PATHWISE_COMPONENTS 18

/* Limits.  MCG_MAX_SOBOL_DIMENSION is RqmcConfig::MAX_SOBOL_DIMENSION
 * (crates/pricing/src/engine/mc/config.rs:88). */
#define MCG_MAX_SOBOL_DIMENSION 21201u
#define MCG_MAX_PRODUCTS 8u

/* Status codes.  They mirror the reference's error variants
 * (crates/pricing/src/api/error.rs:256-301, LocalVolError
 * crates/pricing/src/engine/processes/local_vol.rs:24-73,
 * BarrierBridgeError crates/pricing/src/engine/payoff/barrier_bridge.rs:27-55). */
typedef enum mcg_status {
    MCG_OK = 0,
    MCG_ERR_INVALID_ARGUMENT = 1,      /* malformed descriptor; `mcg_last_error` names the field */
    MCG_ERR_UNSUPPORTED = 2,           /* a combination this engine does not implement */
    MCG_ERR_CUDA = 3,                  /* CUDA runtime failure (no device, launch failure, ...) */
    MCG_ERR_ALLOCATION = 4,            /* device or host allocation failed */
    MCG_ERR_INSUFFICIENT_UNITS = 5,    /* MonteCarloError::InsufficientSamplingUnits */
    MCG_ERR_NON_FINITE_STATE = 6,      /* LocalVolError::NonFiniteState{step,bits} */
    MCG_ERR_INVALID_SURFACE_QUERY = 7, /* MarketError::InvalidSurfaceQuery */
    MCG_ERR_SOBOL_DIMENSION = 8,       /* RqmcPlanError::DimensionLimitExceeded */
    MCG_ERR_BRIDGE = 9,                /* BrownianBridgeError */
    MCG_ERR_BARRIER_BRIDGE = 10,       /* BarrierBridgeError */
    MCG_ERR_MARKET = 11,               /* MarketError (curve, surface, grid) */
    MCG_ERR_LSM = 12,                  /* LsmNumericalError */
    MCG_ERR_TIMEOUT = 13,              /* a bounded device wait ran out */
    MCG_ERR_NOT_BUILT = 14             /* a kernel variant is missing from the compiled library */
} mcg_status;

typedef enum mcg_model_kind {
    MCG_MODEL_BLACK_SCHOLES = 0,
    MCG_MODEL_LOCAL_VOLATILITY = 1
} mcg_model_kind;

typedef enum mcg_engine_kind {
    MCG_ENGINE_PSEUDO = 0, /* PseudoMcConfig, crates/pricing/src/engine/mc/config.rs */
    MCG_ENGINE_RQMC = 1    /* RqmcConfig */
} mcg_engine_kind;

typedef enum mcg_product_kind {
    MCG_PRODUCT_EUROPEAN = 0,
    MCG_PRODUCT_DIGITAL = 1,
    MCG_PRODUCT_ASIAN = 2,
    MCG_PRODUCT_LOOKBACK = 3,
    MCG_PRODUCT_DISCRETE_BARRIER = 4,
    MCG_PRODUCT_CONTINUOUS_BARRIER = 5,
    MCG_PRODUCT_AMERICAN = 6
} mcg_product_kind;

typedef enum mcg_side { MCG_CALL = 0, MCG_PUT = 1 } mcg_side;
typedef enum mcg_barrier_direction { MCG_BARRIER_UP = 0, MCG_BARRIER_DOWN = 1 } mcg_barrier_direction;
typedef enum mcg_barrier_style { MCG_KNOCK_OUT = 0, MCG_KNOCK_IN = 1 } mcg_barrier_style;
typedef enum mcg_digital_payout { MCG_DIGITAL_CASH = 0, MCG_DIGITAL_ASSET = 1 } mcg_digital_payout;

/* Arithmetic of the path bulk.  FP64 reproduces the reference; FP32 runs the
 * state evolution in single precision and keeps payoff and statistics in FP64. */
typedef enum mcg_precision { MCG_PRECISION_F64 = 0, MCG_PRECISION_F32_BULK = 1 } mcg_precision;

/* Log-linear discount curve, LogLinearDiscountCurve
 * (crates/pricing/src/market/curve.rs:38-200). */
typedef struct mcg_curve {
    uint32_t pillar_count;
    const double* times;            /* strictly increasing, times[0] >= 0 */
    const double* discount_factors; /* positive */
} mcg_curve;

/* Dupire local-variance grid, LocalVarianceGrid
 * (crates/pricing/src/market/local_variance.rs:125-206).  `values` is
 * time-major: values[t * log_moneyness_count + x]. */
typedef struct mcg_local_variance_grid {
    uint32_t time_count;
    uint32_t log_moneyness_count;
    const double* time_nodes;          /* time_nodes[0] == +0.0, last == expiry time */
    const double* log_moneyness_nodes; /* strictly increasing */
    const double* values;
    double floor;
    double cap;
} mcg_local_variance_grid;

/* Discrete dividends of the escrowed affine model, AffineDividendTransform
 * with the plan's discount and dividend curves as carry curves
 * (crates/pricing/src/market/dividend.rs:137-520, market/forward.rs:129-160):
 * ex-dividend times (ACT/365F year fractions, finite, >= 0, strictly
 * increasing), fixed cash amounts (finite, >= 0) and proportional fractions
 * (in [0, 1)).  The simulated state f is the canonical continuous martingale
 * with forward S0 Dq(t)/Dr(t); every observed spot is S = A(t) S0 + B(t) f(t),
 * A the discounted cash reserve still to be paid and B the proportional
 * factor, and an observation on an ex-dividend date of a discrete barrier
 * also checks the spot just before the dividend.  A local-volatility plan adds
 * the ex-times up to expiry to its time grid.  count = 0: no dividends. */
typedef struct mcg_dividends {
    uint32_t count;
    const double* ex_times;
    const double* fixed_cash;
    const double* proportional;
} mcg_dividends;

/* One product.  All products of one plan observe the same dates
 * (`observation_times` of the plan); the product's own arrays index those. */
typedef struct mcg_product_desc {
    int32_t kind;      /* mcg_product_kind */
    int32_t side;      /* mcg_side */
    double strike;
    double notional;
    /* Digital, crates/pricing/src/engine/payoff/compile.rs:104-157 */
    int32_t digital_payout; /* mcg_digital_payout */
    double payout;
    /* Barrier, crates/pricing/src/engine/payoff/compile.rs:204-403 */
    int32_t barrier_direction; /* mcg_barrier_direction */
    int32_t barrier_style;     /* mcg_barrier_style */
    int32_t has_rebate;
    double barrier;
    double rebate;
    /* One value per plan observation.  Arithmetic Asian: the weight of the
     * observation (required; crates/pricing/src/engine/payoff/compile.rs:159-202).
     * Discrete barrier and fixed lookback: optional monitoring flags, 0.0 where
     * the observation is not one of the product's monitoring dates (a barrier
     * whose expiry is not monitored); NULL monitors every observation. */
    const double* observation_weights;
    /* Seasoned state, the literals of the reference's graphs for dates before
     * the first simulated observation.  Asian: the weighted sum of the known
     * fixings, accumulated in observation order (compile.rs:162-176).  Fixed
     * lookback: the running extremum before the first simulated monitoring date,
     * from the historical extremum and/or the valuation-date fixing
     * (compile.rs:405-440).  Discrete barrier: 1.0 when the barrier was hit
     * before the valuation date, else 0.0 (compile.rs:293-297).  Ignored
     * unless has_initial_state is nonzero. */
    int32_t has_initial_state;
    double initial_state;
} mcg_product_desc;

/* The compiled plan: the hot-path part of the reference's SimulationPlan. */
typedef struct mcg_plan_desc {
    uint32_t abi_version; /* MCG_ABI_VERSION */
    int32_t model;        /* mcg_model_kind */
    int32_t engine;       /* mcg_engine_kind */
    int32_t precision;    /* mcg_precision */

    /* Engine configuration.  Pseudo: `sampling_units` independent units under
     * `master_seed`.  RQMC: `sampling_units` points per scramble (a power of
     * two) times `scramble_count` scrambles under `master_seed`. */
    uint64_t master_seed;
    uint64_t sampling_units;
    uint32_t scramble_count;
    uint32_t scramble_begin;       /* RQMC: index of the first scramble (shards of one plan) */
    int32_t antithetic;
    int32_t brownian_bridge;
    uint64_t reduction_block_size; /* ExecutionPolicy, default 4096 */
    /* Joe--Kuo direction words for RQMC, `sobol_dimension_count` x 32,
     * dimension-major (the reference's embedded asset
     * crates/pricing/data/joe-kuo-6.21201-u32be.bin, decoded). */
    uint32_t sobol_dimension_count;
    const uint32_t* sobol_directions;

    /* Market. */
    double spot;
    mcg_curve discount_curve;
    mcg_curve dividend_curve;
    double volatility; /* Black-Scholes only */
    mcg_local_variance_grid local_variance; /* local volatility only */

    /* Contract timing.  `observation_times` are ACT/365F year fractions of the
     * product's fixing dates (strictly increasing, > 0); the last one is the
     * expiry.  `payment_time` discounts the payoff. */
    uint32_t observation_count;
    const double* observation_times;
    double payment_time;

    /* Products priced on the same draws. */
    uint32_t product_count;
    const mcg_product_desc* products;

    /* Risk request, RiskRequest (crates/pricing/src/risk/request.rs:227). */
    int32_t request_delta;
    int32_t request_gamma;
    int32_t request_vega;
    int32_t request_local_vega_nodes; /* LV: per-node local-vega sensitivities */
    int32_t gamma_bump_relative;      /* 1: relative, 0: absolute */
    double gamma_bump;                /* relative fraction or absolute amount */
    double smoothing_half_width;      /* PayoffSmoothing::compact_c2; 0 = exact */
    uint32_t checkpoint_interval;     /* LV reverse: steps between stored states */
    /* Discrete dividends (see mcg_dividends).  With dividends the engine prices
     * European, Digital, Asian, Lookback and discrete-barrier products:
     * Black--Scholes with its full pathwise risk, local volatility with price
     * and CRN Delta/Gamma; continuous barriers, early exercise, local Vega and
     * node sensitivities, and the FP32 bulk return MCG_ERR_UNSUPPORTED. */
    mcg_dividends discrete_dividends;
} mcg_plan_desc;

typedef struct mcg_statistics {
    double sum;        /* NeumaierSum (crates/pricing-numerics/src/reduction.rs:3-56) */
    double correction;
    uint64_t count;    /* CenteredMoment (reduction.rs:73-170) */
    double mean;
    double second_moment;
} mcg_statistics;

typedef struct mcg_estimate {
    double value;
    double standard_error;
    double confidence_lower;
    double confidence_upper;
    uint64_t effective_sampling_units;
} mcg_estimate;

typedef struct mcg_product_result {
    mcg_statistics components[MCG_PATHWISE_COMPONENTS];
    mcg_estimate price;
    mcg_estimate delta;
    mcg_estimate gamma;
    mcg_estimate vega;
    mcg_estimate bump_delta;
    mcg_estimate bump_gamma;
    mcg_estimate bump_vega;
    double sampling_variance;
    double estimator_variance;
    /* Local volatility with Vega and Delta requested: the adjoint sweep's spot
     * Delta dP/dS0 and the central difference of adjoint Deltas at S +/- h
     * (beyond the reference, which bumps Delta and Gamma for local vol). */
    mcg_statistics adjoint_components[2];
    mcg_estimate adjoint_delta;
    mcg_estimate adjoint_gamma;
} mcg_product_result;

typedef struct mcg_error_record {
    int32_t code;          /* mcg_status of the first failing unit */
    uint32_t step;         /* step or index inside the unit */
    uint64_t sampling_unit;
    uint64_t value_bits;   /* bit pattern of the offending value */
} mcg_error_record;

typedef struct mcg_result {
    uint32_t product_capacity;       /* entries available in `products` */
    mcg_product_result* products;    /* caller-owned */
    /* Local-volatility node sensitivities (grid value count entries each),
     * caller-owned; NULL when not requested. */
    uint32_t node_capacity;
    mcg_statistics* local_vega_nodes;
    mcg_estimate* local_vega_node_estimates;

    uint64_t independent_sampling_units;
    uint64_t evaluated_paths;
    uint32_t time_steps;       /* path steps per evaluated path */
    uint32_t effective_dimension;
    uint32_t reduction_records;
    uint32_t kernel_launches;  /* kernels this evaluation launched */
    float device_ms;           /* device time of the evaluation (CUDA events) */
    float path_kernel_ms;      /* device time of the path kernel alone */
    mcg_error_record error;
    /* RQMC: every scramble's mean of every component (the replicates whose
     * two-pass moments the statistics above are, crates/pricing/src/engine/risk/valuation.rs:349-361),
     * replicate_means[(s * product_count + k) * MCG_PATHWISE_COMPONENTS + c]
     * for the plan's scrambles s in order; caller-owned, replicate_capacity
     * entries, NULL when not wanted (and left untouched for pseudo-MC).
     * Shards of one plan (scramble_begin) gathered in scramble order give,
     * by the same two-pass, the whole plan's statistics bit for bit. */
    uint32_t replicate_capacity;
    double* replicate_means;
} mcg_result;

typedef struct mcg_plan mcg_plan;

/* Library identity and the last error message of the calling thread. */
uint32_t mcg_abi_version(void);
const char* mcg_last_error(void);

/* Compile a plan: validates the descriptor, builds the time grid, the Brownian
 * bridge, the RQMC scramble table and the device-resident layout.  Replaces
 * SimulationPlan::compile's runtime part (crates/pricing/src/engine/compile/simulation.rs:78-700,
 * crates/pricing/src/engine/compile/local_vol.rs:14-102). */
mcg_status mcg_plan_create(const mcg_plan_desc* desc, mcg_plan** out_plan);

/* Evaluate on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * synchronise.  Replaces SimulationPlan::execute
 * (crates/pricing/src/engine/risk/valuation.rs:19-33). */
mcg_status mcg_plan_evaluate(mcg_plan* plan, void* stream, mcg_result* result);

/* Evaluate from host-resident descriptor arrays in one call: create, evaluate,
 * destroy.  The PricingPlan::compile + evaluate pair of the facade
 * (crates/pricing/src/engine/risk/pricing.rs:53-88). */
mcg_status mcg_price(const mcg_plan_desc* desc, void* stream, mcg_result* result);

void mcg_plan_destroy(mcg_plan* plan);

/* Plan introspection: time steps and effective Sobol dimension. */
mcg_status mcg_plan_shape(const mcg_plan* plan, uint32_t* time_steps,
                          uint32_t* effective_dimension, uint32_t* grid_value_count);

/* ---- Sampling primitives, exposed for replay and known-answer tests ---- */

/* Standard normals of `count` consecutive sampling units, dimension-major
 * out[d * count + i], for the Philox coordinate stream
 * (crates/pricing/src/engine/sampling/random.rs:100-149,176-277). */
mcg_status mcg_philox_normals(uint64_t master_seed, uint64_t first_unit, uint64_t count,
                              uint32_t dimensions, uint32_t domain, double* out_host);

/* Scrambled Sobol words of `count` consecutive points of one scramble,
 * dimension-major out[d * count + i]
 * (crates/pricing/src/engine/sampling/qmc.rs:47-132,204-369).  `directions`
 * holds the Joe--Kuo direction words, dimensions x 32.  When first_point and
 * count are multiples of 32 the words are formed the way the path kernels
 * form them (a warp per 32 aligned points: common Gray-code part by an XOR
 * reduction over the warp, lane part from the low-word table); otherwise one
 * thread per point walks the set Gray-code bits.  first_point + count <= 2^32. */
mcg_status mcg_rqmc_words(const uint32_t* directions, uint32_t dimensions, uint64_t master_seed,
                          uint32_t scramble, uint64_t first_point, uint64_t count,
                          uint32_t* out_host);

/* Dupire local-variance grid from a standard SSVI surface with a power-law
 * phi and PCHIP theta curve, computed on the device
 * (crates/pricing/src/market/local_variance.rs:149-206,
 *  crates/pricing/src/market/ssvi.rs:121-176,226-273,410-479,
 *  crates/pricing/src/market/pchip.rs:111-237).  `values` receives
 * time_count x log_moneyness_count entries; `repairs` (may be NULL) the number
 * of floor/cap repairs. */
mcg_status mcg_ssvi_local_variance_grid(const double* theta_times, const double* theta_values,
                                        uint32_t theta_count, double terminal_slope, double rho,
                                        double eta, double gamma, const double* time_nodes,
                                        uint32_t time_count, const double* log_moneyness_nodes,
                                        uint32_t log_moneyness_count, double floor, double cap,
                                        double* values, uint32_t* repairs);

/* ---- Implied-variance surfaces ----
 *
 * The surfaces LocalVarianceGrid::from_surface turns into a Dupire grid
 * (crates/pricing/src/market/local_variance.rs:149-206):
 *   standard SSVI with a PCHIP theta curve and a power-law or Heston-like phi
 *     (crates/pricing/src/market/ssvi.rs:61-176,347-388,410-525,
 *      crates/pricing/src/market/pchip.rs:111-237);
 *   eSSVI slices (time, theta, psi, rho*psi) interpolated linearly in time,
 *     scaled towards zero before the first slice, theta extended with the
 *     terminal slope after the last (crates/pricing/src/market/essvi.rs:104-396).
 * Validation follows the reference's constructors with its local_vol_vegakt_v1
 * tolerance (absolute 1e-14, relative 1e-12). */
typedef enum {
    MCG_SURFACE_SSVI_POWER_LAW = 0,
    MCG_SURFACE_SSVI_HESTON_LIKE = 1,
    MCG_SURFACE_ESSVI = 2
} mcg_surface_kind;

typedef struct {
    int32_t kind;                  /* mcg_surface_kind */
    /* SSVI: theta curve knots and the PCHIP long-end slope */
    const double* theta_times;
    const double* theta_values;
    uint32_t theta_count;
    double terminal_theta_slope;   /* SSVI and eSSVI: d theta / dt after the last knot/slice */
    double rho;                    /* SSVI correlation */
    double eta, gamma;             /* power-law phi = eta / (theta^gamma (1 + theta)^(1 - gamma)) */
    double lambda;                 /* Heston-like phi = (z - 1 + e^-z) / z^2, z = lambda theta */
    /* eSSVI slices, increasing in time */
    const double* slice_times;
    const double* slice_thetas;
    const double* slice_psis;
    const double* slice_rho_psis;
    uint32_t slice_count;
} mcg_surface_desc;

/* Dupire local-variance grid of any surface kind, computed on the device;
 * as mcg_ssvi_local_variance_grid. */
mcg_status mcg_surface_local_variance_grid(const mcg_surface_desc* surface, const double* time_nodes,
                                           uint32_t time_count, const double* log_moneyness_nodes,
                                           uint32_t log_moneyness_count, double floor, double cap,
                                           double* values, uint32_t* repairs);

/* Total variance and its derivatives at `count` (time, log-moneyness) points,
 * evaluated by the device code the grid uses:
 * out[4 i + 0..3] = w, dw/dk, d2w/dk2, dw/dt
 * (ImpliedVarianceSurface::total_variance_derivatives). */
mcg_status mcg_surface_total_variance(const mcg_surface_desc* surface, const double* times,
                                      const double* log_moneyness, uint32_t count, double* out);

/* ---- VegaKT: local-vega node allocation to reporting-IV buckets ----
 *
 * Replaces allocate_local_vol_nodes and project_local_vega_nodes_to_reporting_iv
 * (crates/pricing/src/engine/risk/local_vol_allocation.rs:108-163,
 *  crates/pricing/src/engine/risk/vegakt.rs:541-570,856-949) with the active
 * density domains of analytic_call_density_rows_from_surface over the
 * reporting-IV surface (vegakt.rs:90-156, compile_local_vol_vega_kt_runtime in
 * crates/pricing/src/engine/compile/local_vol.rs:104-148,
 * crates/pricing/src/engine/processes/local_vol_valuation.rs:67-123).
 * The reference projects every path's node sensitivities and averages; the
 * projection is linear, so the engine projects the node-sensitivity means of
 * mcg_result.local_vega_node_estimates (one call, on the host).  Edge counts
 * are per evaluated path, as the reference counts them. */
typedef struct {
    const double* maturity_nodes;          /* increasing; the grid's positive times must be among them */
    uint32_t maturity_count;
    const double* log_moneyness_nodes;     /* increasing */
    uint32_t log_moneyness_count;
    const double* implied_volatilities;    /* maturity_count x log_moneyness_count, positive */
    const double* forwards;                /* forward at each maturity node */
    double relative_density_threshold;     /* in (0, 1] */
} mcg_vega_kt_basis;

typedef struct {
    uint32_t bucket_capacity;
    double* raw_buckets;                   /* maturity_count x log_moneyness_count */
    double scalar_vega;                    /* sum of the buckets */
    double signed_residual;                /* initial_time + density_excluded, as the report's projection
                                              (crates/pricing/src/engine/risk/report.rs:206-216) */
    double density_excluded;               /* node sensitivity outside the active density domains */
    double pre_projection;                 /* all nodes (the scalar local Vega) = scalar_vega + signed_residual */
    double initial_time;                   /* the t = 0 row */
    double left_edge_sensitivity, right_edge_sensitivity;
    uint64_t left_edge_count, right_edge_count;
} mcg_vega_kt_projection;

mcg_status mcg_vega_kt_project(const double* grid_time_nodes, uint32_t time_count,
                               const double* grid_log_moneyness_nodes, uint32_t log_moneyness_count,
                               const double* node_sensitivities, uint64_t evaluated_paths,
                               const mcg_vega_kt_basis* basis, mcg_vega_kt_projection* out);

/* ---- Early exercise: Longstaff--Schwartz regression ----
 *
 * Replaces SimulationPlan::execute_early_exercise and its RQMC twin
 * (crates/pricing/src/engine/risk/early_exercise.rs:24-120,251-313): path
 * matrices of a training and a valuation engine
 * (crates/pricing/src/engine/mc/early_exercise.rs:28-450), the backward
 * regression train_exercise_policy (crates/pricing/src/engine/mc/lsm.rs:1486-1695)
 * over a polynomial basis in the standardised spot with column-pivoted QR
 * (lsm.rs:1928-2230,2374-2652), and value_exercise_policy (lsm.rs:1347-1482).
 *
 * The plan descriptor holds one product of kind MCG_PRODUCT_AMERICAN; its
 * `observation_times` are the exercise times, the last one the expiry (the
 * American payoff graph observes exactly the exercise dates,
 * crates/pricing/src/engine/payoff/compile.rs:67-101).  Its engine fields are
 * the valuation engine; `mcg_lsm_desc` adds the training engine (same kind) and
 * the regression configuration (LsmConfig).  Risk requests ask for the
 * fixed-policy Greeks of mcg_lsm_result (Black-Scholes and local volatility). */
#define MCG_LSM_MAX_DEGREE 7u
#define MCG_LSM_MAX_BASIS (MCG_LSM_MAX_DEGREE + 1u)

typedef enum mcg_continuation_kind {
    MCG_CONTINUATION_POLYNOMIAL = 0, /* the reference's CPQR regression */
    MCG_CONTINUATION_MLP = 1         /* learned continuation value, see mcg_lsm_desc */
} mcg_continuation_kind;

typedef struct mcg_lsm_desc {
    /* PolynomialBasisSpec(feature_count 1, max_degree) over the spot state
     * variable, CpqrConfig, itm_abs_tolerance and max_matrix_elements of the
     * reference's LsmConfig (crates/pricing/src/engine/mc/lsm.rs:328-495). */
    uint32_t max_degree; /* 1 .. MCG_LSM_MAX_DEGREE */
    double itm_abs_tolerance;
    double cpqr_abs_tolerance;
    double cpqr_rel_tolerance;
    uint64_t max_matrix_elements;
    /* Training engine (LsmConfig::training_engine), the plan's engine kind. */
    uint64_t training_seed;
    uint64_t training_units;          /* pseudo: sampling units; RQMC: points per scramble */
    uint32_t training_scramble_count; /* RQMC only */
    int32_t training_antithetic;
    int32_t training_brownian_bridge;
    int32_t continuation;             /* mcg_continuation_kind */
    /* Learned continuation (MCG_CONTINUATION_MLP, no counterpart in the
     * reference): one 2 -> 64 -> 64 -> 1 SiLU network of the scaled spot
     * 4 (S - K) / K and the scaled time 2 t / T - 1, BF16 operands and FP32
     * accumulation, fitted by Adam in the same backward induction as the
     * regression: at each date, from the previous date's weights, on the ITM
     * training rows and their discounted cash flows.  Its policy exercises
     * an ITM path when the immediate value beats the predicted continuation.
     * The polynomial policy is fitted too and is used instead (fallback) when
     * the network's training diverges or its in-sample value is lower.
     * Adam steps per date: with mlp_epochs = 0, max(batches, 400) at the last
     * non-terminal date (trained from scratch) and max(batches, 50) at the
     * others (warm-started); otherwise epochs x batches, 4x at the last
     * non-terminal date. */
    uint32_t mlp_epochs;      /* passes over each date's rows; 0 = the default schedule */
    uint32_t mlp_batch;       /* training rows per Adam step; 0 = 16384 */
    float mlp_learning_rate;  /* Adam step size; 0 = 2e-3 */
    uint64_t mlp_seed;        /* initial weights */
} mcg_lsm_desc;

/* Parameters of the continuation network, FP32, in this order:
 * W1[64][2], b1[64], W2[64][64], b2[64], W3[64], b3. */
#define MCG_MLP_HIDDEN 64u
#define MCG_MLP_PARAMS (64u * 2u + 64u + 64u * 64u + 64u + 64u + 1u)

/* One non-terminal exercise date's decision model: the reference's
 * ExerciseDecisionModel (lsm.rs:796-818) with the PolynomialRegressionModel
 * fields (lsm.rs:610-790).  Basis column c is the monomial z^c of the
 * standardised spot z. */
typedef struct mcg_lsm_date_model {
    int32_t regression;             /* 0: ContinueAll (no ITM training path) */
    uint32_t itm_rows;              /* ExerciseRegressionDiagnostics::itm_rows */
    uint32_t candidate_rows;
    uint32_t active_columns;        /* basis columns kept (all, or just z^0 when inactive) */
    uint32_t diagonal_count;        /* min(itm_rows, active_columns) */
    uint32_t rank;
    int32_t feature_inactive;       /* FeatureScaling::inactive */
    uint32_t reserved;
    double feature_mean;
    double feature_variance;        /* population variance */
    double feature_scale;
    double zero_scale_threshold;
    uint32_t pivot_order[MCG_LSM_MAX_BASIS]; /* basis columns in pivot order */
    double diagonal_abs[MCG_LSM_MAX_BASIS];  /* |R_kk| in pivot order */
    double rank_threshold;
    double coefficients[MCG_LSM_MAX_BASIS];  /* per basis column (max_degree + 1) */
    double residual_sum_squares;
} mcg_lsm_date_model;

typedef struct mcg_lsm_result {
    uint32_t date_capacity;         /* entries in `models` and `exercise_counts` */
    mcg_lsm_date_model* models;     /* date_count - 1 entries, caller-owned */
    uint64_t* exercise_counts;      /* date_count entries, caller-owned */
    uint64_t stopping_capacity;     /* entries in `stopping_indices` (0 = not wanted) */
    uint32_t* stopping_indices;     /* valuation stopping date per path, caller-owned */

    mcg_statistics price_statistics; /* over sampling units (pseudo) or replicates (RQMC) */
    mcg_estimate price;
    double sampling_variance;
    double estimator_variance;
    double in_sample_value;         /* training paths valued by the policy fitted on them */
    uint64_t training_paths;
    uint64_t valuation_paths;
    uint64_t independent_sampling_units;
    uint32_t date_count;
    uint32_t kernel_launches;
    float device_ms;                /* whole evaluation */
    float path_kernel_ms;           /* both path-matrix kernels */
    float regression_ms;            /* backward regression of the training phase */
    float valuation_ms;             /* policy valuation and statistics */
    /* Fixed-policy risk (the plan's request_delta / request_gamma /
     * request_vega, Black-Scholes): pathwise AAD of each valuation path's
     * discounted exercise value at its stopping date -- Delta and Vega by the
     * reverse sweep, Gamma as the central difference of AAD Deltas, and the
     * bump-and-revalue validation components -- reduced like the plan
     * components (constant_vol_fixed_policy_pseudo/rqmc_statistics,
     * crates/pricing/src/engine/mc/early_exercise.rs:454-600;
     * fixed_policy_pathwise_values, crates/pricing/src/engine/processes/black_scholes.rs:358-415).
     * Under local volatility (local_vol_fixed_policy_pseudo/rqmc_statistics_with_vega_kt,
     * crates/pricing/src/engine/risk/early_exercise.rs:465-700, over
     * local_vol_pathwise_values_and_buckets_inner,
     * crates/pricing/src/engine/risk/pathwise_local_vol.rs:127-361): Delta and
     * Gamma by central bumps of the spot on common paths (bump = the gamma bump,
     * or 1e-4 of spot), Vega by the reverse sweep seeded at the stopping date,
     * and -- with request_local_vega_nodes -- the per-node local-vega means and
     * their statistics in `local_vega_nodes` / `local_vega_node_estimates`
     * (node_capacity >= the grid's value count), which mcg_vega_kt_project
     * turns into VegaKT buckets. */
    mcg_statistics risk_components[MCG_PATHWISE_COMPONENTS];
    mcg_estimate delta;
    mcg_estimate gamma;
    mcg_estimate vega;
    mcg_estimate bump_delta;
    mcg_estimate bump_gamma;
    mcg_estimate bump_vega;
    /* Learned continuation only. */
    int32_t continuation_used;      /* the policy valued: mcg_continuation_kind */
    uint32_t mlp_steps;             /* Adam steps taken */
    float mlp_ms;                   /* device time of the network's training */
    float mlp_final_loss;           /* mean squared error of the last step (scaled targets) */
    double polynomial_in_sample;    /* in-sample value of the regression policy */
    double mlp_in_sample;           /* in-sample value of the network policy */
    uint32_t mlp_param_capacity;    /* entries in `mlp_params` (0 = not wanted) */
    float* mlp_params;              /* trained parameters, caller-owned */
    /* Local volatility with request_local_vega_nodes: per grid node (time-major). */
    uint32_t node_capacity;
    mcg_statistics* local_vega_nodes;
    mcg_estimate* local_vega_node_estimates;
    mcg_error_record error;
} mcg_lsm_result;

/* Train and value an early-exercise policy on the GPU.  Synchronises `stream`. */
mcg_status mcg_lsm_price(const mcg_plan_desc* plan, const mcg_lsm_desc* lsm, void* stream,
                         mcg_lsm_result* result);

/* ---- Andersen--Broadie dual upper bound of an early-exercise price ----
 *
 * Policy-based nested simulation around the fitted LSM policy
 * (AndersenBroadiePlan, crates/pricing/src/engine/risk/dual.rs:132-462;
 * Andersen and Broadie 2004, section 3).  Every outer valuation path is
 * stopped by the policy (the lower bound, equal to mcg_lsm_price's price on
 * the same request); at each exercise date before the last, inner paths from
 * the path's state, run to their own policy stop, estimate the continuation
 * value (exercise_inner_paths where the policy exercises, else
 * continuation_inner_paths); the martingale of those estimates gives each
 * path's duality gap.  Black--Scholes, pseudo-MC training and valuation
 * engines, polynomial continuation, no Greeks, one American product.  Inner
 * normals are Philox words of `inner_seed` at counter (path, dimension / 4,
 * 0x4455414c), path = outer trajectory * max(N2, N3) + inner index,
 * dimension = branch date * exercise dates + date. */
typedef struct mcg_dual_desc {
    uint32_t continuation_inner_paths; /* N2 */
    uint32_t exercise_inner_paths;     /* N3 */
    uint64_t inner_seed;
} mcg_dual_desc;

typedef struct mcg_dual_result {
    /* Per-unit statistics of (lower, upper, gap); an antithetic unit is the
     * average 0.5 primary + 0.5 mate. */
    mcg_statistics components[3];
    mcg_estimate lower_bound;
    mcg_estimate upper_bound;
    mcg_estimate duality_gap;
    double price_confidence_interval_95[2]; /* lower - 1.96 SE, upper + 1.96 SE */
    uint64_t outer_trajectories;
    uint64_t inner_paths;                   /* inner paths simulated */
    uint32_t exercise_date_count;
    uint32_t kernel_launches;
    float device_ms;
    float nested_ms;                        /* the inner-path kernel */
    mcg_error_record error;
} mcg_dual_result;

mcg_status mcg_lsm_dual(const mcg_plan_desc* plan, const mcg_lsm_desc* lsm, const mcg_dual_desc* dual,
                        void* stream, mcg_dual_result* result);

/* The continuation network on given rows, exposed for the gradient checks (no
 * counterpart in the reference): outputs for `count` rows of inputs x[2 i],
 * x[2 i + 1]; and the gradient of sum_i mask_i (f(x_i) - y_i)^2 with respect to
 * the MCG_MLP_PARAMS parameters, with that sum in *loss.  Host arrays. */
mcg_status mcg_mlp_forward(const float* params, const float* x, uint32_t count, float* out);
mcg_status mcg_mlp_gradient(const float* params, const float* x, const float* y, const uint8_t* mask,
                            uint32_t count, float* grad, float* loss);

/* ---- A book of trades in one launch per path family (no counterpart in the reference) ----
 *
 * Thousands of single-product plans -- each with its own model (Black-Scholes
 * or local volatility with its own grid), maturity and step count, strike and
 * product -- priced by one persistent kernel per path family (local
 * volatility with discrete products, two paths per thread; local volatility
 * with a continuous barrier; Black-Scholes single-terminal; Black-Scholes
 * multi-observation), each pulling (trade, tile-range) work items from its
 * own queue ordered heaviest first, followed by the per-trade tile reduction.
 * Each trade's price statistics are bit for bit those of mcg_plan_evaluate on
 * its own plan.  Trades must be pseudo-MC with the same sampling_units, one
 * product, no risk request, FP64, and (local volatility) no antithetic
 * pairing.  The tiles per work item are chosen at creation by timing
 * candidates on a stratified sample of the book (`autotune`), and the
 * evaluation can be captured once in a CUDA graph (`use_graph`) and replayed. */
typedef struct mcg_book mcg_book;

typedef struct mcg_book_options {
    int32_t autotune;        /* 1: time candidate launch shapes at creation and keep the fastest */
    uint32_t tiles_per_item; /* 128-unit tiles per work item when not autotuned; 0 = 4 */
    uint32_t ctas_per_sm;    /* cap on every family's resident CTAs per SM; 0 = as many as fit */
    int32_t use_graph;       /* 1: capture the evaluation in a CUDA graph at creation */
} mcg_book_options;

typedef struct mcg_book_report {
    uint32_t trade_count;
    uint32_t items;            /* work items of one evaluation */
    uint32_t tiles_per_item;   /* the launch shape in use */
    uint32_t ctas_per_sm;      /* of the heaviest family's kernel */
    uint32_t ctas;
    uint32_t kernel_launches;  /* per evaluation */
    int32_t graph;             /* 1: evaluated by replaying the captured graph */
    float device_ms;           /* one evaluation, CUDA events */
    float autotune_ms;         /* host wall time the autotuner spent at creation */
    uint64_t path_steps;       /* simulated path-steps of one evaluation */
    mcg_error_record error;    /* first failing trade: code, its index in `step`, unit, value */
} mcg_book_report;

mcg_status mcg_book_create(const mcg_plan_desc* trades, uint32_t trade_count, const mcg_book_options* options,
                           mcg_book** out_book);
/* `prices` receives one estimate per trade; `report` may be NULL. */
mcg_status mcg_book_evaluate(mcg_book* book, void* stream, mcg_estimate* prices, mcg_book_report* report);
void mcg_book_destroy(mcg_book* book);

/* ---- Correlated multi-asset paths ----
 *
 * MultiAssetPricingPlan::compile / evaluate (crates/pricing/src/engine/multi_asset/compile.rs:200-470,
 * multi_asset/path.rs:24-200, multi_asset/evaluate.rs:92-300) for Black--Scholes
 * and local-volatility assets on one time grid: the union of the expiry, the
 * correlation change times, every local-variance grid's time nodes up to the
 * expiry and the substeps of `maximum_step` (LocalVolTimeGrid::compile).  Per
 * sampling unit each asset's factor takes its own normals -- Philox
 * coordinate (unit, dimension) or scrambled Sobol, dimension factor x steps +
 * step, or step x assets + factor for RQMC with the Brownian bridge (every
 * factor's terminal bridge normal in the first dimensions) -- optionally
 * Brownian-bridged per factor, correlated per step by the lower Cholesky
 * factor of the step's correlation matrix (unpivoted, zero pivots below
 * 1e-12 allowed: CorrelationFactor::compile, crates/pricing-numerics/src/correlation.rs:61-180),
 * and evolves its asset: f <- f F_{s+1}/F_s exp(-sigma^2 dt/2 + sigma sqrt(dt) z)
 * (Black--Scholes) or the Log-Euler step on its grid (local volatility).  The
 * payoff is a basket option on sum_i w_i S_i(T) / scale_i or a worst-of
 * option on min_i S_i(T) / reference_i (crates/pricing/src/product/multi_asset.rs:77-246),
 * exact or compact-C2 smoothed, paid at `payment_time`; statistics as the
 * single-asset plans (antithetic pairs averaged, RQMC two-pass over scramble
 * means).  Price only. */
#define MCG_MAX_ASSETS 8u

typedef enum mcg_multi_product_kind {
    MCG_MULTI_BASKET = 0,   /* sum_i weights[i] S_i(T) / scales[i] */
    MCG_MULTI_WORST_OF = 1  /* min_i S_i(T) / scales[i] (the reference levels) */
} mcg_multi_product_kind;

typedef struct mcg_asset_desc {
    int32_t model;          /* mcg_model_kind */
    double spot;
    mcg_curve dividend_curve;
    double volatility;      /* Black--Scholes */
    mcg_local_variance_grid local_variance; /* local volatility */
} mcg_asset_desc;

typedef struct mcg_multi_asset_desc {
    uint32_t abi_version;   /* MCG_ABI_VERSION */
    uint32_t asset_count;   /* 1 .. MCG_MAX_ASSETS */
    const mcg_asset_desc* assets;
    mcg_curve discount_curve;
    /* Correlation term structure: `correlation_count` matrices (asset_count^2,
     * row-major), matrix k in force from correlation_times[k] (increasing; the
     * first <= 0) until the next. */
    uint32_t correlation_count;
    const double* correlation_times;
    const double* correlations;
    double maximum_step;
    double expiry;
    double payment_time;
    /* engine */
    int32_t engine;         /* mcg_engine_kind */
    uint64_t master_seed;
    uint64_t sampling_units;
    uint32_t scramble_count;
    int32_t antithetic;
    int32_t brownian_bridge;
    uint64_t reduction_block_size;  /* ExecutionPolicy block size of the statistics; 0 = 4096 */
    uint32_t sobol_dimension_count;
    const uint32_t* sobol_directions;
    /* product */
    int32_t product;        /* mcg_multi_product_kind */
    int32_t side;           /* mcg_side */
    double strike;
    double notional;
    const double* weights;  /* basket: per asset (ignored by the worst-of) */
    const double* scales;   /* basket scales / worst-of reference levels, positive */
    double smoothing_half_width;
} mcg_multi_asset_desc;

typedef struct mcg_multi_asset_result {
    mcg_statistics price_statistics;
    mcg_estimate price;
    double sampling_variance;
    uint64_t evaluated_paths;
    uint64_t independent_sampling_units;
    uint32_t time_steps;
    uint32_t dimension;
    uint32_t kernel_launches;
    float device_ms;
    mcg_error_record error;
} mcg_multi_asset_result;

mcg_status mcg_multi_asset_price(const mcg_multi_asset_desc* desc, void* stream, mcg_multi_asset_result* result);

/* ---- Bump-and-revalue on common random numbers ----
 *
 * PricingSource::scenarios / bump_cost and CompiledScenarios::compile /
 * evaluate (crates/pricing/src/engine/risk/bump.rs:362-690): every request
 * moves one input by a half-width h -- the spot (Delta, Gamma) or the
 * Black--Scholes volatility (Vega) -- as an absolute amount or relative to the
 * input's level; requests that move the same input by the same amount share
 * one up/down pair of scenario sides, in first-use order.  Each side is the
 * base plan with that input moved, on the base plan's seeds (the same random
 * coordinates), so the differences are common-random-number differences.  All
 * sides (and the base plan, when a Gamma is requested) are priced in ONE
 * launch: a grid of (tile, scramble, side) CTAs, each staging its side's plan
 * and evaluating a 128-unit tile with the single-plan tile functions.  The
 * estimates pair the sides unit by unit: Delta/Vega the mean of
 * (up_u - down_u) / 2h, Gamma the mean of ((up_u - base_u) + (down_u - base_u)) / h^2,
 * with the standard error of that mean; a unit is a pseudo-random sampling
 * unit (antithetic pairs averaged) or an RQMC scramble's mean over its points.
 * The base plan is single-product, price-only, without discrete dividends. */
typedef enum mcg_bump_measure {
    MCG_BUMP_SPOT_DELTA = 0,
    MCG_BUMP_SPOT_GAMMA = 1,
    MCG_BUMP_VOLATILITY_VEGA = 2  /* Black--Scholes plans */
} mcg_bump_measure;

typedef struct mcg_bump_request {
    int32_t measure;   /* mcg_bump_measure */
    int32_t relative;  /* 1: h = size x the input's level (BumpSize::Relative); 0: h = size */
    double size;       /* positive */
} mcg_bump_request;

typedef struct mcg_bump_estimate {
    int32_t measure;
    uint32_t scenario;       /* the up/down pair used, in first-use order */
    double amount;           /* h */
    double value;
    double standard_error;   /* of the mean of the paired per-unit differences */
    uint64_t units;          /* paired sampling units */
    double up_price, down_price;
} mcg_bump_estimate;

typedef struct mcg_bump_report {
    uint32_t scenarios;
    uint32_t sides;          /* side plans priced by the launch (2 x scenarios, + 1 base for Gamma) */
    uint64_t evaluations;    /* BumpCost::evaluations: 2 x scenarios + 1 when a Gamma is requested */
    mcg_estimate base_price; /* the base plan's price (evaluated when a Gamma is requested) */
    uint64_t path_steps;     /* simulated path-steps of the launch */
    uint32_t kernel_launches;
    float device_ms;
    mcg_error_record error;  /* first failing side: code, the side index in `step`, unit, value */
} mcg_bump_report;

/* `estimates` receives one entry per request; `report` may be NULL. */
mcg_status mcg_bump_evaluate(const mcg_plan_desc* base, const mcg_bump_request* requests, uint32_t request_count,
                             void* stream, mcg_bump_estimate* estimates, mcg_bump_report* report);

/* ---- Pricing without device allocation (no counterpart in the reference) ----
 *
 * For callers that must not allocate GPU memory while pricing (a service that
 * gives the whole device to its own pool at start-up, a host held to a fixed
 * device-memory budget, or a latency-bound caller that cannot take the
 * device-wide synchronisation of cudaFree/cudaMalloc).  Prices one European or
 * Digital Black--Scholes product observed once at expiry, pseudo-MC or RQMC,
 * price-only or full risk, with the same kernels as mcg_plan_evaluate; the
 * kernels' scratch lives in a static device array of MCG_NOALLOC_SCRATCH_BYTES
 * per GPU that loads this library, held until the process exits.  Limits:
 * sampling units x scrambles <= 2^20 and scramble_count <= 64; larger
 * requests return MCG_ERR_INVALID_ARGUMENT.  All calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller.  Every
 * call looks up the array's address on the current device (no address is
 * kept across a device reset); the first call on a device may load the
 * library's device code, so make it before any stream capture.  A call
 * synchronises `stream` before it returns.  The descriptor checks are
 * mcg_plan_create's; a failing sampling unit is reported with its step and
 * value bits as mcg_plan_evaluate reports it.  `result->products` needs one
 * slot; device_ms is not timed; failures are described by mcg_last_error(). */
#define MCG_NOALLOC_SCRATCH_BYTES 5953280u
mcg_status mcg_price_european_noalloc(const mcg_plan_desc* desc, void* stream, mcg_result* result);

/* ---- Diagnostics (no counterpart in the reference) ---- */

/* Dense FP64 FMA throughput of the current device in TFLOP/s (an FMA counts as
 * two flops), measured with independent DFMA chains.  The benchmark uses it as
 * the roofline of the FP64 path kernels. */
mcg_status mcg_measure_fp64_peak(void* stream, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* MCG_H */

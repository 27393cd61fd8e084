// mcg_lsm.cuh -- argument blocks of the early-exercise kernels (mcg_lsm.cu),
// shared with the host orchestration (mcg_host.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mcg_plan.h"

namespace mcg {

// An unevaluated double-double sum hi + lo.
struct DD {
    double hi, lo;
};

struct LsmArgs {
    const double* spots;  // [dates][paths]
    uint64_t paths;
    uint32_t dates;
    uint32_t nb;          // basis columns: max_degree + 1
    int32_t side;
    double strike, notional, itm_tol;
    double abs_tol, rel_tol;
    unsigned long long max_elements;
    const double* df;     // [dates] discount factors of the exercise dates
    double* cf;           // [paths] realised cash flow discounted to time zero
    uint32_t* stop;       // [paths] stopping date
    mcg_lsm_date_model* models;  // [dates - 1]
    double* centers;      // [dates] centre of each date's power sums (a nearby ITM mean)
    DD* partials;         // [CTAs][kLsmPartials]
    unsigned int* tickets;  // [3] per pass kind, zero between launches
    unsigned long long* lsm_error;  // (date << 8) | code of the first failing date, atomicMin
};

struct LsmValueArgs {
    const double* df;
    const mcg_lsm_date_model* models;
    uint32_t dates, nb;
    int32_t side;
    double strike, notional;
    double* unit_values;               // [scrambles * units]: collapsed discounted value
    uint32_t* stops;                   // [paths] or null
    unsigned long long* counts;        // [dates]
    const double* spots;               // stored valuation paths [dates][paths] (local volatility), or
                                       // null: Black--Scholes paths generated in the kernel
    uint64_t paths;
};

struct ErrorWord;

// Fixed-policy risk of the valuation paths (Black--Scholes): the stopping
// date of every path held, the discounted exercise value differentiated.
struct LsmRiskArgs {
    const double* df;        // [dates]
    const uint32_t* stops;   // [paths] valuation stopping dates
    int32_t side;
    double strike, notional;
    int gamma;               // gamma requested: AAD deltas at spot +- gamma_bump
    double gamma_bump, spot_bump, vol_bump;
};

// Andersen--Broadie dual (mcg_dual.cu): the fitted policy, the outer paths'
// states and decisions [date][trajectory], and the continuation estimates of
// the inner rollouts.
struct DualArgs {
    const mcg_lsm_date_model* models;  // [dates - 1]
    uint32_t nb;                       // basis columns: max_degree + 1
    const double* df;                  // [dates]
    const double* sqrt_step;           // [dates]: sqrt(t_j - t_{j-1}), 0 at j = 0
    int32_t side;
    double strike, notional;
    uint64_t trajectories;             // units x lanes
    uint64_t path_stride;              // max(N2, N3)
    uint32_t continuation_inner_paths, exercise_inner_paths;
    uint64_t inner_seed;
    double* spot;                      // [dates][trajectories]
    double* brownian;
    uint8_t* exercise;
    double* continuation;
    unsigned long long* failure;       // first trajectory with a non-finite intermediate
    unsigned long long* inner_count;   // inner paths simulated
};

cudaError_t launch_dual(const DevicePlan& P, const DualArgs& A, StatRecord* partials, cudaStream_t stream,
                        cudaEvent_t nested_begin, cudaEvent_t nested_end, uint32_t& launches);

cudaError_t launch_lsm_bs_spots(const DevicePlan& P, uint32_t domain, double* spots, uint64_t paths,
                                unsigned long long* bad, cudaStream_t stream);
// Local-volatility path store (mcg_lv.cu): date-major spots of every path at
// the exercise dates; the first failing unit in `err`.
cudaError_t launch_lsm_lv_spots(const DevicePlan& P, uint32_t domain, double* spots, uint64_t paths, ErrorWord* err,
                                cudaStream_t stream);
cudaError_t launch_lsm_init(const LsmArgs& A, unsigned ctas, cudaStream_t stream);
cudaError_t launch_lsm_step(const LsmArgs& A, unsigned ctas, int update, int gather, cudaStream_t stream);
cudaError_t launch_lsm_bs_value(const DevicePlan& P, const LsmValueArgs& V, cudaStream_t stream);
cudaError_t launch_lsm_group_sum(const double* values, uint64_t per_group, uint32_t groups, int pairs,
                                 const double* centers, DD* partials, unsigned ctas, DD* out, double* means,
                                 cudaStream_t stream);
// Per-CTA statistics records [scramble][tile][MCG_PATHWISE_COMPONENTS] of the
// fixed-policy risk components; `tiles` = lsm_risk_tiles(units).
cudaError_t launch_lsm_bs_risk(const DevicePlan& P, const LsmRiskArgs& R, StatRecord* partials, cudaStream_t stream);
uint32_t lsm_risk_tiles(uint64_t units);
size_t lsm_partial_stride();

}  // namespace mcg

// mcg_mlp.cuh -- the learned continuation network (2 -> 64 -> 64 -> 1, SiLU)
// of the early-exercise engine: launch interface shared by mcg_mlp.cu and
// the host orchestration (mcg_host.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mcg_lsm.cuh"
#include "mcg_plan.h"

namespace mcg {

constexpr int kMlpHidden = MCG_MLP_HIDDEN;
constexpr int kMlpParams = MCG_MLP_PARAMS;
// Parameter offsets: W1[64][2], b1[64], W2[64][64], b2[64], W3[64], b3.
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + 2 * kMlpHidden;
constexpr int kMlpW2 = kMlpB1 + kMlpHidden;
constexpr int kMlpB2 = kMlpW2 + kMlpHidden * kMlpHidden;
constexpr int kMlpW3 = kMlpB2 + kMlpHidden;
constexpr int kMlpB3 = kMlpW3 + kMlpHidden;
static_assert(kMlpB3 + 1 == kMlpParams, "parameter layout");
// Per-CTA partial record: the gradient sums, then the loss sum and row count.
constexpr int kMlpPartial = kMlpParams + 2;

// Where the rows of one training step come from.
struct MlpRows {
    // early-exercise rows: spots of one date, the paths' discounted cash flows
    const double* spots;
    const double* cf;
    uint64_t first, count;   // path range of this step
    double df, time_input;   // discount factor of the date, scaled time 2 t / T - 1
    int32_t side;
    double strike, notional, itm_tol;
    // explicit rows (gradient checks): inputs x[2 i], x[2 i + 1], targets, masks
    const float* x;
    const float* y;
    const uint8_t* mask;
};

struct MlpDecision {
    const double* spots;     // one date's row
    double* cf;
    uint32_t* stop;
    uint64_t paths;
    uint32_t date;
    double df, time_input;
    int32_t side;
    double strike, notional, itm_tol;
};

cudaError_t launch_mlp_gradient(const float* params, const MlpRows& rows, float* partials, unsigned ctas,
                                cudaStream_t stream);
// A date's `steps` Adam steps over batches of `batch` of its `total` rows
// (batch k mod ceil(total / batch)), one cooperative launch.
cudaError_t launch_mlp_train(float* params, float* moments, float* partials, const MlpRows& rows, uint64_t total,
                             uint64_t batch, uint32_t steps, uint32_t step0, float learning_rate, float* loss_out,
                             cudaStream_t stream);
cudaError_t launch_mlp_adam(const float* partials, unsigned ctas, float* params, float* moments, uint32_t step,
                            float learning_rate, float* loss_out, cudaStream_t stream);
cudaError_t launch_mlp_sum(const float* partials, unsigned ctas, float* out, cudaStream_t stream);
cudaError_t launch_mlp_forward(const float* params, const float* x, uint32_t count, float* out,
                               cudaStream_t stream);
cudaError_t launch_mlp_decide(const float* params, const MlpDecision& D, cudaStream_t stream);
cudaError_t launch_lsm_bs_value_mlp(const DevicePlan& P, const LsmValueArgs& V, const float* params,
                                    double inv_horizon, cudaStream_t stream);
unsigned mlp_gradient_ctas(uint64_t rows);

}  // namespace mcg

// mcg_dual.cu -- Andersen--Broadie dual upper bound of an early-exercise
// price (FP64, compiled with -fmad=false).
//
// AndersenBroadiePlan::evaluate (crates/pricing/src/engine/risk/dual.rs:216-404):
//   1. `dual_outer_kernel`: every outer valuation path (one thread per unit,
//      the antithetic mate in the same thread) at the exercise dates: spot,
//      Brownian value and the fitted policy's decision, as the valuation
//      kernel generates them (path_observations_from_normals,
//      black_scholes.rs:297-331);
//   2. `dual_inner_kernel`: one warp per (outer path, non-terminal exercise
//      date): the rollout_mean of that date (dual.rs:340-400).  Lanes
//      simulate inner paths, each from the outer path's state to its own
//      policy stop; lane 0 adds their discounted payoffs in inner-path order
//      to a Neumaier sum, so the mean is the reference's sequential sum;
//   3. `dual_combine_kernel`: one thread per unit runs DualPath (dual.rs:462-500)
//      over the dates with those continuation estimates and writes the CTA's
//      statistics records of (lower, upper, gap).
// Inner normals are Philox words of the inner seed at counter (inner path,
// dimension / 4, 0x4455414c); a path's four consecutive dimensions share one
// Philox block.
#include "mcg_kernels.cuh"
#include "mcg_lsm.cuh"

namespace mcg {

namespace {

constexpr uint32_t kDualDomain = 0x4455414cu;  // dual.rs:22, INNER_DOMAIN

__device__ __forceinline__ double dual_intrinsic(const DualArgs& A, double s) {
    const double in = A.side == MCG_CALL ? s - A.strike : A.strike - s;
    return (in >= 0.0 ? in : 0.0) * A.notional;
}

// PolynomialRegressionModel::predict (lsm.rs:776-790) of date `d`'s model:
// monomials of the standardised spot by repeated products, summed in basis
// order with a Neumaier sum; ExerciseDecisionModel::should_exercise
// (lsm.rs:805-818): a regression model exercises when the immediate value
// beats it, a continue-all model never does.
__device__ __forceinline__ bool policy_exercises(const DualArgs& A, uint32_t d, double immediate, double x) {
    const mcg_lsm_date_model& m = A.models[d];
    if (!m.regression) return false;
    const double z = m.feature_inactive ? 0.0 : (x - m.feature_mean) / m.feature_scale;
    double sum = 0.0, corr = 0.0, b = 1.0;
    for (uint32_t e = 0; e < A.nb; ++e) {
        if (e) b *= z;
        neumaier_add(sum, corr, b * m.coefficients[e]);
    }
    return immediate > sum + corr;
}

}  // namespace

// Outer paths: spot[d][t], brownian[d][t], exercise[d][t] for trajectory
// t = unit * lanes + lane.
__global__ void __launch_bounds__(kThreads) dual_outer_kernel(const DevicePlan P, DualArgs A) {
    const uint64_t unit = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (unit >= P.units) return;
    NormalSource ns;
    ns.rqmc = false;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = 0;
    ns.dirs = nullptr;
    ns.shift = nullptr;
    ns.cached_block = 0xffffffffu;
    ns.domain = 0;  // Valuation
    const uint32_t n = P.observation_count;
    const int lanes = P.antithetic ? 2 : 1;
    double w[2] = {0.0, 0.0};
    for (uint32_t i = 0; i < n; ++i) {
        const double z = P.zero_variance ? 0.0 : ns.normal(i);
        const double t = P.obs_time[i];
        const double tv = P.vol * P.vol * t;
        for (int e = 0; e < lanes; ++e) {
            const double ze = e == 0 ? z : -z;
            double f, we;
            if (n == 1) {
                we = sqrt(t) * ze;
                f = P.obs_fwd[0] * 1.0 * exp(-0.5 * tv + sqrt(tv) * ze);
            } else {
                w[e] += P.obs_sqrt_step[i] * ze;
                we = w[e];
                f = P.obs_fwd[i] * 1.0 * exp(-0.5 * tv + P.vol * we);
            }
            const uint64_t t_index = unit * lanes + e;
            const size_t at = static_cast<size_t>(i) * A.trajectories + t_index;
            A.spot[at] = f;
            A.brownian[at] = we;
            A.exercise[at] = (i + 1 == n || policy_exercises(A, i, dual_intrinsic(A, f), f)) ? 1 : 0;
        }
    }
}

// rollout_mean of (trajectory, branch date): one warp each, four per CTA;
// tasks [first_task, first_task + tasks) of trajectory x (dates - 1).  Inner
// paths go in chunks of 32 x kDualSlots: in one loop each lane advances its
// current path by one date per iteration and takes its next path of the chunk
// as soon as one stops (so a lane never waits for a slower lane's path), the
// discounted payoffs land in shared memory by inner index, and lane 0 adds
// the chunk to the Neumaier sum in that order.
constexpr int kDualSlots = 8;

__global__ void __launch_bounds__(kThreads) dual_inner_kernel(const DevicePlan P, DualArgs A, uint64_t first_task,
                                                              uint64_t tasks) {
    __shared__ double s_values[kThreads / 32][32 * kDualSlots];
    const uint64_t task = first_task + static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (task >= first_task + tasks) return;  // whole warps leave together
    double* values = s_values[threadIdx.x / 32];
    const uint32_t dates = P.observation_count;
    const uint32_t branches = dates - 1;
    const uint64_t trajectory = task / branches;
    const uint32_t d = static_cast<uint32_t>(task % branches);
    const size_t at = static_cast<size_t>(d) * A.trajectories + trajectory;
    const bool exercise = A.exercise[at] != 0;
    const uint32_t configured = exercise ? A.exercise_inner_paths : A.continuation_inner_paths;
    const uint32_t paths = P.vol == 0.0 ? 1u : configured;
    const double w0 = A.brownian[at];
    double sum = 0.0, corr = 0.0;  // lane 0's sequential Neumaier sum
    bool bad = false;
    for (uint32_t c0 = 0; c0 < paths; c0 += 32u * kDualSlots) {
        int slot = 0;
        uint32_t inner = c0 + static_cast<uint32_t>(lane);
        bool active = inner < paths;
        double w = w0;
        uint32_t j = d + 1;
        uint32_t cached = 0xffffffffu;
        uint4 block = make_uint4(0u, 0u, 0u, 0u);
        while (__any_sync(0xffffffffu, active)) {
            if (!active) continue;
            const uint64_t path = trajectory * A.path_stride + inner;
            double z = 0.0;
            if (P.vol != 0.0) {
                const uint32_t dim = d * dates + j;
                if ((dim >> 2) != cached) {
                    cached = dim >> 2;
                    block = philox_block(A.inner_seed, path, cached, kDualDomain);
                }
                z = as241(open_unit(lane_of(block, dim & 3u)));
            }
            w += A.sqrt_step[j] * z;
            const double variance = P.vol * P.vol * P.obs_time[j];
            const double canonical = P.obs_fwd[j] * exp(-0.5 * variance + P.vol * w);
            const double s = 0.0 * P.spot + 1.0 * canonical;
            if (!isfinite(s)) bad = true;
            const double imm = dual_intrinsic(A, s);
            if (j + 1 == dates || policy_exercises(A, j, imm, s)) {
                values[lane + 32 * slot] = imm * A.df[j];
                ++slot;
                inner += 32;
                active = slot < kDualSlots && inner < paths;
                w = w0;
                j = d + 1;
                cached = 0xffffffffu;
            } else {
                ++j;
            }
        }
        __syncwarp();
        if (lane == 0) {
            const uint32_t count = paths - c0 < 32u * kDualSlots ? paths - c0 : 32u * kDualSlots;
            for (uint32_t i = 0; i < count; ++i) neumaier_add(sum, corr, values[i]);
        }
        __syncwarp();
    }
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
        const double mean = (sum + corr) / static_cast<double>(paths);
        A.continuation[at] = mean;
        if (bad || !isfinite(mean)) atomicMin(A.failure, static_cast<unsigned long long>(trajectory));
    }
}

// DualPath over the dates per trajectory; (lower, upper, gap) per unit, the
// antithetic pair as 0.5 primary + 0.5 mate (dual.rs:247-262); CTA records at
// partials[tile * 3 + c].
__global__ void __launch_bounds__(kThreads) dual_combine_kernel(const DevicePlan P, DualArgs A,
                                                                StatRecord* partials) {
    __shared__ Stat s_red[4 * 3];
    const uint64_t unit = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool valid = unit < P.units;
    const uint32_t dates = P.observation_count;
    const int lanes = P.antithetic ? 2 : 1;
    double out[3] = {0.0, 0.0, 0.0};
    bool bad = false;
    unsigned long long inner = 0;
    if (valid) {
        double res[2][3];
        for (int e = 0; e < lanes; ++e) {
            const uint64_t trajectory = unit * lanes + e;
            double lower = 0.0;
            bool have_lower = false;
            double c_sum = 0.0, c_corr = 0.0;  // the correction's Neumaier sum
            double gap = -INFINITY;
            for (uint32_t d = 0; d < dates; ++d) {
                const size_t at = static_cast<size_t>(d) * A.trajectories + trajectory;
                const bool terminal = d + 1 == dates;
                const bool exercise = A.exercise[at] != 0;
                const double discounted = dual_intrinsic(A, A.spot[at]) * A.df[d];
                if (exercise && !have_lower) {
                    lower = discounted;
                    have_lower = true;
                }
                const double continuation = terminal ? 0.0 : A.continuation[at];
                if (!terminal)
                    inner += P.vol == 0.0 ? 1u : (exercise ? A.exercise_inner_paths : A.continuation_inner_paths);
                const double value = exercise ? discounted : continuation;
                const double candidate = (discounted - value) - (c_sum + c_corr);
                if (!isfinite(candidate)) bad = true;
                gap = fmax(gap, candidate);
                if (exercise && !terminal) neumaier_add(c_sum, c_corr, discounted - continuation);
            }
            res[e][0] = lower;
            res[e][1] = lower + gap;
            res[e][2] = gap;
            if (!isfinite(res[e][1])) bad = true;
        }
        for (int c = 0; c < 3; ++c) out[c] = lanes == 2 ? 0.5 * res[0][c] + 0.5 * res[1][c] : res[0][c];
        if (bad) atomicMin(A.failure, static_cast<unsigned long long>(unit * lanes));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) inner += __shfl_down_sync(0xffffffffu, inner, off);
    if ((threadIdx.x & 31) == 0 && inner) atomicAdd(A.inner_count, inner);
    cta_reduce_write<3>(out, valid, 0x7u, partials + static_cast<size_t>(blockIdx.x) * 3, s_red);
}

cudaError_t launch_dual(const DevicePlan& P, const DualArgs& A, StatRecord* partials, cudaStream_t stream,
                        cudaEvent_t nested_begin, cudaEvent_t nested_end, uint32_t& launches) {
    const unsigned tiles = static_cast<unsigned>((P.units + kThreads - 1) / kThreads);
    dual_outer_kernel<<<tiles, kThreads, 0, stream>>>(P, A);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ++launches;
    cudaEventRecord(nested_begin, stream);
    const uint64_t tasks = A.trajectories * (P.observation_count - 1);
    constexpr uint64_t kWarps = kThreads / 32;
    constexpr uint64_t kMaxCtas = 1u << 30;
    for (uint64_t first = 0; first < tasks; first += kMaxCtas * kWarps) {
        const uint64_t n = tasks - first < kMaxCtas * kWarps ? tasks - first : kMaxCtas * kWarps;
        dual_inner_kernel<<<static_cast<unsigned>((n + kWarps - 1) / kWarps), kThreads, 0, stream>>>(P, A, first, n);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ++launches;
    }
    cudaEventRecord(nested_end, stream);
    dual_combine_kernel<<<tiles, kThreads, 0, stream>>>(P, A, partials);
    ++launches;
    return cudaGetLastError();
}

}  // namespace mcg

// mcg_noalloc.cu -- European/Digital Black--Scholes pricing without any
// device allocation.
//
// Some callers cannot allocate GPU memory when they price: a service that
// hands the whole device to its own memory pool at start-up and treats any
// later allocation as a failure, a host held to a fixed device-memory budget,
// or a latency-bound caller that cannot afford the device-wide
// synchronisation cudaFree (and, when the heap grows, cudaMalloc) imposes on
// every other stream.  For them this file keeps the path kernel's scratch -- per-CTA statistics
// records, the reduced records, the error word and the small plan constants --
// in one file-scope static device array of a fixed size, so a call makes no
// cudaMalloc/cudaFree and no allocating library call.  The kernels are the
// same single-terminal path kernel and tile reduction that mcg_plan_evaluate
// launches; only where their scratch lives differs.
//
// Limits: one product (European or Digital) observed once at expiry; at most
// kMaxTiles CTA tiles of 128 units in total (pseudo: 2^20 units; RQMC:
// points x scrambles <= 2^20) and at most kMaxScrambles scrambles.  The array
// is resident on every GPU that loads the library until the process exits.
// Every call reuses the same array, so calls that overlap on the GPU (two
// streams, or two host threads on one device) race and must be serialised by
// the caller.  Every call resolves the array's device address on the current
// device (cudaGetSymbolAddress, which allocates nothing), so no address is
// kept across a device reset; the first call on a device may load this
// library's device code (CUDA's lazy module loading), so make that first call
// before any stream capture.  A call synchronises its stream before it
// returns.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mcg_kernels.cuh"

namespace mcg {
cudaError_t launch_bs_path(const DevicePlan& P, bool single_terminal, uint64_t unit_begin, uint64_t units,
                           uint32_t scrambles, StatRecord* partials, uint32_t mask, ErrorWord* err,
                           int detail, cudaStream_t stream);
__global__ void scramble_table_kernel(const uint32_t*, uint32_t, uint32_t, uint32_t, uint64_t, uint32_t*,
                                      uint32_t*);
__global__ void reduce_tiles_kernel(const StatRecord*, uint32_t, uint32_t, StatRecord*);
void set_last_error(const std::string& message);
}  // namespace mcg

using namespace mcg;

namespace {

constexpr uint32_t kMaxTiles = 8192;     // 2^20 units of 128-thread tiles
constexpr uint32_t kMaxScrambles = 64;
constexpr size_t kPartialBytes = static_cast<size_t>(kMaxTiles) * kComponents * sizeof(StatRecord);
constexpr size_t kRecordBytes = static_cast<size_t>(kMaxScrambles) * kComponents * sizeof(StatRecord);
constexpr size_t kErrorOffset = kPartialBytes + kRecordBytes;
constexpr size_t kConstOffset = kErrorOffset + 256;
// constants: observation forward/time/sqrt-step (3 doubles), 32 direction
// words, the scramble table (kMaxScrambles x 32 words) and shifts.
constexpr size_t kConstBytes = 3 * sizeof(double) + 32 * 4 + kMaxScrambles * 32 * 4 + kMaxScrambles * 4;
constexpr size_t kScratchBytes = ((kConstOffset + kConstBytes + 255) / 256) * 256;

static_assert(kScratchBytes == MCG_NOALLOC_SCRATCH_BYTES, "mcg.h states the scratch size");

}  // namespace

// The scratch of every no-allocation call on this device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

mcg_status noalloc_fail(mcg_status code, const std::string& why) {
    set_last_error(why);
    return code;
}

// Device address of g_noalloc_scratch on the current device.  Resolved on
// every call: the lookup allocates nothing, and a cached address would go
// stale if the device were reset and the module loaded again.
mcg_status scratch_for_current_device(unsigned char** out) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
        return noalloc_fail(MCG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = static_cast<unsigned char*>(ptr);
    return MCG_OK;
}

int64_t key_of(double x) {
    int64_t b;
    std::memcpy(&b, &x, 8);
    return b ^ static_cast<int64_t>(static_cast<uint64_t>(b >> 63) >> 1);
}

// Log-linear discount curve value at `time` (crates/pricing/src/market/curve.rs:156-205).
bool log_discount(const mcg_curve& c, double time, double& out) {
    if (c.pillar_count < 2 || !c.times || !c.discount_factors || c.times[0] != 0.0 ||
        c.discount_factors[0] != 1.0)
        return false;
    for (uint32_t i = 0; i < c.pillar_count; ++i)
        if (!std::isfinite(c.times[i]) || !std::isfinite(c.discount_factors[i]) || !(c.discount_factors[i] > 0.0) ||
            (i && !(c.times[i] > c.times[i - 1])))
            return false;
    if (time == 0.0) time = 0.0;
    const int64_t key = key_of(time);
    uint32_t lo = 0, hi = c.pillar_count;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (key_of(c.times[mid]) < key) lo = mid + 1; else hi = mid;
    }
    if (lo < c.pillar_count && key_of(c.times[lo]) == key) {
        out = std::log(c.discount_factors[lo]);
        return true;
    }
    const uint32_t right = lo < c.pillar_count ? lo : c.pillar_count - 1;
    const uint32_t left = right - 1;
    const double l = std::log(c.discount_factors[left]), r = std::log(c.discount_factors[right]);
    const double w = (time - (left == 0 ? 0.0 : c.times[left])) / (c.times[right] - (left == 0 ? 0.0 : c.times[left]));
    out = l + w * (r - l);
    return true;
}

void neumaier(double& s, double& c, double v) {
    const double u = s + v;
    if (std::fabs(s) >= std::fabs(v)) c += (s - u) + v;
    else c += (v - u) + s;
    s = u;
}

mcg_estimate estimate(const mcg_statistics& s, uint64_t units) {
    const double inv = 1.0 / static_cast<double>(units);
    const double value = (s.sum + s.correction) * inv;
    const double var = s.count > 1 ? s.second_moment / static_cast<double>(s.count - 1) : 0.0;
    const double se = std::sqrt(var * inv);
    const double hw = 1.959963984540054 * se;
    return {value, se, value - hw, value + hw, units};
}

}  // namespace

extern "C" mcg_status mcg_price_european_noalloc(const mcg_plan_desc* d, void* stream_handle,
                                                 mcg_result* result) {
    if (!d || !result || !result->products || result->product_capacity < 1)
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "null descriptor or result without a product slot");
    if (d->abi_version != MCG_ABI_VERSION) return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "abi_version mismatch");
    if (d->model != MCG_MODEL_BLACK_SCHOLES || d->precision != MCG_PRECISION_F64)
        return noalloc_fail(MCG_ERR_UNSUPPORTED, "the no-allocation entry point prices FP64 Black-Scholes only");
    if (d->product_count != 1 || !d->products ||
        (d->products[0].kind != MCG_PRODUCT_EUROPEAN && d->products[0].kind != MCG_PRODUCT_DIGITAL))
        return noalloc_fail(MCG_ERR_UNSUPPORTED, "the no-allocation entry point prices one European or Digital");
    if (d->observation_count != 1 || !d->observation_times || !(d->observation_times[0] > 0.0) ||
        !std::isfinite(d->observation_times[0]))
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "one positive expiry observation is required");
    if (!(d->spot > 0.0) || !std::isfinite(d->spot) || !(d->volatility >= 0.0) || !std::isfinite(d->volatility))
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "spot and volatility");
    const mcg_product_desc& pd = d->products[0];
    if (!(pd.notional > 0.0) || !(pd.strike > 0.0) || !std::isfinite(pd.strike))
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "product strike/notional must be positive");
    if (pd.has_initial_state)  // as mcg_plan_create: a terminal product has no observation history
        return noalloc_fail(MCG_ERR_UNSUPPORTED, "seasoned state of a product without observation history");
    if (d->discrete_dividends.count)
        return noalloc_fail(MCG_ERR_UNSUPPORTED, "the no-allocation entry point prices without discrete dividends");
    if (!(d->smoothing_half_width >= 0.0) || !std::isfinite(d->smoothing_half_width))
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "smoothing_half_width");
    const bool rqmc = d->engine == MCG_ENGINE_RQMC;
    if (!rqmc && d->engine != MCG_ENGINE_PSEUDO) return noalloc_fail(MCG_ERR_UNSUPPORTED, "engine");
    const uint64_t units = d->sampling_units;
    const uint32_t scrambles = rqmc ? d->scramble_count : 1;
    if (units == 0 || scrambles == 0) return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "sampling_units/scramble_count");
    if (rqmc && (units & (units - 1)) != 0)
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "points_per_scramble must be a power of two");
    const uint64_t tiles = (units + kThreads - 1) / kThreads;
    if (scrambles > kMaxScrambles)
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT,
                            "scramble_count " + std::to_string(scrambles) + " exceeds the no-allocation limit 64");
    if (tiles * scrambles > kMaxTiles)
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT,
                            "sampling units x scrambles exceed the no-allocation limit of 2^20 (" +
                                std::to_string(units) + " x " + std::to_string(scrambles) + ")");
    if (rqmc && (!d->sobol_directions || d->sobol_dimension_count < 1))
        return noalloc_fail(MCG_ERR_SOBOL_DIMENSION, "sobol_directions");
    const double expiry = d->observation_times[0];
    double lr, lq, lp;
    if (!log_discount(d->discount_curve, expiry, lr) || !log_discount(d->dividend_curve, expiry, lq) ||
        !log_discount(d->discount_curve, d->payment_time, lp))
        return noalloc_fail(MCG_ERR_MARKET, "discount or dividend curve");
    const bool risk = d->request_delta || d->request_gamma || d->request_vega;
    const double gamma_bump = d->gamma_bump_relative ? d->spot * d->gamma_bump : d->gamma_bump;
    if (d->request_gamma && (!std::isfinite(gamma_bump) || gamma_bump <= 0.0 || gamma_bump >= d->spot))
        return noalloc_fail(MCG_ERR_INVALID_ARGUMENT, "gamma bump must be positive and below spot");

    unsigned char* scratch = nullptr;
    mcg_status st = scratch_for_current_device(&scratch);
    if (st != MCG_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    StatRecord* partials = reinterpret_cast<StatRecord*>(scratch);
    StatRecord* records = reinterpret_cast<StatRecord*>(scratch + kPartialBytes);
    ErrorWord* error = reinterpret_cast<ErrorWord*>(scratch + kErrorOffset);
    double* consts = reinterpret_cast<double*>(scratch + kConstOffset);
    uint32_t* directions = reinterpret_cast<uint32_t*>(consts + 3);
    uint32_t* table = directions + 32;
    uint32_t* shifts = table + kMaxScrambles * 32;

    // Plan constants (3 doubles) and the error word: the only state that must
    // start from known values; partials and records are fully rewritten.
    const double host_consts[3] = {d->spot * std::exp(lq - lr), expiry, std::sqrt(expiry)};
    const ErrorWord clear{~0ull, 0, 0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(consts, host_consts, sizeof(host_consts), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(error, &clear, sizeof(clear), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && rqmc) {
        e = cudaMemcpyAsync(directions, d->sobol_directions, 32 * sizeof(uint32_t), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) {
            scramble_table_kernel<<<(scrambles + 127) / 128, 128, 0, stream>>>(directions, 1, scrambles,
                                                                              d->scramble_begin, d->master_seed,
                                                                              table, shifts);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess) return noalloc_fail(MCG_ERR_CUDA, cudaGetErrorString(e));

    DevicePlan P{};
    P.model = MCG_MODEL_BLACK_SCHOLES;
    P.engine = d->engine;
    P.precision = MCG_PRECISION_F64;
    P.antithetic = d->antithetic != 0;
    P.seed = d->master_seed;
    P.units = units;
    P.scramble_count = scrambles;
    P.steps = 1;
    P.observation_count = 1;
    P.product_count = 1;
    P.dimension = 1;
    P.obs_fwd = consts;
    P.obs_time = consts + 1;
    P.obs_sqrt_step = consts + 2;
    P.spot = d->spot;
    P.vol = d->volatility;
    P.expiry = expiry;
    P.discount = std::exp(lp);
    P.zero_variance = d->volatility * d->volatility * expiry == 0.0;
    P.scr_dirs = rqmc ? table : nullptr;
    P.scr_shift = rqmc ? shifts : nullptr;
    P.risk = risk;
    P.req_gamma = d->request_gamma != 0;
    P.gamma_bump = gamma_bump;
    P.spot_bump = d->request_gamma ? gamma_bump : std::min(d->spot * 1.0e-4, 0.5 * d->spot);
    P.vol_bump = d->volatility == 0.0 ? 0.0 : std::min(1.0e-4, d->volatility * 0.5);
    P.spot_variant[0] = d->spot;
    P.spot_variant[1] = d->spot - P.spot_bump;
    P.spot_variant[2] = d->spot + P.spot_bump;
    P.smoothing = d->smoothing_half_width;
    ProductParams& q = P.products[0];
    q.kind = pd.kind;
    q.side = pd.side;
    q.strike = pd.strike;
    q.notional = pd.notional;
    q.digital_payout = pd.digital_payout;
    q.payout = pd.payout;
    const uint32_t mask = risk ? 0x3ffu : 1u;

    e = launch_bs_path(P, true, 0, units, scrambles, partials, mask, error, 0, stream);
    if (e == cudaSuccess) {
        reduce_tiles_kernel<<<dim3(kComponents, scrambles), 256, 0, stream>>>(partials, static_cast<uint32_t>(tiles),
                                                                             kComponents, records);
        e = cudaGetLastError();
    }
    StatRecord host[kMaxScrambles * kComponents];
    ErrorWord ew{};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host, records, static_cast<size_t>(scrambles) * kComponents * sizeof(StatRecord),
                            cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ew, error, sizeof(ew), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return noalloc_fail(MCG_ERR_CUDA, cudaGetErrorString(e));
    std::memset(&result->error, 0, sizeof(result->error));
    result->kernel_launches = 2 + (rqmc ? 1 : 0);
    result->device_ms = 0.0f;
    result->path_kernel_ms = 0.0f;
    if (ew.key != ~0ull) {
        // Re-run the first failing unit alone to recover its step and value
        // bits, as mcg_plan_evaluate does.
        const uint64_t unit = ew.key >> 8;
        e = cudaMemcpyAsync(error, &clear, sizeof(clear), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = launch_bs_path(P, true, unit, 1, scrambles, partials, mask, error, 1, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&ew, error, sizeof(ew), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return noalloc_fail(MCG_ERR_CUDA, cudaGetErrorString(e));
        result->error.code = static_cast<int32_t>(ew.key & 0xff);
        result->error.sampling_unit = ew.key >> 8;
        result->error.step = ew.step;
        result->error.value_bits = ew.value_bits;
        return noalloc_fail(static_cast<mcg_status>(result->error.code),
                            "sampling unit " + std::to_string(result->error.sampling_unit) + " failed");
    }
    const uint64_t independent = rqmc ? scrambles : units;
    const double total_variance = d->volatility * d->volatility * expiry;
    if (total_variance > 0.0 && independent < 2)
        return noalloc_fail(MCG_ERR_INSUFFICIENT_UNITS, "at least two independent sampling units are required");
    result->independent_sampling_units = independent;
    result->evaluated_paths = units * scrambles * (d->antithetic ? 2 : 1);
    result->time_steps = 1;
    result->effective_dimension = 1;
    result->reduction_records = static_cast<uint32_t>(tiles * scrambles);
    mcg_product_result& r = result->products[0];
    for (int c = 0; c < kComponents; ++c) {
        mcg_statistics s{0.0, 0.0, 0, 0.0, 0.0};
        const bool active = mask & (1u << c);
        if (!rqmc) {
            if (active) {
                const StatRecord& x = host[c];
                s = {x.sum, x.corr, static_cast<uint64_t>(x.count), x.mean, x.m2};
            } else {
                s.count = units;
            }
        } else {
            // per-scramble means, then the two-pass moments over scrambles
            double reps[kMaxScrambles];
            for (uint32_t k = 0; k < scrambles; ++k)
                reps[k] = active ? (host[k * kComponents + c].sum + host[k * kComponents + c].corr) /
                                       static_cast<double>(units)
                                 : 0.0;
            double sum = 0.0, corr = 0.0;
            for (uint32_t k = 0; k < scrambles; ++k) neumaier(sum, corr, reps[k]);
            const double mean = (sum + corr) / static_cast<double>(scrambles);
            double qs = 0.0, qc = 0.0;
            for (uint32_t k = 0; k < scrambles; ++k) {
                const double dv = reps[k] - mean;
                neumaier(qs, qc, dv * dv);
            }
            s = {sum, corr, scrambles, mean, qs + qc};
        }
        r.components[c] = s;
    }
    r.price = estimate(r.components[MCG_PRICE], independent);
    r.delta = estimate(r.components[MCG_DELTA], independent);
    r.gamma = estimate(r.components[MCG_GAMMA], independent);
    r.vega = estimate(r.components[MCG_VEGA], independent);
    r.bump_delta = estimate(r.components[MCG_BUMP_DELTA], independent);
    r.bump_gamma = estimate(r.components[MCG_BUMP_GAMMA], independent);
    r.bump_vega = estimate(r.components[MCG_BUMP_VEGA], independent);
    const mcg_statistics& ps = r.components[MCG_PRICE];
    const double sv = ps.count > 1 ? ps.second_moment / static_cast<double>(ps.count - 1) : 0.0;
    r.sampling_variance = total_variance == 0.0 ? 0.0 : sv;
    r.estimator_variance = r.sampling_variance / static_cast<double>(independent);
    return MCG_OK;
}

// mcg_lv32.cu -- local-volatility path kernel with an FP32 path bulk.
//
// The plan's precision MCG_PRECISION_F32_BULK: normals, Brownian-bridge
// nodes and the Log-Euler state evolve in single precision, the way the
// FP64 kernel (mcg_lv_tile.cuh) evolves them in double,
//   x = ln(f / F_i),  v = bilinear(t_i, x),  f <- f * (F_{i+1}/F_i) * exp(-v dt/2 + sqrt(v) sqrt(dt) z)
// (crates/pricing/src/engine/processes/local_vol.rs:459-619), with the
// grid staged as FP32 in shared memory and the logarithm and exponential on
// the special-function unit (the logarithm feeds only the grid lookup).  Observed spots are widened to FP64 for the
// payoff accumulators, the barrier bridge and the statistics, which stay as
// in the FP64 path.  Normals come from the same Philox / scrambled-Sobol
// words: the AS241 quantile runs in FP32 with the tail taken from the word
// itself (no rounding of the uniform to 1).  The error against the FP64 path
// is a property of each result; the tests and the benchmark state it.
// No counterpart in the reference (its path arithmetic is FP64 only).
#include "mcg_kernels.cuh"

namespace mcg {
namespace {

constexpr float kTwoM32 = 2.3283064365386963e-10f;

// AS241 in FP32 from the 32-bit word: the centred value (w - 2^31 + 0.5) 2^-32
// and the tail probability min(p, 1 - p) are formed from the integer, so the
// tail never rounds to zero.  Coefficients are Wichura's published ones.  The
// two branches are separate functions so a warp can take the central one for
// every lane and the tail one only for the lanes that need it.
__device__ __forceinline__ float normal32_centered(uint32_t w) {
    return (static_cast<float>(static_cast<int32_t>(w - 0x80000000u)) + 0.5f) * kTwoM32;
}

__device__ __forceinline__ bool normal32_is_tail(float centered) { return !(fabsf(centered) <= 0.425f); }

__device__ __forceinline__ float normal32_central(float centered) {
    const float a = 0.180625f - centered * centered;
    const float num =
        ((((((2509.0809287301227f * a + 33430.575583588128f) * a + 67265.770927008700f) * a +
             45921.953931549871f) * a + 13731.693765509461f) * a + 1971.5909503065514f) * a +
         133.14166789178438f) * a + 3.3871328727963666f;
    const float den =
        ((((((5226.4952788528545f * a + 28729.085735721943f) * a + 39307.895800092710f) * a +
             21213.794301586596f) * a + 5394.1960214247511f) * a + 687.18700749205790f) * a +
         42.313330701600911f) * a + 1.0f;
    return centered * __fdividef(num, den);
}

__device__ __forceinline__ float normal32_tail(uint32_t w, float centered) {
    const uint32_t k = centered < 0.0f ? w : 0xffffffffu - w;
    const float tail = (static_cast<float>(k) + 0.5f) * kTwoM32;
    const float r = sqrtf(-__logf(tail));
    float m;
    if (r <= 5.0f) {
        const float a = r - 1.6f;
        m = ((((((7.74545014278341407640e-4f * a + 2.27238449892691845833e-2f) * a +
                 2.41780725177450611770e-1f) * a + 1.27045825245236838258f) * a +
               3.64784832476320460504f) * a + 5.76949722146069140550f) * a +
             4.63033784615654529590f) * a + 1.42343711074968357734f;
        m = __fdividef(m, ((((((1.05075007164441684324e-9f * a + 5.47593808499534494600e-4f) * a +
                               1.51986665636164571966e-2f) * a + 1.48103976427480074590e-1f) * a +
                             6.89767334985100004550e-1f) * a + 1.67638483018380384940f) * a +
                           2.05319162663775882187f) * a + 1.0f);
    } else {
        const float a = r - 5.0f;
        m = ((((((2.01033439929228813265e-7f * a + 2.71155556874348757815e-5f) * a +
                 1.24266094738807843860e-3f) * a + 2.65321895265761230930e-2f) * a +
               2.96560571828504891230e-1f) * a + 1.78482653991729133580f) * a +
             5.46378491116411436990f) * a + 6.65790464350110377720f;
        m = __fdividef(m, ((((((2.04426310338993978564e-15f * a + 1.42151175831644588870e-7f) * a +
                               1.84631831751005468180e-5f) * a + 7.86869131145613259100e-4f) * a +
                             1.48753612908506148525e-2f) * a + 1.36929880922735805310e-1f) * a +
                           5.99832206555887937690e-1f) * a + 1.0f);
    }
    return centered < 0.0f ? -m : m;
}

// Batched normals, as in the FP64 kernel: kZBatch32 normals of the program per
// thread at a time, in s_z[k][thread] (a float's bits, or the word while its
// tail value is pending).  Every lane takes the central branch; the lanes in
// the tail are listed per warp (s_zlist, 32 * kZBatch32 entries) and the tail
// branch runs 32 list entries at a time, so a warp no longer executes it for
// each normal that one of its lanes sends there.  The values are those of the
// one-at-a-time quantile.
constexpr int kZBatch32 = 8;

template <typename Word>
__device__ __forceinline__ void fill_normals32(const DevicePlan& P, Word word, uint32_t first, uint32_t count,
                                               uint32_t* s_z, uint16_t* s_zlist) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    uint16_t* list = s_zlist + warp * (32u * kZBatch32);
    uint32_t tails = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t w = word(__ldg(P.z_ranks + first + k));
        const float c = normal32_centered(w);
        const bool tail = normal32_is_tail(c);
        const float central = normal32_central(c);
        s_z[k * kThreads + threadIdx.x] = tail ? w : __float_as_uint(central);
        const unsigned m = __ballot_sync(0xffffffffu, tail);
        if (tail) list[tails + __popc(m & ((1u << lane) - 1u))] = static_cast<uint16_t>(k * 32u + lane);
        tails += static_cast<uint32_t>(__popc(m));
    }
    __syncwarp();
    for (uint32_t b = 0; b < tails; b += 32u) {
        const uint32_t i = b + lane;
        if (i < tails) {
            const uint32_t idx = list[i];
            uint32_t* at = s_z + (idx >> 5) * kThreads + warp * 32u + (idx & 31u);
            const uint32_t w = *at;
            *at = __float_as_uint(normal32_tail(w, normal32_centered(w)));
        }
    }
    __syncwarp();
}

// Bilinear local variance on the FP32 grid, x clamped flat to the node range
// (LocalVarianceGrid::interpolate, crates/pricing/src/market/local_variance.rs:273-414);
// the cell is walked from the previous one.
__device__ __forceinline__ float interp_f32(const float* v, const float* xs, int nx, int tc, float tw, float xq,
                                            int& hint) {
    const float xv = fminf(fmaxf(xq, xs[0]), xs[nx - 1]);
    int c = min(hint, nx - 2);
    while (c > 0 && xs[c] > xv) --c;
    while (c < nx - 2 && xs[c + 1] <= xv) ++c;
    hint = c;
    const float xw = (xv - xs[c]) / (xs[c + 1] - xs[c]);
    const float* row = v + tc * nx;
    const float* next = row + nx;
    const float lower = row[c] + (row[c + 1] - row[c]) * xw;
    const float upper = next[c] + (next[c + 1] - next[c]) * xw;
    return lower + (upper - lower) * tw;
}

// RQ / CB specialise on the engine and on "any continuous barrier", as the
// FP64 kernel does; one evolution runs 8 CTAs of 128 threads per SM.
template <int E, int NP, int RQ, int CB>
__global__ void __launch_bounds__(kThreads, (E == 1 && NP <= 2 && CB == 0) ? 8 : 1)
    lv32_path_kernel(const DevicePlan P, StatRecord* partials, uint32_t mask, ErrorWord* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = static_cast<int>(P.nx);
    const int nv = static_cast<int>(P.nt * P.nx);
    float* s_v = reinterpret_cast<float*>(smem_raw);
    float* s_x = s_v + nv;
    float* s_w = s_x + ((nx + 3) & ~3);  // bridge slots [slot][thread]
    Stat* s_red = reinterpret_cast<Stat*>(s_w + static_cast<size_t>(P.slot_count) * kThreads);
    uint32_t* s_z = reinterpret_cast<uint32_t*>(s_red + 4 * kComponents);  // batched normals [k][thread]
    uint16_t* s_zlist = reinterpret_cast<uint16_t*>(s_z + kZBatch32 * kThreads);  // tail lists, per warp
    for (int i = threadIdx.x; i < nv; i += kThreads) s_v[i] = static_cast<float>(P.grid_v[i]);
    for (int i = threadIdx.x; i < nx; i += kThreads) s_x[i] = static_cast<float>(P.grid_x[i]);
    __syncthreads();

    const uint32_t scramble = blockIdx.y;
    const uint64_t point = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < P.units;
    const uint64_t unit = valid ? point : 0;
    NormalSource ns;
    ns.rqmc = RQ != 0;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    // warp-cooperative Sobol words (the launch's points are 32-aligned per warp)
    if (RQ) {
        const uint32_t q = static_cast<uint32_t>(point) & ~31u;
        ns.high_gray = q ^ (q >> 1);
        ns.lane_low = static_cast<uint32_t>(point) & 31u;
        ns.low = P.scr_low + static_cast<size_t>(scramble) * P.dimension * 32u;
    }
    auto word = [&](uint32_t dim) { return RQ ? ns.word_warp(dim) : ns.word(dim); };
    // The program's normals in order, kZBatch32 at a time.
    uint32_t zi = 0, zbase = 0, zend = 0;
    auto next_normal = [&]() -> float {
        if (zi == zend) {
            zbase = zi;
            const uint32_t n = P.z_count - zi < static_cast<uint32_t>(kZBatch32) ? P.z_count - zi
                                                                                : static_cast<uint32_t>(kZBatch32);
            fill_normals32(P, word, zi, n, s_z, s_zlist);
            zend = zi + n;
        }
        return __uint_as_float(s_z[(zi++ - zbase) * kThreads + threadIdx.x]);
    };

    // The state is the forward-normalised spot g = f / F_i, a martingale
    // (f_{i+1} / F_{i+1} = (f_i / F_i) exp(-v dt / 2 + sqrt(v dt) z)): no FP32
    // forward ratio is multiplied in at every step, so the ratio's rounding
    // cannot compound into a drift; the spot f = g F_i is formed in FP64 when
    // a payoff or the barrier bridge observes it.
    float f[E], prev_f[E], prev_v[E];
    int hint[E];
    ProductAcc acc[E][NP];
    bool failed = false;
    bool bad_state = false;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        f[e] = static_cast<float>(P.spot / P.fwd[0]);
        prev_f[e] = f[e];
        prev_v[e] = 0.0f;
        hint[e] = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            acc_init(acc[e][k], P.products[k]);
            if (CB && k < static_cast<int>(P.product_count) && P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                barrier_begin(P.products[k], acc[e][k], P.smoothing, P.spot, failed);
        }
    }
    float* w = s_w + threadIdx.x;
    const uint32_t steps = P.steps;
    for (uint32_t oi = 0; oi < P.op_count; ++oi) {
        const Op op = P.ops[oi];
        if (op.kind == kOpZero) {
            w[op.out * kThreads] = 0.0f;
            continue;
        }
        if (op.kind == kOpTerminal) {
            w[op.out * kThreads] = static_cast<float>(op.sd) * next_normal();
            continue;
        }
        if (op.kind == kOpInterior) {
            const float z = next_normal();
            w[op.out * kThreads] = static_cast<float>(op.wl) * w[op.left * kThreads] +
                                   static_cast<float>(op.wr) * w[op.right * kThreads] + static_cast<float>(op.sd) * z;
            continue;
        }
        const uint32_t s = static_cast<uint32_t>(op.step);
        float shock;
        if (op.kind == kOpStep)
            shock = (w[op.right * kThreads] - w[op.left * kThreads]) * P.step_f[s].w;
        else
            shock = next_normal();
        const int tc = P.time_cell[s];
        const float4 kc = P.step_f[s];
        const float dt = kc.x, sq = kc.y, tw = kc.z;
        const double fwd_prev = P.fwd[s], fwd_next = P.fwd[s + 1];
        const int32_t obs = P.obs_of_node[s + 1];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float z = (e == 0) ? shock : -shock;
            const float x = __logf(f[e]);
            const float v = interp_f32(s_v, s_x, nx, tc, tw, x, hint[e]);
            if (CB && s > 0) {
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count) &&
                        P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                        barrier_interval(P.products[k], acc[e][k], P.smoothing, prev_f[e],
                                         static_cast<double>(f[e]) * fwd_prev, prev_v[e], v, P.dt[s - 1], failed);
            }
            if (CB) {
                prev_f[e] = static_cast<float>(static_cast<double>(f[e]) * fwd_prev);
                prev_v[e] = v;
            }
            f[e] *= expf(-0.5f * v * dt + sqrtf(v) * sq * z);
            bad_state |= !(isfinite(f[e]) && f[e] > 0.0f);
            if (obs >= 0) {
                const double spot = static_cast<double>(f[e]) * fwd_next;
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count))
                        acc_observe(P.products[k], acc[e][k], static_cast<uint32_t>(obs), spot, P.smoothing, failed);
            }
        }
    }
    double price[E][NP];
    double diag_src[NP][8];
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            price[e][k] = 0.0;
            if (k >= static_cast<int>(P.product_count)) continue;
            const ProductParams& pp = P.products[k];
            if (CB && pp.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
                const float x = __logf(f[e]);
                const float v = interp_f32(s_v, s_x, nx, static_cast<int>(P.nt) - 2, 1.0f, x, hint[e]);
                const double terminal = static_cast<double>(f[e]) * P.fwd[steps];
                barrier_interval(pp, acc[e][k], P.smoothing, prev_f[e], terminal, prev_v[e], v, P.dt[steps - 1],
                                 failed);
                double diag[8];
                const double surv = barrier_finish(acc[e][k], P.smoothing, steps, diag);
                price[e][k] = P.discount * barrier_value(pp, terminal, surv);
#pragma unroll
                for (int q = 0; q < 8; ++q) diag_src[k][q] = e == 0 ? diag[q] : (diag_src[k][q] + diag[q]) * 0.5;
            } else {
                price[e][k] = P.discount * acc_payoff(pp, acc[e][k], P.smoothing);
            }
        }
    if (valid && bad_state) report_error(err, unit, MCG_ERR_NON_FINITE_STATE, 0, 0.0, 0);
    else if (valid && failed) report_error(err, unit, MCG_ERR_BARRIER_BRIDGE, 0, 0.0, 0);
    for (int k = 0; k < static_cast<int>(P.product_count) && k < NP; ++k) {
        double vals[kComponents];
#pragma unroll
        for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
        vals[MCG_PRICE] = E == 2 ? (price[0][k] + price[E - 1][k]) * 0.5 : price[0][k];
        if (CB && P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
#pragma unroll
            for (int q = 0; q < 8; ++q) vals[10 + q] = diag_src[k][q];
        }
        StatRecord* out = partials + ((static_cast<size_t>(scramble) * gridDim.x + blockIdx.x) * P.product_count + k) *
                                         kComponents;
        cta_reduce_write<kComponents>(vals, valid, mask, out, s_red);
    }
}

}  // namespace

// The FP32-bulk instantiation for (antithetic pairs, products).
cudaError_t launch_lv32_path(const DevicePlan& P, StatRecord* partials, uint32_t mask, ErrorWord* err,
                             cudaStream_t stream) {
    const int E = P.antithetic ? 2 : 1;
    const int np = static_cast<int>(P.product_count);
    const size_t smem = (static_cast<size_t>(P.nt) * P.nx + ((P.nx + 3) & ~3u)) * sizeof(float) +
                        static_cast<size_t>(P.slot_count) * kThreads * sizeof(float) + 4 * kComponents * sizeof(Stat) +
                        kZBatch32 * kThreads * sizeof(uint32_t) + (kThreads / 32) * 32 * kZBatch32 * sizeof(uint16_t);
    const dim3 grid(static_cast<unsigned>((P.units + kThreads - 1) / kThreads), P.scramble_count);
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<grid, kThreads, smem, stream>>>(P, partials, mask, err);
        return cudaGetLastError();
    };
    bool cb = false;
    for (int k = 0; k < np; ++k) cb |= P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
    const bool rq = P.engine == MCG_ENGINE_RQMC;
#define MCG_LV32_PICK(EE, NN)                                                         \
    do {                                                                              \
        if (rq && cb) return go(lv32_path_kernel<EE, NN, 1, 1>);                      \
        if (rq) return go(lv32_path_kernel<EE, NN, 1, 0>);                            \
        if (cb) return go(lv32_path_kernel<EE, NN, 0, 1>);                            \
        return go(lv32_path_kernel<EE, NN, 0, 0>);                                    \
    } while (0)
    if (E == 1 && np == 1) MCG_LV32_PICK(1, 1);
    if (E == 1 && np == 2) MCG_LV32_PICK(1, 2);
    if (E == 1 && np <= 4) MCG_LV32_PICK(1, 4);
    if (E == 2 && np == 1) MCG_LV32_PICK(2, 1);
    if (E == 2 && np == 2) MCG_LV32_PICK(2, 2);
    if (E == 2 && np <= 4) MCG_LV32_PICK(2, 4);
#undef MCG_LV32_PICK
    return cudaErrorNotSupported;
}

}  // namespace mcg

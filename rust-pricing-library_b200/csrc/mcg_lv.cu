// mcg_lv.cu -- local-volatility Log-Euler path kernel (FP64).
//
// Compiled with -fmad=false: every a*b+c of the reference's arithmetic rounds
// twice, as Rust evaluates it.
//
// Per unit: normals (Philox or scrambled Sobol) -> time-ordered Brownian-bridge
// program -> Log-Euler steps on the forward-normalised state
//   x = ln(f / F_i),  v = bilinear(t_i, x),  f <- f * (F_{i+1}/F_i) * exp(-v dt/2 + sqrt(v) sqrt(dt) z)
// (crates/pricing/src/engine/processes/local_vol.rs:459-619) for up to three
// spot runtimes (base, S-h, S+h for CRN Delta/Gamma,
// crates/pricing/src/engine/risk/pathwise_local_vol.rs:332-355) and both
// antithetic signs, with streaming payoffs and the continuous-barrier bridge
// (crates/pricing/src/engine/processes/local_vol_valuation.rs:251-434).
#include "mcg_kernels.cuh"

namespace mcg {

// Evolution e of E: runtime (0 base, 1 down, 2 up) and shock sign.
template <int E>
__device__ __forceinline__ int ev_which(int e) {
    if constexpr (E == 1 || E == 2) return 0;
    else return e % 3;
}
template <int E>
__device__ __forceinline__ double ev_sign(int e) {
    if constexpr (E == 2) return e == 0 ? 1.0 : -1.0;
    else if constexpr (E == 6) return e < 3 ? 1.0 : -1.0;
    else return 1.0;
}

template <int E, int NP>
__global__ void __launch_bounds__(kThreads) lv_path_kernel(const DevicePlan P, uint64_t unit_begin,
                                                           StatRecord* partials, uint32_t mask,
                                                           ErrorWord* err, int detail) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = static_cast<int>(P.nx);
    const size_t nv = static_cast<size_t>(P.nt) * P.nx;
    double* s_v = reinterpret_cast<double*>(smem_raw);
    double* s_x = s_v + nv;
    long long* s_xk = reinterpret_cast<long long*>(s_x + nx);
    double* s_w = reinterpret_cast<double*>(s_xk + nx);  // bridge slots [slot][thread]
    Stat* s_red = reinterpret_cast<Stat*>(s_w + static_cast<size_t>(P.slot_count) * kThreads);
    for (size_t i = threadIdx.x; i < nv; i += kThreads) s_v[i] = P.grid_v[i];
    for (int i = threadIdx.x; i < nx; i += kThreads) {
        s_x[i] = P.grid_x[i];
        s_xk[i] = total_key(P.grid_x[i]);
    }
    __syncthreads();
    const GridView g{s_v, s_x, s_xk, nx};

    const uint32_t scramble = blockIdx.y;
    const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < unit_begin + (detail ? 1 : P.units) && point < P.units;
    const uint64_t unit = valid ? point : 0;

    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;

    double f[E], prev_f[E], prev_v[E];
    int hint[E];
    ProductAcc acc[E][NP];
    bool failed = false;
    int fail_code = 0;
    uint32_t fail_step = 0;
    double fail_value = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        f[e] = P.spot_variant[ev_which<E>(e)];
        prev_f[e] = f[e];
        prev_v[e] = 0.0;
        hint[e] = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            acc_init(acc[e][k]);
            if (k < static_cast<int>(P.product_count) &&
                P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                barrier_begin(P.products[k], acc[e][k], P.smoothing, f[e], failed);
        }
    }
    double* w = s_w + threadIdx.x;
    const uint32_t steps = P.steps;
    for (uint32_t oi = 0; oi < P.op_count; ++oi) {
        const Op op = P.ops[oi];
        if (op.kind == kOpZero) {
            w[op.out * kThreads] = 0.0;
            continue;
        }
        if (op.kind == kOpTerminal) {
            w[op.out * kThreads] = op.sd * ns.normal(op.rank);
            continue;
        }
        if (op.kind == kOpInterior) {
            const double z = ns.normal(op.rank);
            w[op.out * kThreads] =
                op.wl * w[op.left * kThreads] + op.wr * w[op.right * kThreads] + op.sd * z;
            continue;
        }
        const uint32_t s = static_cast<uint32_t>(op.step);
        double shock;
        if (op.kind == kOpStep)
            shock = (w[op.right * kThreads] - w[op.left * kThreads]) * P.inv_sqrt_dt[s];
        else
            shock = ns.normal(op.rank);
        const int tc = P.time_cell[s];
        const double tw = P.time_weight[s];
        const double dt = P.dt[s];
        const double sq = P.sqrt_dt[s];
        const int32_t obs = P.obs_of_node[s + 1];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int which = ev_which<E>(e);
            const double* F = P.fwd + static_cast<size_t>(which) * (steps + 1);
            const double z = ev_sign<E>(e) * shock;
            const double x = log(f[e] / F[s]);
            const double v = interp_variance(g, tc, tw, x, hint[e]);
            if (s > 0) {
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count) &&
                        P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                        barrier_interval(P.products[k], acc[e][k], P.smoothing, prev_f[e], f[e],
                                         prev_v[e], v, P.dt[s - 1], failed);
            }
            const double ratio = P.ratio[static_cast<size_t>(which) * steps + s];
            const double e_factor = ratio * exp(-0.5 * v * dt + sqrt(v) * sq * z);
            prev_f[e] = f[e];
            prev_v[e] = v;
            f[e] *= e_factor;
            if (!(isfinite(f[e]) && f[e] > 0.0) && !fail_code) {
                fail_code = MCG_ERR_NON_FINITE_STATE;
                fail_step = s + 1;
                fail_value = f[e];
            }
            if (obs >= 0) {
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count))
                        acc_observe(P.products[k], acc[e][k], static_cast<uint32_t>(obs), f[e],
                                    P.smoothing, failed);
            }
        }
    }
    // Close the last bridge interval: the terminal node's variance.
    double diag_src[NP][8];
    double price[E][NP];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int which = ev_which<E>(e);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            price[e][k] = 0.0;
            if (k >= static_cast<int>(P.product_count)) continue;
            const ProductParams& pp = P.products[k];
            if (pp.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
                const double* F = P.fwd + static_cast<size_t>(which) * (steps + 1);
                const double x = log(f[e] / F[steps]);
                const double v = interp_variance(g, static_cast<int>(P.nt) - 2, 1.0, x, hint[e]);
                barrier_interval(pp, acc[e][k], P.smoothing, prev_f[e], f[e], prev_v[e], v,
                                 P.dt[steps - 1], failed);
                double diag[8];
                const double surv = barrier_finish(acc[e][k], P.smoothing, steps, diag);
                price[e][k] = P.discount * barrier_value(pp, f[e], surv);
                if (which == 0 && ev_sign<E>(e) > 0.0) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) diag_src[k][q] = diag[q];
                } else if (which == 0) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) diag_src[k][q] = (diag_src[k][q] + diag[q]) * 0.5;
                }
            } else {
                price[e][k] = P.discount * acc_payoff(pp, acc[e][k], P.smoothing);
            }
        }
    }
    if (failed && !fail_code) fail_code = MCG_ERR_BARRIER_BRIDGE;
    if (valid && fail_code) report_error(err, unit, fail_code, fail_step, fail_value, detail);

    // Components of each product (pathwise_local_vol.rs:206-355), antithetic
    // pairs averaged component-wise (valuation.rs:144-149).
    constexpr int kPairs = (E == 2 || E == 6) ? 2 : 1;
    constexpr int kPer = E / kPairs;
    const uint32_t tiles = gridDim.x;
    for (int k = 0; k < static_cast<int>(P.product_count) && k < NP; ++k) {
        double vals[kComponents];
#pragma unroll
        for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
        double comp[2][kComponents];
#pragma unroll
        for (int pr = 0; pr < kPairs; ++pr) {
#pragma unroll
            for (int c = 0; c < kComponents; ++c) comp[pr][c] = 0.0;
            const double base = price[pr * kPer + 0][k];
            comp[pr][MCG_PRICE] = base;
            if (kPer == 3) {
                const double down = price[pr * kPer + 1][k];
                const double up = price[pr * kPer + 2][k];
                const double h = P.spot_bump;
                const double delta = (up - down) / (2.0 * h);
                comp[pr][MCG_DELTA] = delta;
                comp[pr][MCG_BUMP_DELTA] = delta;
                if (P.req_gamma) {
                    const double gamma = (up - 2.0 * base + down) / (h * h);
                    comp[pr][MCG_GAMMA] = gamma;
                    comp[pr][MCG_BUMP_GAMMA] = gamma;
                }
            }
        }
#pragma unroll
        for (int c = 0; c < kComponents; ++c)
            vals[c] = kPairs == 2 ? (comp[0][c] + comp[1][c]) * 0.5 : comp[0][c];
        if (P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
#pragma unroll
            for (int q = 0; q < 8; ++q) vals[10 + q] = diag_src[k][q];
        }
        StatRecord* out =
            partials + ((static_cast<size_t>(scramble) * tiles + blockIdx.x) * P.product_count + k) *
                           kComponents;
        cta_reduce_write<kComponents>(vals, valid, mask, out, s_red);
    }
}

template __global__ void lv_path_kernel<1, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<1, 2>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<1, 4>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<2, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<2, 2>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<3, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<3, 2>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<6, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);

// Launch helper: picks the instantiation for (evolutions, products).
cudaError_t launch_lv_path(const DevicePlan& P, uint64_t unit_begin, uint64_t units, uint32_t scrambles,
                           StatRecord* partials, uint32_t mask, ErrorWord* err, int detail,
                           cudaStream_t stream, int& evolutions_out) {
    const int pairs = P.antithetic ? 2 : 1;
    const int per = P.lv_bumps ? 3 : 1;
    const int E = pairs * per;
    evolutions_out = E;
    const int np = static_cast<int>(P.product_count);
    const size_t smem = (static_cast<size_t>(P.nt) * P.nx + 2 * P.nx) * sizeof(double) +
                        static_cast<size_t>(P.slot_count) * kThreads * sizeof(double) +
                        4 * kComponents * sizeof(Stat);
    const dim3 grid(static_cast<unsigned>((units + kThreads - 1) / kThreads), scrambles);
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<grid, kThreads, smem, stream>>>(P, unit_begin, partials, mask, err, detail);
        return cudaGetLastError();
    };
    if (E == 1 && np == 1) return go(lv_path_kernel<1, 1>);
    if (E == 1 && np == 2) return go(lv_path_kernel<1, 2>);
    if (E == 1 && np <= 4) return go(lv_path_kernel<1, 4>);
    if (E == 2 && np == 1) return go(lv_path_kernel<2, 1>);
    if (E == 2 && np == 2) return go(lv_path_kernel<2, 2>);
    if (E == 3 && np == 1) return go(lv_path_kernel<3, 1>);
    if (E == 3 && np == 2) return go(lv_path_kernel<3, 2>);
    if (E == 6 && np == 1) return go(lv_path_kernel<6, 1>);
    return cudaErrorNotSupported;
}

}  // namespace mcg

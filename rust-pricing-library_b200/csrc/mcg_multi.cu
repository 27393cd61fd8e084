// mcg_multi.cu -- correlated multi-asset paths (FP64, compiled with -fmad=false).
//
// MultiAssetPricingPlan's shocks and paths
// (crates/pricing/src/engine/multi_asset/path.rs:24-200) on the GPU, one
// thread per sampling unit: every asset's factor takes its own normals --
// Philox coordinate or scrambled Sobol word, dimension f x steps + step, or
// step x assets + f for RQMC with the Brownian bridge -- bridged per factor by
// the time-ordered program the single-asset tiles use, correlated per step by
// the lower Cholesky factor of the step's correlation matrix
// (sum_{k <= i} L_ik z_k in k order), and evolves its asset: the
// Black--Scholes step f F_{s+1}/F_s exp(-sigma^2 dt/2 + sigma sqrt(dt) z) or
// the Log-Euler step on the asset's own local-variance grid.  The antithetic
// mate negates every independent normal, so it runs beside the primary path
// on the same normals and bridge values.  The unit's value is the discounted
// basket or worst-of payoff (crates/pricing/src/product/multi_asset.rs:77-246),
// averaged with its mate; a CTA reduces its 128 units into one statistics
// record with the fixed tree of the single-asset kernels.
#include "mcg_multi.cuh"

namespace mcg {

namespace {

// The basket's value (sum of weighted, scaled terminal spots) or the
// worst-of's (the smallest scaled spot), then the option on it.
template <int NA>
__device__ __forceinline__ double multi_payoff(const MultiAssetDev& M, const double (&s)[NA]) {
    double w;
    if (M.product == MCG_MULTI_BASKET) {
        w = 0.0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
            if (i < static_cast<int>(M.n)) w = w + (M.weights[i] * s[i]) / M.scales[i];
    } else {
        w = s[0] / M.scales[0];
#pragma unroll
        for (int i = 1; i < NA; ++i) {
            if (i >= static_cast<int>(M.n)) break;
            const double x = s[i] / M.scales[i];
            if (M.smoothing > 0.0) {
                // CompactC2Smoothing::minimum: left - positive_part(left - right)
                const double diff = w - x;
                if (diff >= M.smoothing) w = x;
                else if (diff > -M.smoothing) w = w - smooth_positive_part(M.smoothing, diff).value;
            } else {
                w = w <= x ? w : x;
            }
        }
    }
    const double intrinsic = M.side == MCG_CALL ? w - M.strike : M.strike - w;
    double positive;
    if (M.smoothing > 0.0) {
        double dl, dr;
        positive = smooth_maximum(M.smoothing, intrinsic, 0.0, dl, dr);
    } else {
        positive = intrinsic >= 0.0 ? intrinsic : 0.0;
    }
    return 0.0 + (M.notional * positive) * M.df;
}

// 5 CTAs per SM (96 registers; left free it took 128 and 4 CTAs, 24.66 against 23.64 ms for the
// four-asset basket at 2^20 antithetic units).
template <int NA>
__global__ void __launch_bounds__(kThreads, 5) multi_asset_kernel(const MultiAssetDev M, StatRecord* partials,
                                                               ErrorWord* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Stat* s_red = reinterpret_cast<Stat*>(smem_raw);
    double* s_z = reinterpret_cast<double*>(s_red + 4);                                 // batched normals [k][thread]
    uint16_t* s_zlist = reinterpret_cast<uint16_t*>(s_z + z_batch<1>() * kThreads);      // tail lists, per warp
    double* s_w = reinterpret_cast<double*>(s_zlist + (kThreads / 32) * 32 * z_batch<1>());  // bridge slots
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < M.units;
    const uint64_t unit = valid ? point : 0;
    const uint32_t n = M.n;
    NormalSource ns;
    ns.rqmc = M.engine == MCG_ENGINE_RQMC;
    ns.seed = M.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = M.scr_dirs ? M.scr_dirs + static_cast<size_t>(scramble) * M.dimension * 32u : nullptr;
    ns.shift = M.scr_shift ? M.scr_shift + static_cast<size_t>(scramble) * M.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    if (ns.rqmc) {  // the grid starts at point 0: every warp holds 32 aligned points
        const uint32_t q = static_cast<uint32_t>(point) & ~31u;
        ns.high_gray = q ^ (q >> 1);
        ns.lane_low = static_cast<uint32_t>(point) & 31u;
        ns.low = M.scr_low + static_cast<size_t>(scramble) * M.dimension * 32u;
    }
    constexpr int kSides = 2;  // primary and antithetic mate
    const int sides = M.antithetic ? 2 : 1;
    double f[kSides][NA], xs[kSides][NA];
    int hint[kSides][NA];
#pragma unroll
    for (int e = 0; e < kSides; ++e)
#pragma unroll
        for (int i = 0; i < NA; ++i) {
            f[e][i] = i < static_cast<int>(n) ? M.spot[i] : 1.0;
            xs[e][i] = 0.0;
            hint[e][i] = 0;
        }
    bool bad = false;
    uint32_t bad_step = 0;
    double bad_value = 0.0;
    double* w = s_w + threadIdx.x;
    // The unit's normals in consumption order (M.z_dims), eight at a time with
    // AS241's tail branch compacted across the warp (fill_normals); every
    // thread walks the same program, so the warp-collective batches line up.
    NormalSource nsq[1] = {ns};
    uint32_t zi = 0, zbase = 0, zend = 0;
    auto next_normal = [&]() -> double {
        if (zi == zend) {
            zbase = zi;
            constexpr uint32_t kBatch = static_cast<uint32_t>(z_batch<1>());
            const uint32_t cnt = M.z_count - zi < kBatch ? M.z_count - zi : kBatch;
            fill_normals<1>(nsq, ns.rqmc, zi, cnt, s_z, s_zlist, M.z_dims);
            zend = zi + cnt;
        }
        const uint32_t k = zi++ - zbase;
        return s_z[k * kThreads + threadIdx.x];
    };
    const size_t fstride = static_cast<size_t>(M.slot_count) * kThreads;  // factor f's slots: w + f * fstride
    if (M.bridge)
        for (uint32_t q = 0; q < n; ++q) w[q * fstride + M.zero_slot * kThreads] = 0.0;
    for (uint32_t s = 0; s < M.steps; ++s) {
        double ind[NA];
        if (M.bridge) {
            const int4 prog = M.step_prog[s];
            for (int32_t j = 0; j < prog.y; ++j) {
                const BridgeNode nd = M.bridge_nodes[prog.x + j];
                for (uint32_t q = 0; q < n; ++q) {
                    double* wq = w + q * fstride;
                    const double z = next_normal();
                    wq[nd.out * kThreads] = nd.wl * wq[nd.left * kThreads] + nd.wr * wq[nd.right * kThreads] + nd.sd * z;
                }
            }
#pragma unroll
            for (int q = 0; q < NA; ++q)
                ind[q] = q < static_cast<int>(n)
                             ? (w[q * fstride + prog.w * kThreads] - w[q * fstride + prog.z * kThreads]) * M.inv_sqrt_dt[s]
                             : 0.0;
        } else {
#pragma unroll
            for (int q = 0; q < NA; ++q) ind[q] = q < static_cast<int>(n) ? next_normal() : 0.0;
        }
        // correlated shocks, path.rs:76-96
        const double* l = M.lower + static_cast<size_t>(M.step_entry[s]) * n * n;
        double c[NA];
#pragma unroll
        for (int i = 0; i < NA; ++i) {
            double value = 0.0;
            if (i < static_cast<int>(n))
                for (int k = 0; k <= i; ++k) value += l[i * n + k] * ind[k];
            c[i] = value;
        }
        const double dt = M.dt[s], sq = M.sqrt_dt[s];
#pragma unroll
        for (int e = 0; e < kSides; ++e) {
            if (e >= sides) break;
            const double sign = e == 0 ? 1.0 : -1.0;
#pragma unroll
            for (int i = 0; i < NA; ++i) {
                if (i >= static_cast<int>(n)) break;
                const double z = sign * c[i];
                const double ratio = M.ratio[static_cast<size_t>(i) * M.steps + s];
                double next;
                if (M.model[i] == MCG_MODEL_BLACK_SCHOLES) {
                    const double vol = M.vol[i];
                    next = f[e][i] * ratio * exp(-0.5 * vol * vol * dt + vol * sq * z);
                } else {
                    const GridView g{nullptr, nullptr, nullptr, M.nx[i], M.bounds[i], M.cells[i], M.x_first[i],
                                     M.x_last[i]};
                    const size_t at = static_cast<size_t>(i) * M.steps + s;
                    const double v = interp_variance_walk(g, M.time_cell[at], M.time_weight[at], xs[e][i], hint[e][i]);
                    const double incr = -0.5 * v * dt + sqrt(v) * sq * z;
                    xs[e][i] += incr;
                    next = f[e][i] * (ratio * exp(incr));
                }
                if (!(isfinite(next) && next > 0.0) && !bad) {
                    bad = true;
                    bad_step = s + 1;
                    bad_value = next;
                }
                f[e][i] = next;
            }
        }
    }
    double value = multi_payoff<NA>(M, f[0]);
    if (M.antithetic) value = (value + multi_payoff<NA>(M, f[1])) * 0.5;
    if (valid && bad) report_error(err, unit, MCG_ERR_NON_FINITE_STATE, bad_step, bad_value, false);
    const double vals[1] = {value};
    cta_reduce_write<1>(vals, valid, 1u, partials + static_cast<size_t>(scramble) * gridDim.x + blockIdx.x, s_red);
}

}  // namespace

size_t multi_asset_smem(const MultiAssetDev& M) {
    return 4 * sizeof(Stat) + static_cast<size_t>(z_batch<1>()) * kThreads * sizeof(double) +
           (kThreads / 32) * 32 * static_cast<size_t>(z_batch<1>()) * sizeof(uint16_t) +
           (M.bridge ? static_cast<size_t>(M.n) * M.slot_count * kThreads * sizeof(double) : 0);
}

cudaError_t launch_multi_asset(const MultiAssetDev& M, uint32_t scrambles, StatRecord* partials, ErrorWord* err,
                               cudaStream_t stream) {
    const size_t smem = multi_asset_smem(M);
    const dim3 grid(static_cast<unsigned>((M.units + kThreads - 1) / kThreads), scrambles);
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<grid, kThreads, smem, stream>>>(M, partials, err);
        return cudaGetLastError();
    };
    if (M.n <= 2) return go(multi_asset_kernel<2>);
    if (M.n <= 4) return go(multi_asset_kernel<4>);
    return go(multi_asset_kernel<8>);
}

}  // namespace mcg

// mcg_lv_tile.cuh -- the local-volatility per-tile path evaluation, shared
// by the single-plan kernel (mcg_lv.cu) and the batched book (mcg_book.cu).
//
// Every translation unit that includes it compiles with -fmad=false: every
// a*b+c of the reference's arithmetic rounds twice, as Rust evaluates it.
//
// Per unit: normals (Philox or scrambled Sobol) -> time-ordered Brownian-bridge
// program -> Log-Euler steps on the forward-normalised state
//   x = ln(f / F_i),  v = bilinear(t_i, x),  f <- f * (F_{i+1}/F_i) * exp(-v dt/2 + sqrt(v) sqrt(dt) z),
//   with x advanced by the same exponent (x <- x - v dt/2 + sqrt(v) sqrt(dt) z)
// (crates/pricing/src/engine/processes/local_vol.rs:459-619) for up to three
// spot runtimes (base, S-h, S+h for CRN Delta/Gamma,
// crates/pricing/src/engine/risk/pathwise_local_vol.rs:332-355) and both
// antithetic signs, with streaming payoffs and the continuous-barrier bridge
// (crates/pricing/src/engine/processes/local_vol_valuation.rs:251-434).
#pragma once

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

// One 128-unit tile of Log-Euler paths: unit `point` of scramble `scramble`
// per thread, the grid `g` and the bridge slots `s_w` ([slot][thread]) in
// shared memory, the CTA's records written at tile_out[k * kComponents + c].
// RQ / CB: 1 or 0 specialise the kernel on the engine (RQMC or Philox) and
// on whether any product is a continuous barrier, so the code and state of
// the other case are compiled out; -1 decides both from the plan at run
// time.  The arithmetic is the same either way.
// Batched normals: kZBatch normals of the program per thread at a time, in
// s_z[k][thread].  The warp forms the uniforms, takes AS241's central branch
// for every lane, and evaluates the tail branch only for the lanes that need
// it, 32 at a time from a compacted list (s_zlist, 32 * kZBatch entries per
// warp); the values are those of as241 bit for bit, without a warp executing
// the tail branch for each normal that one of its lanes sends there.
constexpr int kZBatch = 8;

__device__ __forceinline__ void fill_normals(const DevicePlan& P, NormalSource& ns, bool wsob, uint32_t first,
                                             uint32_t count, double* s_z, uint16_t* s_zlist) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    uint16_t* list = s_zlist + warp * (32u * kZBatch);
    uint32_t tails = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t rank = __ldg(P.z_ranks + first + k);
        const double p = open_unit(wsob ? ns.word_warp(rank) : ns.word(rank));
        const double c = p - 0.5;
        const bool tail = !(fabs(c) <= 0.425);
        const double central = as241_central(c);
        s_z[k * kThreads + threadIdx.x] = tail ? p : central;
        const unsigned m = __ballot_sync(0xffffffffu, tail);
        if (tail) list[tails + __popc(m & ((1u << lane) - 1u))] = static_cast<uint16_t>(k * 32u + lane);
        tails += static_cast<uint32_t>(__popc(m));
    }
    __syncwarp();
    for (uint32_t b = 0; b < tails; b += 32u) {
        const uint32_t i = b + lane;
        if (i < tails) {
            const uint32_t idx = list[i];
            double* at = s_z + (idx >> 5) * kThreads + warp * 32u + (idx & 31u);
            const double p = *at;
            *at = as241_tail(p, p - 0.5);
        }
    }
    __syncwarp();
}

template <int E, int NP, int RQ = -1, int CB = -1>
__device__ __forceinline__ void lv_tile(const DevicePlan& P, const GridView& g, double* s_w, Stat* s_red,
                                        uint32_t scramble, uint64_t point, bool valid, StatRecord* tile_out,
                                        uint32_t mask, ErrorWord* err, int detail, bool warp_sobol = false,
                                        double* s_z = nullptr, uint16_t* s_zlist = nullptr) {
    const uint64_t unit = valid ? point : 0;

    NormalSource ns;
    ns.rqmc = RQ < 0 ? P.engine == MCG_ENGINE_RQMC : RQ != 0;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    // Warp-cooperative Sobol words when the warp's points form one aligned block of 32.
    const bool wsob = warp_sobol && ns.rqmc;
    if (wsob) {
        const uint32_t q = static_cast<uint32_t>(point) & ~31u;
        ns.high_gray = q ^ (q >> 1);
        ns.lane_low = static_cast<uint32_t>(point) & 31u;
        ns.low = P.scr_low + static_cast<size_t>(scramble) * P.dimension * 32u;
    }

    double f[E], xs[E], prev_f[E], prev_v[E];
    int hint[E];
    ProductAcc acc[E][NP];
    bool failed = false;
    int fail_code = 0;
    uint32_t fail_step = 0;
    double fail_value = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        f[e] = P.spot_variant[ev_which<E>(e)];
        xs[e] = 0.0;  // ln(f / F_0): F_0 is the spot of the runtime
        prev_f[e] = f[e];
        prev_v[e] = 0.0;
        hint[e] = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            acc_init(acc[e][k], P.products[k]);
            if (CB != 0 && k < static_cast<int>(P.product_count) &&
                P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                barrier_begin(P.products[k], acc[e][k], P.smoothing, f[e], failed);
        }
    }
    double* w = s_w + threadIdx.x;
    const uint32_t steps = P.steps;
    // The program's normals in order: from the batch in shared memory, or
    // one at a time (s_z null).
    uint32_t zi = 0, zbase = 0, zend = 0;
    auto next_normal = [&](uint32_t rank) -> double {
        if (s_z == nullptr) return wsob ? ns.normal_warp(rank) : ns.normal(rank);
        if (zi == zend) {
            zbase = zi;
            const uint32_t n = P.z_count - zi < static_cast<uint32_t>(kZBatch) ? P.z_count - zi
                                                                              : static_cast<uint32_t>(kZBatch);
            fill_normals(P, ns, wsob, zi, n, s_z, s_zlist);
            zend = zi + n;
        }
        return s_z[(zi++ - zbase) * kThreads + threadIdx.x];
    };
    for (uint32_t oi = 0; oi < P.op_count; ++oi) {
        const Op op = P.ops[oi];
        if (op.kind == kOpZero) {
            w[op.out * kThreads] = 0.0;
            continue;
        }
        if (op.kind == kOpTerminal) {
            w[op.out * kThreads] = op.sd * next_normal(op.rank);
            continue;
        }
        if (op.kind == kOpInterior) {
            // wl W_L + wr W_R + sd z (bridge.rs:290-305), the sums fused
            const double z = next_normal(op.rank);
            w[op.out * kThreads] = fma(op.wl, w[op.left * kThreads], fma(op.wr, w[op.right * kThreads], op.sd * z));
            continue;
        }
        const uint32_t s = static_cast<uint32_t>(op.step);
        const LvStep st = P.lv_steps[s];
        double shock;
        if (op.kind == kOpStep)
            shock = (w[op.right * kThreads] - w[op.left * kThreads]) * st.inv_sqrt_dt;
        else
            shock = next_normal(op.rank);
        const int tc = st.time_cell;
        const double tw = st.time_weight;
        const double dt = st.dt;
        const double sq = st.sqrt_dt;
        const double mhdt = -0.5 * dt;  // exact: (-0.5 v) dt and v (-0.5 dt) round alike
        const int32_t obs = st.obs_next;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int which = ev_which<E>(e);
            const double z = ev_sign<E>(e) * shock;
            // x = ln(f / F_s), carried by the steps' own exponents (the forward
            // ratios cancel) in place of a division and a logarithm per step;
            // it differs from the reference's ln(f / F_s) by rounding only
            // (~1e-16 per step), and only through the interpolated variance.
            // The state f itself follows the reference's recurrence.
            const double x = xs[e];
            const double v = interp_variance_walk(g, tc, tw, x, hint[e]);
            if (CB != 0 && s > 0) {
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count) &&
                        P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                        barrier_interval(P.products[k], acc[e][k], P.smoothing, prev_f[e], f[e],
                                         prev_v[e], v, P.dt[s - 1], failed);
            }
            const double ratio = which == 0 ? st.ratio : P.ratio[static_cast<size_t>(which) * steps + s];
            // -v dt / 2 + sqrt(v) sqrt(dt) z with the last product and the sum fused
            const double incr = fma(sqrt(v) * sq, z, v * mhdt);
            const double e_factor = ratio * exp(incr);
            xs[e] += incr;
            if (CB != 0) {
                prev_f[e] = f[e];
                prev_v[e] = v;
            }
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
            if (CB != 0 && pp.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
                const double* F = P.fwd + static_cast<size_t>(which) * (steps + 1);
                const double x = log(f[e] / F[steps]);
                const double v = interp_variance_walk(g, static_cast<int>(P.nt) - 2, 1.0, x, hint[e]);
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
        if (CB != 0 && P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
#pragma unroll
            for (int q = 0; q < 8; ++q) vals[10 + q] = diag_src[k][q];
        }
        cta_reduce_write<kComponents>(vals, valid, mask, tile_out + static_cast<size_t>(k) * kComponents, s_red);
    }
}


}  // namespace mcg

// mcg_lv_tile.cuh -- the local-volatility per-tile path evaluation, shared
// by the single-plan kernel (mcg_lv.cu) and the batched book (mcg_book.cu).
//
// Every translation unit that includes it compiles with -fmad=false: every
// a*b+c of the reference's arithmetic rounds twice, as Rust evaluates it,
// except where a fused multiply-add is written out (bridge nodes, the step's
// increment, the bilinear interpolation), whose results are held to 1e-12 of
// the reference rather than to the bit.
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

// One or two 128-unit tiles of Log-Euler paths.  Thread t evaluates unit
// `point` (tile 0) and, for Q = 2, unit `point + 128` of the next tile, each
// with its own normals, state and accumulators; the per-step record, the grid
// row addresses, the product dispatch and (RQMC) the Sobol direction row are
// shared by the thread's paths, and their two dependency chains interleave.
// The bridge slots are s_w[q][slot][thread], the batched normals
// s_z[k][q][thread].  Tile q's records go to tile_out[q] (k * kComponents + c);
// a null tile_out[1] means the second tile does not exist (its units are
// beyond the plan).  Each tile's records are those of the one-path-per-thread
// form bit for bit: the same per-unit arithmetic and the same CTA tree.
// RQ / CB: 1 or 0 specialise the kernel on the engine (RQMC or Philox) and
// on whether any product is a continuous barrier, so the code and state of
// the other case are compiled out; -1 decides both from the plan at run
// time; CB = 2 is a continuous barrier under a positive smoothing width, whose
// exact-bridge code is compiled out.  The arithmetic is the same either way.
// Q = 2 needs E = 1.
template <int E, int NP, int RQ = -1, int CB = -1, int Q = 1>
__device__ __forceinline__ void lv_tile(const DevicePlan& P, const GridView& g, double* s_w, Stat* s_red,
                                        uint32_t scramble, uint64_t point, bool valid, StatRecord* tile_out,
                                        uint32_t mask, ErrorWord* err, int detail, bool warp_sobol = false,
                                        double* s_z = nullptr, uint16_t* s_zlist = nullptr,
                                        bool valid_second = false, StatRecord* tile_out_second = nullptr,
                                        double* unit_price = nullptr) {
    static_assert(Q == 1 || (Q == 2 && E == 1), "two paths per thread take one evolution each");
    constexpr int QE = Q * E;
    // The plan's smoothing width, read where it is used (a kernel parameter,
    // so no register holds it); positive under CB = 2.
    auto smoothing_width = [&]() -> double {
        const double h = P.smoothing;
        if constexpr (CB == 2) __builtin_assume(h > 0.0);
        return h;
    };
    const bool valid_q[2] = {valid, valid_second};
    uint64_t unit_q[Q];
    NormalSource ns[Q];
    const bool rqmc = RQ < 0 ? P.engine == MCG_ENGINE_RQMC : RQ != 0;
    // Warp-cooperative Sobol words when the warp's points form one aligned block of 32.
    const bool wsob = warp_sobol && rqmc;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const uint64_t pt = point + static_cast<uint64_t>(q) * kThreads;
        unit_q[q] = valid_q[q] ? pt : 0;
        ns[q].rqmc = rqmc;
        ns[q].seed = P.seed;
        ns[q].unit = unit_q[q];
        ns[q].gray = static_cast<uint32_t>(unit_q[q] ^ (unit_q[q] >> 1));
        ns[q].dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
        ns[q].shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
        ns[q].cached_block = 0xffffffffu;
        if (wsob) {
            const uint32_t blk = static_cast<uint32_t>(pt) & ~31u;
            ns[q].high_gray = blk ^ (blk >> 1);
            ns[q].lane_low = static_cast<uint32_t>(pt) & 31u;
            ns[q].low = P.scr_low + static_cast<size_t>(scramble) * P.dimension * 32u;
        }
    }

    // Evolution i = q * E + e: path q, evolution e of that path's normals.
    double f[QE], xs[QE], prev_f[QE], prev_v[QE];
    int hint[QE];
    ProductAcc acc[NP][QE];  // product-major: one observation dispatch per product for all paths
    bool failed[Q];
    int fail_code[Q];
    uint32_t fail_step[Q];
    double fail_value[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        failed[q] = false;
        fail_code[q] = 0;
        fail_step[q] = 0;
        fail_value[q] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < QE; ++i) {
        const int e = i % E;
        f[i] = P.spot_variant[ev_which<E>(e)];
        xs[i] = 0.0;  // ln(f / F_0): F_0 is the spot of the runtime
        prev_f[i] = f[i];
        prev_v[i] = 0.0;
        hint[i] = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            acc_init(acc[k][i], P.products[k]);
            if (CB != 0 && k < static_cast<int>(P.product_count) &&
                P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                barrier_begin(P.products[k], acc[k][i], smoothing_width(), f[i], failed[i / E]);
        }
    }
    double* w = s_w + threadIdx.x;
    const size_t q_stride = static_cast<size_t>(P.slot_count) * kThreads;  // path q's slots: w + q * q_stride
    const uint32_t steps = P.steps;
    // The program's normals in order: from the batch in shared memory, or
    // one at a time (s_z null, one path per thread).
    uint32_t zi = 0, zbase = 0, zend = 0;
    auto next_normals = [&](uint32_t rank, double (&z)[Q]) {
        if (s_z == nullptr) {
            z[0] = wsob ? ns[0].normal_warp(rank) : ns[0].normal(rank);
            return;
        }
        if (zi == zend) {
            zbase = zi;
            constexpr uint32_t kBatch = static_cast<uint32_t>(z_batch<Q>());
            const uint32_t n = P.z_count - zi < kBatch ? P.z_count - zi : kBatch;
            fill_normals<Q>(ns, wsob, zi, n, s_z, s_zlist, P.z_ranks);
            zend = zi + n;
        }
        const uint32_t k = zi++ - zbase;
#pragma unroll
        for (int q = 0; q < Q; ++q) z[q] = s_z[(k * Q + q) * kThreads + threadIdx.x];
    };
#pragma unroll
    for (int q = 0; q < Q; ++q) w[q * q_stride + P.zero_slot * kThreads] = 0.0;  // W(0)
    for (uint32_t s = 0; s < steps; ++s) {
        const int4 prog = P.step_prog[s];
        // The bridge nodes this step needs first: wl W_L + wr W_R + sd z
        // (bridge.rs:290-305), the sums fused.
        for (int32_t j = 0; j < prog.y; ++j) {
            const BridgeNode nd = P.bridge_nodes[prog.x + j];
            double z[Q];
            next_normals(static_cast<uint32_t>(nd.rank), z);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                double* wq = w + q * q_stride;
                wq[nd.out * kThreads] = fma(nd.wl, wq[nd.left * kThreads], fma(nd.wr, wq[nd.right * kThreads], nd.sd * z[q]));
            }
        }
        const LvStep st = P.lv_steps[s];
        double shock[Q];
        if (prog.z >= 0) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const double* wq = w + q * q_stride;
                shock[q] = (wq[prog.w * kThreads] - wq[prog.z * kThreads]) * st.inv_sqrt_dt;
            }
        } else {
            next_normals(s, shock);
        }
        const int tc = st.time_cell;
        const double tw = st.time_weight;
        const double dt = st.dt;
        const double sq = st.sqrt_dt;
        const double mhdt = -0.5 * dt;  // exact: (-0.5 v) dt and v (-0.5 dt) round alike
        const int32_t obs = st.obs_next;
#pragma unroll
        for (int i = 0; i < QE; ++i) {
            const int q = i / E, e = i % E;
            const int which = ev_which<E>(e);
            const double z = ev_sign<E>(e) * shock[q];
            // x = ln(f / F_s), carried by the steps' own exponents (the forward
            // ratios cancel) in place of a division and a logarithm per step;
            // it differs from the reference's ln(f / F_s) by rounding only
            // (~1e-16 per step), and only through the interpolated variance.
            // The state f itself follows the reference's recurrence.
            const double x = xs[i];
            const double v = interp_variance_walk(g, tc, tw, x, hint[i]);
            if (CB != 0 && s > 0) {
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count) &&
                        P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                        barrier_interval(P.products[k], acc[k][i], smoothing_width(), prev_f[i], f[i],
                                         prev_v[i], v, P.dt[s - 1], failed[q]);
            }
            const double ratio = which == 0 ? st.ratio : P.ratio[static_cast<size_t>(which) * steps + s];
            // -v dt / 2 + sqrt(v) sqrt(dt) z with the last product and the sum fused
            const double incr = fma(sqrt(v) * sq, z, v * mhdt);
            const double e_factor = ratio * exp_step(incr);
            xs[i] += incr;
            if (CB != 0) {
                prev_f[i] = f[i];
                prev_v[i] = v;
            }
            f[i] *= e_factor;
            if (!(isfinite(f[i]) && f[i] > 0.0) && !fail_code[q]) {
                fail_code[q] = MCG_ERR_NON_FINITE_STATE;
                fail_step[q] = s + 1;
                fail_value[q] = f[i];
            }
        }
        if (obs >= 0) {
            if constexpr (Q == 1) {
                // Observed spots: the state itself, or with discrete dividends the
                // node coordinate a S + b f of each evolution's spot runtime (and
                // the pre-dividend one on an ex-date), local_vol_valuation.rs:221-247.
                double spot[QE], pre[QE];
                bool with_pre = false;
#pragma unroll
                for (int i = 0; i < QE; ++i) spot[i] = pre[i] = f[i];
                if (P.dividends) {
                    with_pre = P.obs_div[obs].w != 0.0;
#pragma unroll
                    for (int i = 0; i < QE; ++i) {
                        const int which = ev_which<E>(i % E);
                        const double4 c = P.lv_obs_div[static_cast<size_t>(which) * P.observation_count + obs];
                        const double s0 = P.spot_variant[which];
                        spot[i] = c.x * s0 + c.y * f[i];
                        pre[i] = c.z * s0 + c.w * f[i];
                    }
                }
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count))
                        acc_observe_n<QE>(P.products[k], acc[k], static_cast<uint32_t>(obs), spot,
                                          smoothing_width(), pre, with_pre);
            } else {
                // Two paths per thread: plans without dividends (the launch
                // helper's choice), so the observed spot is the state.
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (k < static_cast<int>(P.product_count))
                        acc_observe_n<QE, false>(P.products[k], acc[k], static_cast<uint32_t>(obs), f,
                                                 smoothing_width(), f, false);
            }
        }
    }
    // Close the last bridge interval: the terminal node's variance.
    double diag_src[Q][NP][8];
    double price[QE][NP];
#pragma unroll
    for (int i = 0; i < QE; ++i) {
        const int q = i / E, e = i % E;
        const int which = ev_which<E>(e);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            price[i][k] = 0.0;
            if (k >= static_cast<int>(P.product_count)) continue;
            const ProductParams& pp = P.products[k];
            if (CB != 0 && pp.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
                const double* F = P.fwd + static_cast<size_t>(which) * (steps + 1);
                const double x = log(f[i] / F[steps]);
                const double v = interp_variance_walk(g, static_cast<int>(P.nt) - 2, 1.0, x, hint[i]);
                barrier_interval(pp, acc[k][i], smoothing_width(), prev_f[i], f[i], prev_v[i], v,
                                 P.dt[steps - 1], failed[q]);
                double diag[8];
                const double surv = barrier_finish(acc[k][i], smoothing_width(), steps, diag);
                price[i][k] = P.discount * barrier_value(pp, f[i], surv);
                if (which == 0 && ev_sign<E>(e) > 0.0) {
#pragma unroll
                    for (int d = 0; d < 8; ++d) diag_src[q][k][d] = diag[d];
                } else if (which == 0) {
#pragma unroll
                    for (int d = 0; d < 8; ++d) diag_src[q][k][d] = (diag_src[q][k][d] + diag[d]) * 0.5;
                }
            } else {
                price[i][k] = P.discount * acc_payoff(pp, acc[k][i], smoothing_width());
            }
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (failed[q] && !fail_code[q]) fail_code[q] = MCG_ERR_BARRIER_BRIDGE;
        if (valid_q[q] && fail_code[q]) report_error(err, unit_q[q], fail_code[q], fail_step[q], fail_value[q], detail);
    }

    // Components of each product (pathwise_local_vol.rs:206-355), antithetic
    // pairs averaged component-wise (valuation.rs:144-149); one CTA record per
    // tile and product.
    constexpr int kPairs = (E == 2 || E == 6) ? 2 : 1;
    constexpr int kPer = E / kPairs;
    StatRecord* const outs[2] = {tile_out, tile_out_second};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q > 0 && outs[q] == nullptr) break;  // uniform: the CTA's second tile lies beyond the plan
        for (int k = 0; k < static_cast<int>(P.product_count) && k < NP; ++k) {
            double vals[kComponents];
#pragma unroll
            for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
            double comp[2][kComponents];
#pragma unroll
            for (int pr = 0; pr < kPairs; ++pr) {
#pragma unroll
                for (int c = 0; c < kComponents; ++c) comp[pr][c] = 0.0;
                const double base = price[q * E + pr * kPer + 0][k];
                comp[pr][MCG_PRICE] = base;
                if (kPer == 3) {
                    const double down = price[q * E + pr * kPer + 1][k];
                    const double up = price[q * E + pr * kPer + 2][k];
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
                for (int d = 0; d < 8; ++d) vals[10 + d] = diag_src[q][k][d];
            }
            // unit_price (optional, one path per thread): the first product's
            // discounted price of each unit, antithetic pairs averaged.
            if (Q == 1 && unit_price != nullptr && k == 0 && valid_q[q]) unit_price[unit_q[q]] = vals[MCG_PRICE];
            cta_reduce_write<kComponents>(vals, valid_q[q], mask, outs[q] + static_cast<size_t>(k) * kComponents,
                                          s_red);
        }
    }
}


}  // namespace mcg

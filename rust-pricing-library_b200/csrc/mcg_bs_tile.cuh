// mcg_bs_tile.cuh -- the Black--Scholes per-tile path evaluation, shared by
// the single-plan kernels (mcg_bs.cu) and the batched book (mcg_book.cu).
//
// Single-terminal products take the exact lognormal step and the pathwise
// adjoint of pathwise_aad_single_terminal
// (crates/pricing/src/engine/processes/black_scholes.rs:757-793), evaluated
// at the base point and the six bumped points of pathwise_values (:417-472):
// spot bumps reuse the base exponential bit for bit, only the two volatility
// bumps need their own.  Multi-observation products follow the cumulative
// Brownian motion of path_observations_from_normals (:297-331) with streaming
// payoffs and the continuous-barrier bridge (:94-293).
#pragma once

#include "mcg_kernels.cuh"

namespace mcg {

struct Aad {
    double price, delta, vega;
};

// Payoff value and dPayoff/dTerminal of a single-terminal product
// (European or Digital), tape.rs:594-781 reverse semantics.
__device__ __forceinline__ double terminal_payoff(const ProductParams& p, double s, double h,
                                                 double& adj) {
    const bool call = p.side == MCG_CALL;
    if (p.kind == MCG_PRODUCT_DIGITAL) {
        const double dist = call ? s - p.strike : p.strike - s;
        double ind, first = 0.0;
        if (h > 0.0) {
            double comp;
            const SmoothD d = smooth_indicator(h, dist, comp);
            ind = d.value;
            first = d.first;
        } else {
            ind = dist >= 0.0 ? 1.0 : 0.0;
        }
        const bool asset = p.digital_payout == MCG_DIGITAL_ASSET;
        const double base = asset ? s * p.payout : p.payout;
        double a = 0.0;
        if (asset) a += ind * p.payout;
        if (h > 0.0) a += (call ? 1.0 : -1.0) * (base * first);
        adj = a;
        return ind * base;
    }
    const double in = call ? s - p.strike : p.strike - s;
    adj = (in >= 0.0 ? p.notional : 0.0) * (call ? 1.0 : -1.0);
    return (in >= 0.0 ? in : 0.0) * p.notional;
}

// The coordinate of observation i at a spot runtime: the plan's dividend
// coordinate refit to `spot` (AffineDividendCoordinate::at_spot), or the
// identity (a = 0, b = 1) without dividends.
__device__ __forceinline__ DivCoord obs_coord(const DevicePlan& P, uint32_t i, double spot) {
    return P.dividends ? div_at_spot(P.obs_div[i], P.spot, spot) : DivCoord{0.0, 1.0, 1.0};
}

// The observed spot of state f at observation i and, on an ex-date, the spot
// before the dividend (path_observation, black_scholes.rs:335-354).
__device__ __forceinline__ double obs_spot(const DevicePlan& P, uint32_t i, double spot, double f, double& pre,
                                           bool& with_pre) {
    with_pre = false;
    pre = f;
    if (!P.dividends) return f;
    const DivCoord c = div_at_spot(P.obs_div[i], P.spot, spot);
    with_pre = P.obs_div[i].w != 0.0;
    if (with_pre) {
        const DivCoord b = div_at_spot(P.obs_div_pre[i], P.spot, spot);
        pre = b.a * spot + b.b * f;
    }
    return c.a * spot + c.b * f;
}

// pathwise_aad_single_terminal with the exponential supplied by the caller.
__device__ __forceinline__ Aad single_terminal(const DevicePlan& P, const ProductParams& p,
                                               double spot, double vol, double z, double e_lr) {
    const double t = P.expiry;
    const double bf = P.obs_fwd[0] * (spot / P.spot);
    const double f = bf * e_lr;
    const DivCoord c = obs_coord(P, 0, spot);
    // S = a spot + b f (the identity coordinate: f itself)
    const double terminal = P.dividends ? c.a * spot + c.b * f : f;
    double a;
    const double value = terminal_payoff(p, terminal, P.smoothing, a);
    Aad r;
    r.price = P.discount * value;
    r.delta = P.discount * a * c.spot_scale * f / spot;
    const double tvega = c.b * f * (-vol * t + sqrt(t) * z);
    r.vega = P.discount * a * tvega;
    return r;
}

__device__ __forceinline__ double exp_log_return(double vol, double t, double z) {
    const double tv = vol * vol * t;
    const double sd = sqrt(tv);
    return exp(-0.5 * tv + sd * z);
}

// The 10 risk components of one primary/mate path (pathwise_values).
__device__ __forceinline__ void single_terminal_values(const DevicePlan& P, const ProductParams& p,
                                                       double z, double* v) {
    const double e0 = exp_log_return(P.vol, P.expiry, z);
    const Aad base = single_terminal(P, p, P.spot, P.vol, z, e0);
    double gamma = 0.0;
    if (P.req_gamma) {
        const double b = P.gamma_bump;
        const Aad dn = single_terminal(P, p, P.spot - b, P.vol, z, e0);
        const Aad up = single_terminal(P, p, P.spot + b, P.vol, z, e0);
        gamma = (up.delta - dn.delta) / (2.0 * b);
    }
    const double sb = P.spot_bump;
    const Aad dn = single_terminal(P, p, P.spot - sb, P.vol, z, e0);
    const Aad up = single_terminal(P, p, P.spot + sb, P.vol, z, e0);
    const double bump_delta = (up.price - dn.price) / (2.0 * sb);
    const double bump_gamma = (up.price - 2.0 * base.price + dn.price) / (sb * sb);
    double bump_vega = 0.0;
    if (P.vol_bump != 0.0) {
        const double vb = P.vol_bump;
        const double vd = P.vol - vb, vu = P.vol + vb;
        const double a = single_terminal(P, p, P.spot, vd, z, exp_log_return(vd, P.expiry, z)).price;
        const double b = single_terminal(P, p, P.spot, vu, z, exp_log_return(vu, P.expiry, z)).price;
        bump_vega = (b - a) / (2.0 * vb);
    }
    v[MCG_PRICE] = base.price;
    v[MCG_DELTA] = base.delta;
    v[MCG_VEGA] = base.vega;
    v[MCG_GAMMA] = gamma;
    v[MCG_BUMP_DELTA] = bump_delta;
    v[MCG_DELTA_DIFFERENCE] = bump_delta - base.delta;
    v[MCG_BUMP_VEGA] = bump_vega;
    v[MCG_VEGA_DIFFERENCE] = bump_vega - base.vega;
    v[MCG_BUMP_GAMMA] = bump_gamma;
    v[MCG_GAMMA_DIFFERENCE] = bump_gamma - gamma;
}

// One 128-unit tile of the single-terminal path (European/Digital at expiry),
// price-only or risk: unit `point` of scramble `scramble` per thread, the
// CTA's statistics records written at tile_out[k * kComponents + c].
// unit_price (optional): receives the first product's discounted price of
// each unit (antithetic pairs averaged) at unit_price[point].
template <bool kRisk>
__device__ __forceinline__ void bs_terminal_tile(const DevicePlan& P, Stat* s_red, uint32_t scramble, uint64_t point,
                                                 bool valid, StatRecord* tile_out, uint32_t mask,
                                                 double* unit_price = nullptr) {
    const uint64_t unit = valid ? point : 0;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    const double z = P.zero_variance ? 0.0 : ns.normal(0);
    for (int k = 0; k < static_cast<int>(P.product_count); ++k) {
        const ProductParams& pp = P.products[k];
        double vals[kComponents];
#pragma unroll
        for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
        if constexpr (kRisk) {
            single_terminal_values(P, pp, z, vals);
            if (P.antithetic) {
                double mate[kComponents];
#pragma unroll
                for (int c = 0; c < kComponents; ++c) mate[c] = 0.0;
                single_terminal_values(P, pp, -z, mate);
#pragma unroll
                for (int c = 0; c < 10; ++c) vals[c] = (vals[c] + mate[c]) * 0.5;
            }
        } else {
            // discounted_payoff_from_normals, black_scholes.rs:41-55
            double a, pre;
            bool with_pre;
            const double t = P.expiry;
            const double tv = P.vol * P.vol * t;
            const double sd = sqrt(tv);
            const double f0 = P.obs_fwd[0] * 1.0 * exp(-0.5 * tv + sd * z);
            double price = P.discount * terminal_payoff(pp, obs_spot(P, 0, P.spot, f0, pre, with_pre), P.smoothing, a);
            if (P.antithetic) {
                const double f1 = P.obs_fwd[0] * 1.0 * exp(-0.5 * tv + sd * -z);
                const double mate =
                    P.discount * terminal_payoff(pp, obs_spot(P, 0, P.spot, f1, pre, with_pre), P.smoothing, a);
                price = (price + mate) * 0.5;
            }
            vals[MCG_PRICE] = price;
        }
        if (unit_price != nullptr && k == 0 && valid) unit_price[point] = vals[MCG_PRICE];
        cta_reduce_write<kComponents>(vals, valid, mask, tile_out + static_cast<size_t>(k) * kComponents, s_red);
    }
}


// One 128-unit tile of a multi-observation path, price and barrier
// diagnostics (NP products), records at tile_out[k * kComponents + c].  With
// s_z / s_zlist (z_batch<1>() x kThreads doubles, 32 x z_batch<1>() entries
// per warp) the normals are formed eight at a time per thread with AS241's
// tail branch compacted across the warp (fill_normals); without them one at a
// time.  Either way the CTA's threads call it together.  EV: the path's
// evolutions, 1, or 2 with its antithetic mate (P.antithetic), so the state
// of both stays in registers.
template <int NP, int EV>
__device__ __forceinline__ void bs_path_tile(const DevicePlan& P, Stat* s_red, uint32_t scramble, uint64_t point,
                                             bool valid, StatRecord* tile_out, uint32_t mask, ErrorWord* err,
                                             int detail, double* unit_price = nullptr, double* s_z = nullptr,
                                             uint16_t* s_zlist = nullptr) {
    const uint64_t unit = valid ? point : 0;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    constexpr int pairs = EV;
    double wsum[2] = {0.0, 0.0};
    double prev_f[2] = {P.spot, P.spot};
    ProductAcc acc[2][NP];
    bool failed = false;
    const double var = P.vol * P.vol;
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            acc_init(acc[e][k], P.products[k]);
            if (k < static_cast<int>(P.product_count) &&
                P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
                barrier_begin(P.products[k], acc[e][k], P.smoothing, P.spot, failed);
        }
    double prev_t = 0.0;
    const uint32_t n = P.observation_count;
    const bool batched = s_z != nullptr && !P.zero_variance;
    NormalSource nsq[1] = {ns};
    uint32_t zbase = 0, zend = 0;
    for (uint32_t i = 0; i < n; ++i) {
        double z;
        if (batched) {
            if (i == zend) {
                zbase = i;
                const uint32_t cnt = n - i < static_cast<uint32_t>(z_batch<1>()) ? n - i : z_batch<1>();
                fill_normals<1>(nsq, false, i, cnt, s_z, s_zlist, nullptr);
                zend = i + cnt;
            }
            z = s_z[(i - zbase) * kThreads + threadIdx.x];
        } else {
            z = P.zero_variance ? 0.0 : ns.normal(i);
        }
        const double t = P.obs_time[i];
        const double tv = P.vol * P.vol * t;
        const double dt = t - prev_t;
        prev_t = t;
#pragma unroll
        for (int e = 0; e < pairs; ++e) {
            const double ze = e == 0 ? z : -z;
            wsum[e] += P.obs_sqrt_step[i] * ze;
            const double f = P.obs_fwd[i] * 1.0 * exp(-0.5 * tv + P.vol * wsum[e]);
            double pre[1];
            bool with_pre;
            const double spot[1] = {obs_spot(P, i, P.spot, f, pre[0], with_pre)};
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                if (k >= static_cast<int>(P.product_count)) continue;
                if (P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
                    barrier_interval(P.products[k], acc[e][k], P.smoothing, prev_f[e], f, var, var,
                                     dt, failed);
                } else {
                    ProductAcc one[1] = {acc[e][k]};
                    acc_observe_n<1>(P.products[k], one, i, spot, P.smoothing, pre, with_pre);
                    acc[e][k] = one[0];
                }
            }
            prev_f[e] = f;
        }
    }
    if (valid && failed) report_error(err, unit, MCG_ERR_BARRIER_BRIDGE, 0, 0.0, detail);
    for (int k = 0; k < static_cast<int>(P.product_count) && k < NP; ++k) {
        const ProductParams& pp = P.products[k];
        double vals[kComponents];
#pragma unroll
        for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
#pragma unroll
        for (int e = 0; e < pairs; ++e) {
            double comp[kComponents];
#pragma unroll
            for (int c = 0; c < kComponents; ++c) comp[c] = 0.0;
            if (pp.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
                double diag[8];
                const double surv = barrier_finish(acc[e][k], P.smoothing, n, diag);
                comp[MCG_PRICE] = P.discount * barrier_value(pp, prev_f[e], surv);
#pragma unroll
                for (int q = 0; q < 8; ++q) comp[10 + q] = diag[q];
            } else {
                comp[MCG_PRICE] = P.discount * acc_payoff(pp, acc[e][k], P.smoothing);
            }
            if (e == 0) {
#pragma unroll
                for (int c = 0; c < kComponents; ++c) vals[c] = comp[c];
            } else {
#pragma unroll
                for (int c = 0; c < kComponents; ++c) vals[c] = (vals[c] + comp[c]) * 0.5;
            }
        }
        if (unit_price != nullptr && k == 0 && valid) unit_price[point] = vals[MCG_PRICE];
        cta_reduce_write<kComponents>(vals, valid, mask, tile_out + static_cast<size_t>(k) * kComponents, s_red);
    }
}


}  // namespace mcg

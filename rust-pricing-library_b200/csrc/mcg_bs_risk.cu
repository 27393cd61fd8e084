// mcg_bs_risk.cu -- Black--Scholes pathwise risk of multi-observation
// products (FP64, compiled with -fmad=false).
//
// pathwise_values (crates/pricing/src/engine/processes/black_scholes.rs:417-472)
// evaluates pathwise_aad (:476-563) at the base point and six bumped points:
// spot -/+ the gamma bump (Gamma as the central difference of the adjoint
// Deltas), spot -/+ the validation bump and volatility -/+ the validation
// bump (the bump-and-revalue checks).  Each evaluation rebuilds the
// observations of path_observations_from_normals (:297-331) from the same
// cumulative Brownian values W_k, runs the product's payoff forward and pulls
// dPayoff/dS_k back through the payoff graph (payoff/tape.rs:594-781 reverse
// semantics): Delta = sum_k adj_k f_k / S and Vega = sum_k adj_k f_k
// (-sigma t_k + W_k), summed from the last observation down as the tape
// reverse pushes them.  The continuous barrier assembles its state adjoints
// from the bridge intervals (:648-753) and adds the variance adjoint
// 2 sigma sum dlog q / dv.
//
// One thread per sampling unit.  W_k is independent of spot and volatility,
// and the antithetic mate's is its exact negation, so each unit computes it
// once into the per-thread scratch tape ([k][thread], coalesced) and all
// fourteen evaluations read it back; a smoothed discrete barrier also keeps
// its hit states, weights and weight slopes there for the reverse sweep, a
// continuous barrier its observed states.
#include "mcg_bs_tile.cuh"

namespace mcg {

namespace {

struct PathAad {
    double price, delta, vega;
};

// Per-thread scratch rows ([row][thread], `stride` threads apart): the
// cumulative Brownian values W_k of the primary path, the exponentials
// exp(-sigma^2 t_k / 2 + sigma W_k) of the path being evaluated at the plan's
// volatility, and the product's extra rows.
struct Scratch {
    const double* w;
    double* e;
    double* x;
    size_t stride;
};

// Spot at observation k of the path with sign `sign` (antithetic mate -1):
// F_k (S/S0) exp(-sigma^2 t_k / 2 + sigma W_k).  The five evaluations at the
// plan's volatility read the exponential from the scratch (the same value the
// expression gives), only the two volatility bumps evaluate it.
__device__ __forceinline__ double observe(const DevicePlan& P, const Scratch& T, uint32_t k, double sign,
                                          double scale, double vol, bool cached, double& w) {
    const size_t at = static_cast<size_t>(k) * T.stride;
    w = sign * T.w[at];
    if (cached) return P.obs_fwd[k] * scale * T.e[at];
    const double tv = vol * vol * P.obs_time[k];
    return P.obs_fwd[k] * scale * exp(-0.5 * tv + vol * w);
}

// pathwise_aad of a discrete product (European, Digital, Asian, lookback,
// discrete barrier) on one path.
__device__ __forceinline__ PathAad discrete_aad(const DevicePlan& P, const ProductParams& pp, const Scratch& T,
                                                double sign, double spot, double vol, bool cached, bool& failed) {
    const uint32_t n = P.observation_count;
    double* h_tape = T.x;
    const size_t stride = T.stride;
    const double scale = spot / P.spot;
    const double h = P.smoothing;
    const bool call = pp.side == MCG_CALL;
    const bool smooth_barrier = pp.kind == MCG_PRODUCT_DISCRETE_BARRIER && h > 0.0;
    ProductAcc acc;
    acc_init(acc, pp);
    int32_t arg = -1;  // lookback: observation holding the extremum (-1: the seasoned literal)
    // With dividends a smoothed barrier also keeps, per observation, the shares
    // of the pre- and post-dividend distances in the smooth maximum.
    double* share_tape = h_tape + 3 * static_cast<size_t>(n) * stride;
    for (uint32_t k = 0; k < n; ++k) {
        double w;
        const double f = observe(P, T, k, sign, scale, vol, cached, w);
        double pre[1];
        bool with_pre;
        const double sk[1] = {obs_spot(P, k, spot, f, pre[0], with_pre)};
        if (pp.kind == MCG_PRODUCT_LOOKBACK && monitored(pp, k) &&
            (acc.counts == 0u || (call ? !(acc.a >= sk[0]) : !(acc.a <= sk[0]))))
            arg = static_cast<int32_t>(k);
        if (smooth_barrier) {
            // hit state before k, hit weight and its slope (compile.rs:204-403)
            double weight = 0.0, first = 0.0, pre_share = 0.0, post_share = 1.0;
            if (monitored(pp, k)) {
                const bool upb = pp.barrier_direction == MCG_BARRIER_UP;
                double dist = upb ? sk[0] - pp.barrier : pp.barrier - sk[0];
                if (with_pre) {
                    const double pd = upb ? pre[0] - pp.barrier : pp.barrier - pre[0];
                    dist = smooth_maximum(h, pd, dist, pre_share, post_share);
                }
                double comp;
                const SmoothD d = smooth_indicator(h, dist, comp);
                weight = d.value;
                first = d.first;
            }
            h_tape[(3 * static_cast<size_t>(k) + 0) * stride] = acc.a;
            h_tape[(3 * static_cast<size_t>(k) + 1) * stride] = weight;
            h_tape[(3 * static_cast<size_t>(k) + 2) * stride] = first;
            if (P.dividends) {
                share_tape[(2 * static_cast<size_t>(k) + 0) * stride] = pre_share;
                share_tape[(2 * static_cast<size_t>(k) + 1) * stride] = post_share;
            }
        }
        ProductAcc one[1] = {acc};
        acc_observe_n<1>(pp, one, k, sk, h, pre, with_pre);
        acc = one[0];
    }
    const double value = acc_payoff(pp, acc, h);
    // d payoff / d observed spot at the terminal observation and, for the
    // average-type products, the common factor of every observation's seed.
    double terminal_adj = 0.0, g = 0.0, a_hit = 0.0;
    const double term = acc.terminal;
    switch (pp.kind) {
    case MCG_PRODUCT_EUROPEAN: {
        const double in = call ? term - pp.strike : pp.strike - term;
        terminal_adj = (in >= 0.0 ? pp.notional : 0.0) * (call ? 1.0 : -1.0);
        break;
    }
    case MCG_PRODUCT_DIGITAL: {
        const double dist = call ? term - pp.strike : pp.strike - term;
        double ind, first = 0.0;
        if (h > 0.0) {
            double comp;
            const SmoothD dd = smooth_indicator(h, dist, comp);
            ind = dd.value;
            first = dd.first;
        } else {
            ind = dist >= 0.0 ? 1.0 : 0.0;
        }
        const bool asset = pp.digital_payout == MCG_DIGITAL_ASSET;
        const double base = asset ? term * pp.payout : pp.payout;
        double a = 0.0;
        if (asset) a += ind * pp.payout;
        if (h > 0.0) a += (call ? 1.0 : -1.0) * (base * first);
        terminal_adj = a;
        break;
    }
    case MCG_PRODUCT_ASIAN:
    case MCG_PRODUCT_LOOKBACK: {
        const double in = call ? acc.a - pp.strike : pp.strike - acc.a;
        g = (in >= 0.0 ? pp.notional : 0.0) * (call ? 1.0 : -1.0);
        break;
    }
    case MCG_PRODUCT_DISCRETE_BARRIER: {
        const double in = call ? term - pp.strike : pp.strike - term;
        const double vanilla = (in >= 0.0 ? in : 0.0) * pp.notional;
        const bool ko = pp.barrier_style == MCG_KNOCK_OUT;
        const double active = ko ? 1.0 - acc.a : acc.a;
        double a_active = vanilla;
        if (pp.has_rebate) a_active = a_active + (-pp.rebate);
        a_hit = ko ? -a_active : a_active;
        terminal_adj = (in >= 0.0 ? active * pp.notional : 0.0) * (call ? 1.0 : -1.0);
        break;
    }
    default:
        break;
    }
    // Reverse sweep, last observation first (the order the tape reverse
    // pushes the terminal adjoints); the pre-dividend adjoints of a barrier's
    // ex-dates follow them (black_scholes.rs:525-562).
    double delta = 0.0, vega = 0.0, delta_pre = 0.0, vega_pre = 0.0;
    const double up_sign = pp.barrier_direction == MCG_BARRIER_UP ? 1.0 : -1.0;
    for (int32_t k = static_cast<int32_t>(n) - 1; k >= 0; --k) {
        double adj = 0.0, pre_adj = 0.0;
        switch (pp.kind) {
        case MCG_PRODUCT_ASIAN:
            adj = g * pp.weights[k];
            break;
        case MCG_PRODUCT_LOOKBACK:
            adj = k == arg ? g : 0.0;
            break;
        case MCG_PRODUCT_DISCRETE_BARRIER:
            if (smooth_barrier) {
                const double hist = h_tape[(3 * static_cast<size_t>(k) + 0) * stride];
                const double weight = h_tape[(3 * static_cast<size_t>(k) + 1) * stride];
                const double first = h_tape[(3 * static_cast<size_t>(k) + 2) * stride];
                const double a_w = a_hit * (1.0 - hist);
                a_hit = a_hit * (1.0 - weight);
                if (P.dividends) {
                    const double a_dist = a_w * first;
                    adj += up_sign * (a_dist * share_tape[(2 * static_cast<size_t>(k) + 1) * stride]);
                    pre_adj = up_sign * (a_dist * share_tape[(2 * static_cast<size_t>(k) + 0) * stride]);
                } else {
                    adj += up_sign * (a_w * first);
                }
            }
            if (k == static_cast<int32_t>(n) - 1) adj += terminal_adj;
            break;
        default:
            if (k == static_cast<int32_t>(n) - 1) adj = terminal_adj;
            break;
        }
        if (adj == 0.0 && pre_adj == 0.0) continue;
        double w;
        const double f = observe(P, T, static_cast<uint32_t>(k), sign, scale, vol, cached, w);
        if (adj != 0.0) {
            const DivCoord c = obs_coord(P, static_cast<uint32_t>(k), spot);
            delta += adj * c.spot_scale * f / spot;
            vega += adj * c.b * f * (-vol * P.obs_time[k] + w);
        }
        if (pre_adj != 0.0) {
            const DivCoord c = div_at_spot(P.obs_div_pre[k], P.spot, spot);
            delta_pre += pre_adj * c.spot_scale * f / spot;
            vega_pre += pre_adj * c.b * f * (-vol * P.obs_time[k] + w);
        }
    }
    if (P.dividends) {
        delta += delta_pre;
        vega += vega_pre;
    }
    PathAad r;
    r.price = P.discount * value;
    r.delta = P.discount * delta;
    r.vega = P.discount * vega;
    return r;
}

// pathwise_aad of a continuous barrier: the bridge over [0, t_1], ..., and
// its adjoint (black_scholes.rs:94-293, 648-753); diag receives components
// 10..17 of the evaluation.  Scratch rows: f_k at [0, n) of `f_tape`.  Each
// node's bridge endpoint is evaluated once per sweep and shared by the two
// intervals that meet there.
template <bool kSmooth>
__device__ __forceinline__ PathAad continuous_aad(const DevicePlan& P, const ProductParams& pp, const Scratch& T,
                                                  double sign, double spot, double vol, bool cached, double* diag,
                                                  bool& failed) {
    const uint32_t n = P.observation_count;
    double* f_tape = T.x;
    const size_t stride = T.stride;
    const double* w_tape = T.w;
    const double scale = spot / P.spot;
    // The launch picks the instantiation by the plan's smoothing width (> 0:
    // smoothed, 0: exact), so each compiles one form of the bridge.
    const double h = kSmooth ? P.smoothing : 0.0;
    if constexpr (kSmooth) __builtin_assume(h > 0.0);
    const double var = vol * vol;
    const bool up = pp.barrier_direction == MCG_BARRIER_UP;
    const double B = pp.barrier;
    ProductAcc acc;
    acc_init(acc, pp);
    double ld = 0.0, lld = 0.0;  // smoothed: the left endpoint's effective log distance and its log
    if (h > 0.0) {
        double safety;
        smooth_endpoint(up, spot, B, h, safety, ld, failed);
        lld = log(ld);
        acc.hit_log = 0.0 + log(safety);
        acc.hit_prod = 1.0 * safety;
    } else {
        barrier_begin(pp, acc, h, spot, failed);
    }
    double prev_f = spot, prev_t = 0.0, f = spot, w_last = 0.0;
    for (uint32_t k = 0; k < n; ++k) {
        double w;
        f = observe(P, T, k, sign, scale, vol, cached, w);
        w_last = w;
        f_tape[static_cast<size_t>(k) * stride] = f;
        const double t = P.obs_time[k];
        const double dt = t - prev_t;
        if (h > 0.0) {
            // barrier_interval with the left endpoint carried over
            double rsafe, rd, log_surv;
            smooth_endpoint(up, f, B, h, rsafe, rd, failed);
            const double lrd = log(rd);
            if (dt > 0.0) {
                const int status = smooth_interval(ld, rd, lld, lrd, var, var, dt, log_surv, failed);
                if (rsafe != 1.0) {  // log(1) = +0 leaves the hit factor unchanged
                    acc.hit_log = acc.hit_log + log(rsafe);
                    acc.hit_prod = acc.hit_prod * rsafe;
                }
                acc.log_sum += log_surv;
                count_status(acc, status);
            }
            ld = rd;
            lld = lrd;
        } else {
            barrier_interval(pp, acc, h, prev_f, f, var, var, dt, failed);
        }
        prev_f = f;
        prev_t = t;
    }
    const double surv = barrier_finish(acc, h, n, diag);
    // continuous_barrier_payoff_terms (barrier.rs:307-355)
    const bool call = pp.side == MCG_CALL;
    const double in = call ? f - pp.strike : pp.strike - f;
    const double vanilla = fmax(in, 0.0) * pp.notional;
    const double vd = in >= 0.0 ? (call ? 1.0 : -1.0) * pp.notional : 0.0;
    const double rebate = pp.has_rebate ? pp.rebate : 0.0;
    double value, td, sd;
    if (pp.barrier_style == MCG_KNOCK_OUT) {
        value = rebate + surv * (vanilla - rebate);
        td = surv * vd;
        sd = vanilla - rebate;
    } else {
        value = vanilla + surv * (rebate - vanilla);
        td = (1.0 - surv) * vd;
        sd = rebate - vanilla;
    }
    const bool exact_active = !(acc.initial_touched || acc.touched);
    const bool flows = h > 0.0 || exact_active;
    const double lsa = sd * surv;
    // One sweep over the intervals: the variance adjoint in interval order and
    // sa_k = ((0 + right part of interval k-1) + left part of interval k)
    // + the smoothed hit factor at k; the terminal seed enters sa_n first.
    // Each sa_k is final when its interval is done, so the sweep also takes the
    // state adjoint's Delta term sa_k f_{k-1} / S and Vega term
    // sa_k f_{k-1} (-sigma t_{k-1} + W_{k-1}) of the node before it (delta
    // starts from sa_0); the Vega terms are summed apart from the variance
    // adjoint's 2 sigma var_adj, which is complete only after the sweep.
    double var_adj = 0.0;
    double delta = 0.0, vega_terms = 0.0;
    if (flows) {
        double carry = n == 0 ? 0.0 + td * 1.0 : 0.0;  // sa of the next node before its left part
        // Each node's bridge quantities are computed once and carried into the next interval.
        const double lb = h > 0.0 ? 0.0 : log(B);
        BarrierEndpoint nl = barrier_endpoint(up, B, lb, h, spot);
        prev_f = spot;
        prev_t = 0.0;
        double prev_w = 0.0;
        for (uint32_t k = 0; k < n; ++k) {
            const double fk = f_tape[static_cast<size_t>(k) * stride];
            const double wk = sign * w_tape[static_cast<size_t>(k) * stride];
            const double t = P.obs_time[k];
            const double dt = t - prev_t;
            const BarrierEndpoint nr = barrier_endpoint(up, B, lb, h, fk);
            const IntervalAdjoint ia = bridge_interval_adjoint(up, h, lsa, nl, nr, prev_f, fk, var, var, dt);
            var_adj += ia.left_var + ia.right_var;
            double sa = carry + ia.left_state;
            if (h > 0.0) sa += hit_factor_adjoint(nl, lsa);
            if (k == 0) {
                delta = sa;
            } else {
                delta += sa * prev_f / spot;
                vega_terms += sa * prev_f * (-vol * prev_t + prev_w);
            }
            carry = (k + 1 == n) ? (0.0 + td * 1.0) + ia.right_state : 0.0 + ia.right_state;
            nl = nr;
            prev_f = fk;
            prev_w = wk;
            prev_t = t;
        }
        if (h > 0.0) carry += hit_factor_adjoint(nl, lsa);
        if (n == 0) {
            delta = carry;
        } else {
            delta += carry * prev_f / spot;
            vega_terms += carry * prev_f * (-vol * prev_t + prev_w);
        }
    } else {
        // No flow through the bridge: every sa_k is 0 but the terminal's.
        const double carry = 0.0 + td * 1.0;
        if (n == 0) {
            delta = carry;
        } else {
            delta = carry * f / spot;
            vega_terms = carry * f * (-vol * P.obs_time[n - 1] + w_last);
        }
    }
    const double vega = 2.0 * vol * var_adj + vega_terms;
    PathAad r;
    r.price = P.discount * value;
    r.delta = P.discount * delta;
    r.vega = P.discount * vega;
    return r;
}

// kCont: 0 no continuous barrier, 1 exact continuous barrier, 2 smoothed.
template <int kCont>
__device__ __forceinline__ PathAad path_aad(const DevicePlan& P, const ProductParams& pp, const Scratch& T,
                                            double sign, double spot, double vol, bool cached, double* diag,
                                            bool& failed) {
    if constexpr (kCont != 0)
        return continuous_aad<kCont == 2>(P, pp, T, sign, spot, vol, cached, diag, failed);
    else
        return discrete_aad(P, pp, T, sign, spot, vol, cached, failed);
}

// The components of one primary or mate path (pathwise_values, :417-472).
// The seven evaluations run in one loop over (spot, volatility) points, so the
// evaluation body is instantiated once.
template <int kCont>
__device__ __forceinline__ void path_values(const DevicePlan& P, const ProductParams& pp, const Scratch& T,
                                            double sign, double* v, bool& failed) {
    // the exponentials of this path at the plan's volatility
    for (uint32_t k = 0; k < P.observation_count; ++k) {
        const size_t at = static_cast<size_t>(k) * T.stride;
        const double tv = P.vol * P.vol * P.obs_time[k];
        T.e[at] = exp(-0.5 * tv + P.vol * (sign * T.w[at]));
    }
    double diag[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double scratch[8];
    const double b = P.gamma_bump, sb = P.spot_bump, vb = P.vol_bump;
    // base, gamma down/up, validation spot down/up, validation volatility down/up
    const double spots[7] = {P.spot, P.spot - b, P.spot + b, P.spot - sb, P.spot + sb, P.spot, P.spot};
    const double vols[7] = {P.vol, P.vol, P.vol, P.vol, P.vol, P.vol - vb, P.vol + vb};
    PathAad r[7];
    auto evaluate = [&](int i) {
        r[i] = PathAad{0.0, 0.0, 0.0};
        if ((i == 1 || i == 2) && !P.req_gamma) return;
        if (i >= 5 && P.vol_bump == 0.0) return;
        r[i] = path_aad<kCont>(P, pp, T, sign, spots[i], vols[i], i < 5, i == 0 ? diag : scratch, failed);
    };
    if constexpr (kCont) {
        // one copy of the (large) bridge body
#pragma unroll 1
        for (int i = 0; i < 7; ++i) evaluate(i);
    } else {
#pragma unroll
        for (int i = 0; i < 7; ++i) evaluate(i);
    }
    const PathAad base = r[0];
    const double gamma = P.req_gamma ? (r[2].delta - r[1].delta) / (2.0 * b) : 0.0;
    const double bump_delta = (r[4].price - r[3].price) / (2.0 * sb);
    const double bump_gamma = (r[4].price - 2.0 * base.price + r[3].price) / (sb * sb);
    const double bump_vega = vb != 0.0 ? (r[6].price - r[5].price) / (2.0 * vb) : 0.0;
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
#pragma unroll
    for (int q = 0; q < 8; ++q) v[10 + q] = kCont ? diag[q] : 0.0;
}

}  // namespace

// One thread per unit of [unit_begin, unit_end); CTA records of tile
// unit/128 of scramble blockIdx.y.  The continuous-barrier forms run 5 CTAs
// per SM (96 registers; at 4 CTAs and 125 registers the smoothed barrier took
// 204 against 184 ms at 2^20 paths).
template <int kCont>
__global__ void __launch_bounds__(kThreads, kCont ? 5 : 6) bs_path_risk_kernel(const DevicePlan P, uint64_t unit_begin,
                                                                uint64_t unit_end, StatRecord* partials,
                                                                uint32_t mask, ErrorWord* err, int detail) {
    __shared__ Stat s_red[4 * kComponents];
    __shared__ double s_z[z_batch<1>() * kThreads];                    // batched normals [k][thread]
    __shared__ uint16_t s_zlist[(kThreads / 32) * 32 * z_batch<1>()];  // tail lists, per warp
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < unit_end && point < P.units;
    const uint64_t unit = valid ? point : 0;
    const size_t stride = static_cast<size_t>(gridDim.x) * gridDim.y * kThreads;
    const size_t local = (static_cast<size_t>(blockIdx.y) * gridDim.x + blockIdx.x) * kThreads + threadIdx.x;
    const size_t n = P.observation_count;
    double* w_tape = P.bs_tape + local;
    const Scratch T{w_tape, P.bs_tape + n * stride + local, P.bs_tape + 2 * n * stride + local, stride};
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    // The path's normals, dimension k at observation k, eight at a time with
    // AS241's tail branch compacted across the warp (fill_normals); every
    // thread of the CTA walks the same observations.
    NormalSource nsq[1] = {ns};
    uint32_t zbase = 0, zend = 0, zi = 0;
    auto next_normal = [&]() -> double {
        if (zi == zend) {
            zbase = zi;
            constexpr uint32_t kBatch = static_cast<uint32_t>(z_batch<1>());
            const uint32_t cnt = P.observation_count - zi < kBatch ? P.observation_count - zi : kBatch;
            fill_normals<1>(nsq, false, zi, cnt, s_z, s_zlist, nullptr);
            zend = zi + cnt;
        }
        const uint32_t kk = zi++ - zbase;
        return s_z[kk * kThreads + threadIdx.x];
    };
    // W_k of the primary path (path_observations_from_normals, :297-331)
    double w = 0.0;
    for (uint32_t k = 0; k < P.observation_count; ++k) {
        const double z = P.zero_variance ? 0.0 : next_normal();
        w += P.obs_sqrt_step[k] * z;
        w_tape[static_cast<size_t>(k) * stride] = w;
    }
    const ProductParams& pp = P.products[0];
    bool failed = false;
    double vals[kComponents];
    path_values<kCont>(P, pp, T, 1.0, vals, failed);
    if (P.antithetic) {
        double mate[kComponents];
        path_values<kCont>(P, pp, T, -1.0, mate, failed);
#pragma unroll
        for (int c = 0; c < kComponents; ++c) vals[c] = (vals[c] + mate[c]) * 0.5;
    }
    if (valid && failed) report_error(err, unit, MCG_ERR_BARRIER_BRIDGE, 0, 0.0, detail);
    const uint64_t tiles = (P.units + kThreads - 1) / kThreads;
    const uint64_t tile = (unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads) / kThreads;
    StatRecord* tile_out = partials + (static_cast<size_t>(scramble) * tiles + tile) * kComponents;
    cta_reduce_write<kComponents>(vals, valid, mask, tile_out, s_red);
}

// Single-sweep form of pathwise_values for the products whose adjoint seeds
// need no reverse pass over the path: European, Digital and an exact discrete
// barrier seed only the terminal observation, a lookback only the observation
// holding its extremum, an Asian every observation with weight_k times a
// factor g that is either 0 or +-notional (in or out of the money at the end).
// The seven (spot, volatility) evaluations of both antithetic signs therefore
// run in one forward loop over the observations with no scratch tape: per
// observation one normal, W_k, the exponential at the plan's volatility per
// sign (shared by the five spot points, whose observations are
// F_k (S/S0) e_k as above) and the two volatility-bump exponentials; the
// Asian adjoint sums carry the seed with g = +-notional and are dropped when
// g is 0; the lookback keeps the extremum's observation.  Each term is the
// reference's ((adj spot_scale) f_k) / S and ((adj b) f_k)(-sigma t_k + W_k);
// only the Asian sums add them in observation order instead of the reverse.
// Plans without dividends; a smoothed discrete barrier (whose hit weights do
// need the reverse pass) and a continuous barrier use the tape kernel.
// Occupancy: 5 CTAs per SM without the mate (Asian, 2^20 x 252: 5.49 against
// 5.62 ms at 4), 2 with it (at 4 the antithetic Asian took 14.4 against 12.3 ms).
template <bool kAnti>
__global__ void __launch_bounds__(kThreads, kAnti ? 2 : 5) bs_path_sweep_kernel(const DevicePlan P, uint64_t unit_begin,
                                                                  uint64_t unit_end, StatRecord* partials,
                                                                  uint32_t mask, ErrorWord* err, int detail) {
    (void)err;
    (void)detail;
    __shared__ Stat s_red[4 * kComponents];
    __shared__ double s_z[z_batch<1>() * kThreads];                    // batched normals [k][thread]
    __shared__ uint16_t s_zlist[(kThreads / 32) * 32 * z_batch<1>()];  // tail lists, per warp
    constexpr int S = kAnti ? 2 : 1;  // path signs: primary and antithetic mate
    constexpr int N = 7 * S;          // evaluation i of sign s at 7 s + i
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < unit_end && point < P.units;
    const uint64_t unit = valid ? point : 0;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    const ProductParams& pp = P.products[0];
    const uint32_t n = P.observation_count;
    const double h = P.smoothing;
    const bool call = pp.side == MCG_CALL;
    const bool asian = pp.kind == MCG_PRODUCT_ASIAN;
    const bool lookback = pp.kind == MCG_PRODUCT_LOOKBACK;
    const double b = P.gamma_bump, sb = P.spot_bump, vb = P.vol_bump;
    const bool vbump = vb != 0.0;
    // base, gamma down/up, validation spot down/up, validation volatility down/up
    const double spots[7] = {P.spot, P.spot - b, P.spot + b, P.spot - sb, P.spot + sb, P.spot, P.spot};
    const double vols[7] = {P.vol, P.vol, P.vol, P.vol, P.vol, P.vol - vb, P.vol + vb};
    double scale[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) scale[i] = spots[i] / P.spot;
    const double gstar = pp.notional * (call ? 1.0 : -1.0);
    ProductAcc acc[N];
#pragma unroll
    for (int j = 0; j < N; ++j) acc_init(acc[j], pp);
    // adjoint sums of the base and gamma points (Asian), the extremum's
    // observation (lookback: its spot per point, W and time for the base Vega)
    double ad[3 * S], av[S], fa[3 * S], wa[S], ta[S];
    bool has_arg[3 * S];
#pragma unroll
    for (int j = 0; j < 3 * S; ++j) {
        ad[j] = 0.0;
        fa[j] = 0.0;
        has_arg[j] = false;
    }
#pragma unroll
    for (int s = 0; s < S; ++s) av[s] = wa[s] = ta[s] = 0.0;
    // The path's normals, dimension k at observation k, eight at a time with
    // AS241's tail branch compacted across the warp (fill_normals); every
    // thread of the CTA walks the same observations.
    NormalSource nsq[1] = {ns};
    uint32_t zbase = 0, zend = 0, zi = 0;
    auto next_normal = [&]() -> double {
        if (zi == zend) {
            zbase = zi;
            constexpr uint32_t kBatch = static_cast<uint32_t>(z_batch<1>());
            const uint32_t cnt = P.observation_count - zi < kBatch ? P.observation_count - zi : kBatch;
            fill_normals<1>(nsq, false, zi, cnt, s_z, s_zlist, nullptr);
            zend = zi + cnt;
        }
        const uint32_t kk = zi++ - zbase;
        return s_z[kk * kThreads + threadIdx.x];
    };
    double w = 0.0, wlast[S], sk[N];
#pragma unroll
    for (int j = 0; j < N; ++j) sk[j] = 0.0;
    for (uint32_t k = 0; k < n; ++k) {
        const double z = P.zero_variance ? 0.0 : next_normal();
        w += P.obs_sqrt_step[k] * z;
        const double t = P.obs_time[k];
        const double F = P.obs_fwd[k];
        const double tv = P.vol * P.vol * t;
        const bool mon = lookback && monitored(pp, k);
        const double wg = asian ? pp.weights[k] : 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double ws = (s == 0 ? 1.0 : -1.0) * w;
            wlast[s] = ws;
            const double e = exp(-0.5 * tv + P.vol * ws);
#pragma unroll
            for (int i = 0; i < 5; ++i) sk[7 * s + i] = F * scale[i] * e;
            if (vbump) {
#pragma unroll
                for (int i = 5; i < 7; ++i) {
                    const double tvb = vols[i] * vols[i] * t;
                    sk[7 * s + i] = F * 1.0 * exp(-0.5 * tvb + vols[i] * ws);
                }
            }
            if (asian) {
                const double a = (gstar * wg) * 1.0;
#pragma unroll
                for (int i = 0; i < 3; ++i) ad[3 * s + i] += a * sk[7 * s + i] / spots[i];
                av[s] += a * 1.0 * sk[7 * s] * (-P.vol * t + ws);
            }
            if (mon) {
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const ProductAcc& q = acc[7 * s + i];
                    const double x = sk[7 * s + i];
                    if (q.counts == 0u || (call ? !(q.a >= x) : !(q.a <= x))) {
                        fa[3 * s + i] = x;
                        has_arg[3 * s + i] = true;
                        if (i == 0) {
                            wa[s] = ws;
                            ta[s] = t;
                        }
                    }
                }
            }
        }
        acc_observe_n<N, false>(pp, acc, k, sk, h, sk, false);
    }
    const double t_last = n ? P.obs_time[n - 1] : 0.0;
    double vals[kComponents];
#pragma unroll
    for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        PathAad r[7];
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            r[i] = PathAad{0.0, 0.0, 0.0};
            if ((i == 1 || i == 2) && !P.req_gamma) continue;
            if (i >= 5 && !vbump) continue;
            const ProductAcc& q = acc[7 * s + i];
            const double value = acc_payoff(pp, q, h);
            double delta = 0.0, vega = 0.0;
            if (i < 3) {
                // the seed of this point (discrete_aad's switch) and its pull-back
                double terminal_adj = 0.0, g = 0.0;
                const double term = q.terminal;
                switch (pp.kind) {
                case MCG_PRODUCT_EUROPEAN: {
                    const double in = call ? term - pp.strike : pp.strike - term;
                    terminal_adj = (in >= 0.0 ? pp.notional : 0.0) * (call ? 1.0 : -1.0);
                    break;
                }
                case MCG_PRODUCT_DIGITAL: {
                    const double dist = call ? term - pp.strike : pp.strike - term;
                    double ind, first = 0.0;
                    if (h > 0.0) {
                        double comp;
                        const SmoothD dd = smooth_indicator(h, dist, comp);
                        ind = dd.value;
                        first = dd.first;
                    } else {
                        ind = dist >= 0.0 ? 1.0 : 0.0;
                    }
                    const bool asset = pp.digital_payout == MCG_DIGITAL_ASSET;
                    const double base = asset ? term * pp.payout : pp.payout;
                    double a = 0.0;
                    if (asset) a += ind * pp.payout;
                    if (h > 0.0) a += (call ? 1.0 : -1.0) * (base * first);
                    terminal_adj = a;
                    break;
                }
                case MCG_PRODUCT_ASIAN:
                case MCG_PRODUCT_LOOKBACK: {
                    const double in = call ? q.a - pp.strike : pp.strike - q.a;
                    g = (in >= 0.0 ? pp.notional : 0.0) * (call ? 1.0 : -1.0);
                    break;
                }
                case MCG_PRODUCT_DISCRETE_BARRIER: {
                    const double in = call ? term - pp.strike : pp.strike - term;
                    const double active = pp.barrier_style == MCG_KNOCK_OUT ? 1.0 - q.a : q.a;
                    terminal_adj = (in >= 0.0 ? active * pp.notional : 0.0) * (call ? 1.0 : -1.0);
                    break;
                }
                default:
                    break;
                }
                if (asian) {
                    if (g != 0.0) {
                        delta = ad[3 * s + i];
                        if (i == 0) vega = av[s];
                    }
                } else if (lookback) {
                    if (g != 0.0 && has_arg[3 * s + i]) {
                        delta = g * 1.0 * fa[3 * s + i] / spots[i];
                        if (i == 0) vega = g * 1.0 * fa[3 * s] * (-P.vol * ta[s] + wa[s]);
                    }
                } else if (terminal_adj != 0.0 && n > 0) {
                    delta = terminal_adj * 1.0 * term / spots[i];
                    if (i == 0) vega = terminal_adj * 1.0 * term * (-P.vol * t_last + wlast[s]);
                }
            }
            r[i] = PathAad{P.discount * value, P.discount * delta, P.discount * vega};
        }
        const double gamma = P.req_gamma ? (r[2].delta - r[1].delta) / (2.0 * b) : 0.0;
        const double bump_delta = (r[4].price - r[3].price) / (2.0 * sb);
        const double bump_gamma = (r[4].price - 2.0 * r[0].price + r[3].price) / (sb * sb);
        const double bump_vega = vb != 0.0 ? (r[6].price - r[5].price) / (2.0 * vb) : 0.0;
        double v[kComponents];
#pragma unroll
        for (int c = 0; c < kComponents; ++c) v[c] = 0.0;
        v[MCG_PRICE] = r[0].price;
        v[MCG_DELTA] = r[0].delta;
        v[MCG_VEGA] = r[0].vega;
        v[MCG_GAMMA] = gamma;
        v[MCG_BUMP_DELTA] = bump_delta;
        v[MCG_DELTA_DIFFERENCE] = bump_delta - r[0].delta;
        v[MCG_BUMP_VEGA] = bump_vega;
        v[MCG_VEGA_DIFFERENCE] = bump_vega - r[0].vega;
        v[MCG_BUMP_GAMMA] = bump_gamma;
        v[MCG_GAMMA_DIFFERENCE] = bump_gamma - gamma;
        if (s == 0) {
#pragma unroll
            for (int c = 0; c < kComponents; ++c) vals[c] = v[c];
        } else {
#pragma unroll
            for (int c = 0; c < kComponents; ++c) vals[c] = (vals[c] + v[c]) * 0.5;
        }
    }
    const uint64_t tiles = (P.units + kThreads - 1) / kThreads;
    const uint64_t tile = (unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads) / kThreads;
    StatRecord* tile_out = partials + (static_cast<size_t>(scramble) * tiles + tile) * kComponents;
    cta_reduce_write<kComponents>(vals, valid, mask, tile_out, s_red);
}

// Units are launched in chunks of at most P.bs_tape_units threads (all
// scrambles of a chunk in one launch), so the scratch tape stays bounded.
cudaError_t launch_bs_path_risk(const DevicePlan& P, uint64_t unit_begin, uint64_t units, uint32_t scrambles,
                                StatRecord* partials, uint32_t mask, ErrorWord* err, int detail,
                                cudaStream_t stream) {
    if (P.product_count != 1) return cudaErrorNotSupported;
    if (P.bs_sweep) {
        const dim3 grid(static_cast<unsigned>((units + kThreads - 1) / kThreads), scrambles);
        if (P.antithetic)
            bs_path_sweep_kernel<true><<<grid, kThreads, 0, stream>>>(P, unit_begin, unit_begin + units, partials,
                                                                      mask, err, detail);
        else
            bs_path_sweep_kernel<false><<<grid, kThreads, 0, stream>>>(P, unit_begin, unit_begin + units, partials,
                                                                       mask, err, detail);
        return cudaGetLastError();
    }
    if (!P.bs_tape) return cudaErrorNotSupported;
    const bool cont = P.products[0].kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
    const uint64_t per_launch = P.bs_tape_units / scrambles / kThreads * kThreads;
    if (per_launch == 0) return cudaErrorInvalidValue;
    const uint64_t end = unit_begin + units;
    for (uint64_t begin = unit_begin; begin < end; begin += per_launch) {
        const uint64_t n = end - begin < per_launch ? end - begin : per_launch;
        const dim3 grid(static_cast<unsigned>((n + kThreads - 1) / kThreads), scrambles);
        if (cont && P.smoothing > 0.0)
            bs_path_risk_kernel<2><<<grid, kThreads, 0, stream>>>(P, begin, begin + n, partials, mask, err, detail);
        else if (cont)
            bs_path_risk_kernel<1><<<grid, kThreads, 0, stream>>>(P, begin, begin + n, partials, mask, err, detail);
        else
            bs_path_risk_kernel<0><<<grid, kThreads, 0, stream>>>(P, begin, begin + n, partials, mask, err, detail);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace mcg

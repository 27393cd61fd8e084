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
// its hit states, weights and weight slopes there for the reverse sweep.
#include "mcg_kernels.cuh"

namespace mcg {

namespace {

struct PathAad {
    double price, delta, vega;
};

// Spot at observation k of the path with sign `sign` (antithetic mate -1).
__device__ __forceinline__ double observe(const DevicePlan& P, const double* w_tape, size_t stride,
                                          uint32_t k, double sign, double scale, double vol, double& w) {
    w = sign * w_tape[static_cast<size_t>(k) * stride];
    const double tv = vol * vol * P.obs_time[k];
    return P.obs_fwd[k] * scale * exp(-0.5 * tv + vol * w);
}

// pathwise_aad of a discrete product (European, Digital, Asian, lookback,
// discrete barrier) on one path.
__device__ PathAad discrete_aad(const DevicePlan& P, const ProductParams& pp, const double* w_tape,
                                double* h_tape, size_t stride, double sign, double spot, double vol,
                                bool& failed) {
    const uint32_t n = P.observation_count;
    const double scale = spot / P.spot;
    const double h = P.smoothing;
    const bool call = pp.side == MCG_CALL;
    const bool smooth_barrier = pp.kind == MCG_PRODUCT_DISCRETE_BARRIER && h > 0.0;
    ProductAcc acc;
    acc_init(acc, pp);
    int32_t arg = -1;  // lookback: observation holding the extremum (-1: the seasoned literal)
    for (uint32_t k = 0; k < n; ++k) {
        double w;
        const double f = observe(P, w_tape, stride, k, sign, scale, vol, w);
        if (pp.kind == MCG_PRODUCT_LOOKBACK && monitored(pp, k) &&
            (acc.counts == 0u || (call ? !(acc.a >= f) : !(acc.a <= f))))
            arg = static_cast<int32_t>(k);
        if (smooth_barrier) {
            // hit state before k, hit weight and its slope (compile.rs:204-403)
            double weight = 0.0, first = 0.0;
            if (monitored(pp, k)) {
                const double dist = pp.barrier_direction == MCG_BARRIER_UP ? f - pp.barrier : pp.barrier - f;
                double comp;
                const SmoothD d = smooth_indicator(h, dist, comp);
                weight = d.value;
                first = d.first;
            }
            h_tape[(3 * static_cast<size_t>(k) + 0) * stride] = acc.a;
            h_tape[(3 * static_cast<size_t>(k) + 1) * stride] = weight;
            h_tape[(3 * static_cast<size_t>(k) + 2) * stride] = first;
        }
        acc_observe(pp, acc, k, f, h, failed);
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
    // pushes the terminal adjoints).
    double delta = 0.0, vega = 0.0;
    const double up_sign = pp.barrier_direction == MCG_BARRIER_UP ? 1.0 : -1.0;
    for (int32_t k = static_cast<int32_t>(n) - 1; k >= 0; --k) {
        double adj = 0.0;
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
                adj += up_sign * (a_w * first);
            }
            if (k == static_cast<int32_t>(n) - 1) adj += terminal_adj;
            break;
        default:
            if (k == static_cast<int32_t>(n) - 1) adj = terminal_adj;
            break;
        }
        if (adj == 0.0) continue;
        double w;
        const double f = observe(P, w_tape, stride, static_cast<uint32_t>(k), sign, scale, vol, w);
        delta += adj * 1.0 * f / spot;
        vega += adj * 1.0 * f * (-vol * P.obs_time[k] + w);
    }
    PathAad r;
    r.price = P.discount * value;
    r.delta = P.discount * delta;
    r.vega = P.discount * vega;
    return r;
}

// pathwise_aad of a continuous barrier: the bridge over [0, t_1], ..., and
// its adjoint (black_scholes.rs:94-293, 648-753); diag receives components
// 10..17 of the evaluation.
__device__ PathAad continuous_aad(const DevicePlan& P, const ProductParams& pp, const double* w_tape,
                                  size_t stride, double sign, double spot, double vol, double* diag,
                                  bool& failed) {
    const uint32_t n = P.observation_count;
    const double scale = spot / P.spot;
    const double h = P.smoothing;
    const double var = vol * vol;
    const bool up = pp.barrier_direction == MCG_BARRIER_UP;
    ProductAcc acc;
    acc_init(acc, pp);
    barrier_begin(pp, acc, h, spot, failed);
    double prev_f = spot, prev_t = 0.0, f = spot;
    for (uint32_t k = 0; k < n; ++k) {
        double w;
        f = observe(P, w_tape, stride, k, sign, scale, vol, w);
        const double t = P.obs_time[k];
        barrier_interval(pp, acc, h, prev_f, f, var, var, t - prev_t, failed);
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
    // Variance adjoint over the intervals in order, then the state adjoints
    // node by node: sa_k = right part of interval k-1 + left part of
    // interval k + the smoothed hit factor (the terminal seed first at n).
    double var_adj = 0.0;
    if (flows) {
        prev_f = spot;
        prev_t = 0.0;
        for (uint32_t k = 0; k < n; ++k) {
            double w;
            const double fk = observe(P, w_tape, stride, k, sign, scale, vol, w);
            const double t = P.obs_time[k];
            const IntervalAdjoint ia = barrier_interval_adjoint(up, pp.barrier, h, lsa, prev_f, fk, var, var, t - prev_t);
            var_adj += ia.left_var + ia.right_var;
            prev_f = fk;
            prev_t = t;
        }
    }
    double delta = 0.0;
    double vega = 2.0 * vol * var_adj;
    {
        // node 0: the initial state
        double sa = 0.0;
        double f_next = 0.0, w_next = 0.0;
        if (n > 0) f_next = observe(P, w_tape, stride, 0, sign, scale, vol, w_next);
        IntervalAdjoint right{0.0, 0.0, 0.0, 0.0};
        if (flows) {
            right = barrier_interval_adjoint(up, pp.barrier, h, lsa, spot, f_next, var, var, P.obs_time[0]);
            sa += right.left_state;
            if (h > 0.0) sa += hit_factor_adjoint(up, pp.barrier, h, lsa, spot);
        }
        delta = sa;
        double prev_t2 = P.obs_time[0];
        for (uint32_t k = 0; k < n; ++k) {
            // node k + 1 holds observation k
            const double fk = f_next, wk = w_next;
            double s = 0.0;
            if (k + 1 == n) s += td * 1.0;
            if (flows) s += right.right_state;
            if (k + 1 < n) {
                f_next = observe(P, w_tape, stride, k + 1, sign, scale, vol, w_next);
                if (flows) {
                    const double t = P.obs_time[k + 1];
                    right = barrier_interval_adjoint(up, pp.barrier, h, lsa, fk, f_next, var, var, t - prev_t2);
                    prev_t2 = t;
                    s += right.left_state;
                }
            }
            if (flows && h > 0.0) s += hit_factor_adjoint(up, pp.barrier, h, lsa, fk);
            delta += s * fk / spot;
            vega += s * fk * (-vol * P.obs_time[k] + wk);
        }
    }
    PathAad r;
    r.price = P.discount * value;
    r.delta = P.discount * delta;
    r.vega = P.discount * vega;
    return r;
}

template <bool kCont>
__device__ __forceinline__ PathAad path_aad(const DevicePlan& P, const ProductParams& pp, const double* w_tape,
                                            double* h_tape, size_t stride, double sign, double spot, double vol,
                                            double* diag, bool& failed) {
    if constexpr (kCont)
        return continuous_aad(P, pp, w_tape, stride, sign, spot, vol, diag, failed);
    else
        return discrete_aad(P, pp, w_tape, h_tape, stride, sign, spot, vol, failed);
}

// The components of one primary or mate path (pathwise_values, :417-472).
template <bool kCont>
__device__ void path_values(const DevicePlan& P, const ProductParams& pp, const double* w_tape, double* h_tape,
                            size_t stride, double sign, double* v, bool& failed) {
    double diag[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double scratch[8];
    const PathAad base = path_aad<kCont>(P, pp, w_tape, h_tape, stride, sign, P.spot, P.vol, diag, failed);
    double gamma = 0.0;
    if (P.req_gamma) {
        const double b = P.gamma_bump;
        const PathAad dn = path_aad<kCont>(P, pp, w_tape, h_tape, stride, sign, P.spot - b, P.vol, scratch, failed);
        const PathAad up = path_aad<kCont>(P, pp, w_tape, h_tape, stride, sign, P.spot + b, P.vol, scratch, failed);
        gamma = (up.delta - dn.delta) / (2.0 * b);
    }
    const double sb = P.spot_bump;
    const PathAad dn = path_aad<kCont>(P, pp, w_tape, h_tape, stride, sign, P.spot - sb, P.vol, scratch, failed);
    const PathAad up = path_aad<kCont>(P, pp, w_tape, h_tape, stride, sign, P.spot + sb, P.vol, scratch, failed);
    const double bump_delta = (up.price - dn.price) / (2.0 * sb);
    const double bump_gamma = (up.price - 2.0 * base.price + dn.price) / (sb * sb);
    double bump_vega = 0.0;
    if (P.vol_bump != 0.0) {
        const double vb = P.vol_bump;
        const double a = path_aad<kCont>(P, pp, w_tape, h_tape, stride, sign, P.spot, P.vol - vb, scratch, failed).price;
        const double b = path_aad<kCont>(P, pp, w_tape, h_tape, stride, sign, P.spot, P.vol + vb, scratch, failed).price;
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
#pragma unroll
    for (int q = 0; q < 8; ++q) v[10 + q] = kCont ? diag[q] : 0.0;
}

}  // namespace

// One thread per unit of [unit_begin, unit_end); CTA records of tile
// unit/128 of scramble blockIdx.y.
template <bool kCont>
__global__ void __launch_bounds__(kThreads) bs_path_risk_kernel(const DevicePlan P, uint64_t unit_begin,
                                                                uint64_t unit_end, StatRecord* partials,
                                                                uint32_t mask, ErrorWord* err, int detail) {
    __shared__ Stat s_red[4 * kComponents];
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < unit_end && point < P.units;
    const uint64_t unit = valid ? point : 0;
    const size_t stride = static_cast<size_t>(gridDim.x) * gridDim.y * kThreads;
    const size_t local = (static_cast<size_t>(blockIdx.y) * gridDim.x + blockIdx.x) * kThreads + threadIdx.x;
    double* w_tape = P.bs_tape + local;
    double* h_tape = P.bs_tape + static_cast<size_t>(P.observation_count) * stride + local;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    // W_k of the primary path (path_observations_from_normals, :297-331)
    double w = 0.0;
    for (uint32_t k = 0; k < P.observation_count; ++k) {
        const double z = P.zero_variance ? 0.0 : ns.normal(k);
        w += P.obs_sqrt_step[k] * z;
        w_tape[static_cast<size_t>(k) * stride] = w;
    }
    const ProductParams& pp = P.products[0];
    bool failed = false;
    double vals[kComponents];
    path_values<kCont>(P, pp, w_tape, h_tape, stride, 1.0, vals, failed);
    if (P.antithetic) {
        double mate[kComponents];
        path_values<kCont>(P, pp, w_tape, h_tape, stride, -1.0, mate, failed);
#pragma unroll
        for (int c = 0; c < kComponents; ++c) vals[c] = (vals[c] + mate[c]) * 0.5;
    }
    if (valid && failed) report_error(err, unit, MCG_ERR_BARRIER_BRIDGE, 0, 0.0, detail);
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
    if (P.product_count != 1 || !P.bs_tape) return cudaErrorNotSupported;
    const bool cont = P.products[0].kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
    const uint64_t per_launch = P.bs_tape_units / scrambles / kThreads * kThreads;
    if (per_launch == 0) return cudaErrorInvalidValue;
    const uint64_t end = unit_begin + units;
    for (uint64_t begin = unit_begin; begin < end; begin += per_launch) {
        const uint64_t n = end - begin < per_launch ? end - begin : per_launch;
        const dim3 grid(static_cast<unsigned>((n + kThreads - 1) / kThreads), scrambles);
        if (cont)
            bs_path_risk_kernel<true><<<grid, kThreads, 0, stream>>>(P, begin, begin + n, partials, mask, err, detail);
        else
            bs_path_risk_kernel<false><<<grid, kThreads, 0, stream>>>(P, begin, begin + n, partials, mask, err, detail);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace mcg

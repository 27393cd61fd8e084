// mcg_lv_adjoint.cu -- reverse (adjoint) path kernel of the local-volatility
// Log-Euler model (FP64, -fmad=false).
//
// The reference stores a full step cache per path (state, variance,
// interpolation, exponential: ~130 B per step,
// crates/pricing/src/engine/processes/local_vol.rs:807-815) and reverses it
// (local_vol.rs:723-803, local_vol/direct_adjoints.rs:97-159).  Here the
// forward pass checkpoints only the state and the shock of every step
// (16 B per path-step, coalesced [step][unit] in global memory); the reverse
// sweep recomputes the interpolation cell and weights, the local variance, its
// x-derivative and the exponential of each step from them.
//
// One launch evaluates one spot runtime (base, S-h or S+h) and one antithetic
// sign.  Outputs per unit: local Vega (sum over grid nodes of 2 sqrt(v) times
// the node adjoint, pathwise_local_vol.rs:310-321) and the adjoint spot Delta
// dP/dS0 = lambda_0 - (1/S0) sum_i dP/dx_i.  For the base runtime the node
// adjoints of a CTA's units are summed in a sliding window of three grid rows
// in shared memory and written per CTA tile.
#include "mcg_kernels.cuh"

namespace mcg {

constexpr int kAdjThreads = 128;
static_assert(kAdjThreads == kThreads, "the batched normals index [k][thread] with kThreads");

struct AdjointArgs {
    int32_t which;          // spot runtime: 0 base, 1 down, 2 up
    double sign;            // antithetic sign of the shocks
    double node_weight;     // 1, or 0.5 for each sign of an antithetic pair
    int32_t node_add;       // add to (1) or overwrite (0) the tile node sums
    uint32_t scramble;
    uint64_t unit_begin;    // first unit of this chunk
    uint64_t units;         // units in this chunk
    uint32_t tile_offset;   // global tile index of blockIdx.x = 0
    double* tape_f;         // [(steps + 1)][units]
    double* tape_z;         // [steps][units]
    double* out_vega;       // [units]
    double* out_delta;      // [units]
    double* node_tiles;     // [global tile][nt * nx] or null
    double* out_price;      // [units] discounted payoff of the forward pass, or null
    double* out_diag;       // [8][units] continuous-barrier diagnostics, or null
    // Early exercise under a fixed policy: when set, the payoff is the exercise
    // value max(+-(S_k - K), 0) * notional at the path's stopping date
    // k = stops[local * stop_stride], discounted by exercise_df[k]
    // (the American payoff graph's output k with its cash-flow discount).
    const uint32_t* stops;
    uint32_t stop_stride;
    const double* exercise_df;
};

struct InterpFull {
    int tc, c;
    double tw, xw, value, dvdx;
};

// Interpolation with cell, weights and the x-derivative of
// LocalVarianceGrid::interpolation_log_moneyness_derivative (local_variance.rs:398-414).
__device__ __forceinline__ InterpFull interp_full(const GridView& g, int tc, double tw, double xq,
                                                  int& hint) {
    InterpFull r;
    double xv = xq;
    bool in_range = true;
    if (xq < g.x[0]) {
        xv = g.x[0];
        in_range = false;
    } else if (xq > g.x[g.nx - 1]) {
        xv = g.x[g.nx - 1];
        in_range = false;
    }
    const long long k = total_key(xv);
    int count = min(hint + 1, g.nx);
    while (count < g.nx && g.xkey[count] <= k) ++count;
    while (count > 0 && g.xkey[count - 1] > k) --count;
    const int c = min(max(count - 1, 0), g.nx - 2);
    hint = c;
    const double width = g.x[c + 1] - g.x[c];
    const double xw = (xv - g.x[c]) / width;
    const double* row = g.v + static_cast<size_t>(tc) * g.nx;
    const double* next = row + g.nx;
    const double lower = row[c] * (1.0 - xw) + row[c + 1] * xw;
    const double upper = next[c] * (1.0 - xw) + next[c + 1] * xw;
    r.tc = tc;
    r.c = c;
    r.tw = tw;
    r.xw = xw;
    r.value = lower * (1.0 - tw) + upper * tw;
    if (in_range) {
        const double ls = (row[c + 1] - row[c]) / width;
        const double us = (next[c + 1] - next[c]) / width;
        r.dvdx = ls * (1.0 - tw) + us * tw;
    } else {
        r.dvdx = 0.0;
    }
    return r;
}

// Adjoint of one grid interpolation: the transpose deposit of `seed` on the
// four corners (LocalVarianceInterpolation::transpose_accumulate,
// local_variance.rs:109-124), weighted by 2 sqrt(v) of each node, into Vega
// and, for the base runtime, the CTA's row window.  The window uses shared
// memory atomics: node sums may differ in the last bits between runs; every
// other output of the engine is bit-reproducible.
__device__ __forceinline__ void deposit(const InterpFull& in, double seed, const double* vol2, int nx,
                                       double& vega, double* window, double weight, bool nodes) {
    const double tl = 1.0 - in.tw, tr = in.tw;
    const double xl = 1.0 - in.xw, xr = in.xw;
    const double a00 = seed * tl * xl;
    const double a01 = seed * tl * xr;
    const double a10 = seed * tr * xl;
    const double a11 = seed * tr * xr;
    const int r0 = in.tc * nx + in.c;
    const int r1 = r0 + nx;
    // node sensitivity = node adjoint x 2 sqrt(v_node) (pathwise_local_vol.rs:304-309)
    const double n00 = a00 * vol2[r0], n01 = a01 * vol2[r0 + 1];
    const double n10 = a10 * vol2[r1], n11 = a11 * vol2[r1 + 1];
    vega += n00 + n01 + n10 + n11;
    if (nodes) {
        const int w0 = (in.tc % 3) * nx + in.c;
        const int w1 = ((in.tc + 1) % 3) * nx + in.c;
        atomicAdd(window + w0, weight * n00);
        atomicAdd(window + w0 + 1, weight * n01);
        atomicAdd(window + w1, weight * n10);
        atomicAdd(window + w1 + 1, weight * n11);
    }
}

// Write (or add) finished rows [lo, hi] of the window to the CTA tile and clear them.
__device__ __forceinline__ void flush_rows(double* window, int lo, int hi, int nx, double* tile,
                                           bool add) {
    __syncthreads();
    for (int r = lo; r <= hi; ++r) {
        double* w = window + (r % 3) * nx;
        for (int j = threadIdx.x; j < nx; j += kAdjThreads) {
            const double v = w[j];
            if (add) tile[static_cast<size_t>(r) * nx + j] += v;
            else tile[static_cast<size_t>(r) * nx + j] = v;
            w[j] = 0.0;
        }
    }
    __syncthreads();
}

// The grid values and their 2 sqrt(v) are read through L1 (shared memory
// holds the x nodes, the node window and the bridge slots), which lets 5 CTAs
// share an SM.  kBridge: the product's continuous-barrier bridge, 0 none
// (another product), 1 exact, 2 smoothed; the launch picks it from the
// product and the smoothing width, so each instantiation holds one form.
template <int kBridge>
__global__ void __launch_bounds__(kAdjThreads, 5) lv_adjoint_kernel(const DevicePlan P, AdjointArgs A,
                                                                    ErrorWord* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = static_cast<int>(P.nx);
    const int nt = static_cast<int>(P.nt);
    const size_t nv = static_cast<size_t>(nt) * nx;
    const double* s_vol2 = P.grid_vol2;
    double* s_x = reinterpret_cast<double*>(smem_raw);
    long long* s_xk = reinterpret_cast<long long*>(s_x + nx);
    double* s_win = reinterpret_cast<double*>(s_xk + nx);
    double* s_w = s_win + 3 * nx;  // bridge slots [slot][thread]
    // batched normals [k][thread] and their per-warp tail lists (fill_normals)
    double* s_z = s_w + static_cast<size_t>(P.slot_count) * kAdjThreads;
    uint16_t* s_zlist = reinterpret_cast<uint16_t*>(s_z + z_batch<1>() * kAdjThreads);
    for (int i = threadIdx.x; i < nx; i += kAdjThreads) {
        s_x[i] = P.grid_x[i];
        s_xk[i] = total_key(P.grid_x[i]);
    }
    for (int i = threadIdx.x; i < 3 * nx; i += kAdjThreads) s_win[i] = 0.0;
    __syncthreads();
    const GridView g{P.grid_v, s_x, s_xk, nx};

    const uint64_t local = static_cast<uint64_t>(blockIdx.x) * kAdjThreads + threadIdx.x;
    const bool valid = local < A.units;
    const uint64_t unit = A.unit_begin + (valid ? local : 0);
    const uint64_t ustride = A.units;
    const uint32_t steps = P.steps;
    const int which = A.which;
    const double* F = P.fwd + static_cast<size_t>(which) * (steps + 1);
    const double* ratio = P.ratio + static_cast<size_t>(which) * steps;
    const ProductParams& pp = P.products[0];
    constexpr bool barrier = kBridge != 0;
    const bool up = pp.barrier_direction == MCG_BARRIER_UP;
    const double h = kBridge == 1 ? 0.0 : P.smoothing;
    if constexpr (kBridge == 2) __builtin_assume(h > 0.0);
    const bool call = pp.side == MCG_CALL;

    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(A.scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(A.scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;

    // ------------------------------------------------------------ forward
    double f = P.spot_variant[which];
    double prev_f = f, prev_v = 0.0;
    int hint = 0;
    ProductAcc acc;
    acc_init(acc, pp);
    bool failed = false;
    int fail_code = 0;
    uint32_t fail_step = 0;
    int32_t argmax = -1;  // observation holding the lookback extremum (-1: the seasoned literal)
    const bool fixed = A.stops != nullptr;
    const uint32_t k_stop = fixed && valid ? A.stops[local * A.stop_stride] : 0u;
    double f_stop = f;
    if (barrier) barrier_begin(pp, acc, h, f, failed);
    if (valid) A.tape_f[local] = f;
    double* w = s_w + threadIdx.x;
    // The program's normals in order (P.z_ranks), eight at a time with AS241's
    // tail branch compacted across the warp; every thread of the CTA walks the
    // same program, so the warp-collective batches line up.
    NormalSource nsq[1] = {ns};
    uint32_t zi = 0, zbase = 0, zend = 0;
    auto next_normal = [&]() -> double {
        if (zi == zend) {
            zbase = zi;
            constexpr uint32_t kBatch = static_cast<uint32_t>(z_batch<1>());
            const uint32_t n = P.z_count - zi < kBatch ? P.z_count - zi : kBatch;
            fill_normals<1>(nsq, false, zi, n, s_z, s_zlist, P.z_ranks);
            zend = zi + n;
        }
        const uint32_t k = zi++ - zbase;
        return s_z[k * kAdjThreads + threadIdx.x];
    };
    for (uint32_t oi = 0; oi < P.op_count; ++oi) {
        const Op op = P.ops[oi];
        if (op.kind == kOpZero) {
            w[op.out * kAdjThreads] = 0.0;
            continue;
        }
        if (op.kind == kOpTerminal) {
            w[op.out * kAdjThreads] = op.sd * next_normal();
            continue;
        }
        if (op.kind == kOpInterior) {
            const double z = next_normal();
            w[op.out * kAdjThreads] = op.wl * w[op.left * kAdjThreads] + op.wr * w[op.right * kAdjThreads] + op.sd * z;
            continue;
        }
        const uint32_t s = static_cast<uint32_t>(op.step);
        double shock;
        if (op.kind == kOpStep)
            shock = (w[op.right * kAdjThreads] - w[op.left * kAdjThreads]) * P.inv_sqrt_dt[s];
        else
            shock = next_normal();
        const double z = A.sign * shock;
        const double x = log(f / F[s]);
        const double v = interp_variance(g, P.time_cell[s], P.time_weight[s], x, hint);
        if (barrier && s > 0) barrier_interval(pp, acc, h, prev_f, f, prev_v, v, P.dt[s - 1], failed);
        const double e = ratio[s] * exp(-0.5 * v * P.dt[s] + sqrt(v) * P.sqrt_dt[s] * z);
        prev_f = f;
        prev_v = v;
        f *= e;
        if (!(isfinite(f) && f > 0.0) && !fail_code) {
            fail_code = MCG_ERR_NON_FINITE_STATE;
            fail_step = s + 1;
        }
        if (valid) {
            A.tape_z[static_cast<size_t>(s) * ustride + local] = z;
            A.tape_f[static_cast<size_t>(s + 1) * ustride + local] = f;
        }
        const int32_t obs = P.obs_of_node[s + 1];
        if (fixed && obs == static_cast<int32_t>(k_stop)) f_stop = f;
        if (obs >= 0) {
            if (pp.kind == MCG_PRODUCT_LOOKBACK) {
                if (monitored(pp, static_cast<uint32_t>(obs)) &&
                    (acc.counts == 0u || (call ? !(acc.a >= f) : !(acc.a <= f))))
                    argmax = obs;
            }
            acc_observe(pp, acc, static_cast<uint32_t>(obs), f, h, failed);
        }
    }
    // ----------------------------------------------------- payoff adjoints
    // Terminal node: interpolation for the last bridge interval and the
    // direct variance seed.
    InterpFull inN = interp_full(g, nt - 2, 1.0, log(f / F[steps]), hint);
    double lsa = 0.0;         // log-survival adjoint (continuous barrier)
    double terminal_adj = 0.0;
    double asian_g = 0.0;     // Asian: d payoff / d average
    bool exact_active = false;
    if (barrier) {
        barrier_interval(pp, acc, h, prev_f, f, prev_v, inN.value, P.dt[steps - 1], failed);
        double diag[8];
        const double surv = barrier_finish(acc, h, steps, diag);
        if (A.out_price && valid) {
            A.out_price[local] = P.discount * barrier_value(pp, f, surv);
#pragma unroll
            for (int q = 0; q < 8; ++q) A.out_diag[static_cast<size_t>(q) * ustride + local] = diag[q];
        }
        const double in = call ? f - pp.strike : pp.strike - f;
        const double vanilla = fmax(in, 0.0) * pp.notional;
        const double vd = in >= 0.0 ? (call ? 1.0 : -1.0) * pp.notional : 0.0;
        const double rebate = pp.has_rebate ? pp.rebate : 0.0;
        double td, sd;
        if (pp.barrier_style == MCG_KNOCK_OUT) {
            td = surv * vd;
            sd = vanilla - rebate;
        } else {
            td = (1.0 - surv) * vd;
            sd = rebate - vanilla;
        }
        terminal_adj = P.discount * td * 1.0;
        exact_active = !(acc.initial_touched || acc.touched);
        lsa = P.discount * sd * surv;
    } else if (fixed) {
        // exercise value at the stopping date and its spot adjoint
        const double dfk = A.exercise_df[k_stop];
        const double in = call ? f_stop - pp.strike : pp.strike - f_stop;
        if (A.out_price && valid) A.out_price[local] = dfk * ((in >= 0.0 ? in : 0.0) * pp.notional);
        terminal_adj = dfk * ((in >= 0.0 ? pp.notional : 0.0) * (call ? 1.0 : -1.0)) * 1.0;
    } else {
        if (A.out_price && valid) A.out_price[local] = P.discount * acc_payoff(pp, acc, h);
        // d payoff / d observed spot (tape.rs:594-781 reverse semantics)
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
            asian_g = (in >= 0.0 ? pp.notional : 0.0) * (call ? 1.0 : -1.0);
            break;
        }
        case MCG_PRODUCT_DISCRETE_BARRIER: {
            const double in = call ? term - pp.strike : pp.strike - term;
            const double active = pp.barrier_style == MCG_KNOCK_OUT ? 1.0 - acc.a : acc.a;
            terminal_adj = (in >= 0.0 ? active * pp.notional : 0.0) * (call ? 1.0 : -1.0);
            break;
        }
        default:
            break;
        }
        terminal_adj = P.discount * terminal_adj * 1.0;
    }
    const bool bridge_adjoint = barrier && (h > 0.0 || exact_active);
    // Seed of a discrete product at observation node k (not the terminal).
    auto obs_seed = [&](uint32_t node) -> double {
        const int32_t obs = P.obs_of_node[node];
        if (obs < 0 || barrier) return 0.0;
        if (fixed) return obs == static_cast<int32_t>(k_stop) ? terminal_adj : 0.0;
        if (pp.kind == MCG_PRODUCT_ASIAN) return P.discount * (asian_g * pp.weights[obs]) * 1.0;
        if (pp.kind == MCG_PRODUCT_LOOKBACK) return obs == argmax ? P.discount * asian_g * 1.0 : 0.0;
        return 0.0;
    };

    // ------------------------------------------------------------ reverse
    const bool nodes = A.node_tiles != nullptr;
    double* tile = nodes ? A.node_tiles + static_cast<size_t>(A.tile_offset + blockIdx.x) * nv : nullptr;
    int base = nt;  // lowest row held in the window
    double vega = 0.0, x_sum = 0.0;
    // node N
    double f_next = f;
    InterpFull in_next = inN;
    double sa_next = obs_seed(steps);
    if (!barrier && !fixed &&
        (pp.kind == MCG_PRODUCT_EUROPEAN || pp.kind == MCG_PRODUCT_DIGITAL || pp.kind == MCG_PRODUCT_DISCRETE_BARRIER))
        sa_next += terminal_adj;
    // The bridge quantities of node s + 1, carried down from the previous step.
    const bool endpoints = bridge_adjoint || (barrier && h > 0.0);
    const double lb = endpoints && !(h > 0.0) ? log(pp.barrier) : 0.0;
    BarrierEndpoint node_next{};
    if (endpoints) node_next = barrier_endpoint(up, pp.barrier, lb, h, f);
    if (barrier) {
        sa_next += terminal_adj;
        if (h > 0.0) sa_next += hit_factor_adjoint(node_next, lsa);
    }
    double vs_next = 0.0;
    for (int s = static_cast<int>(steps) - 1; s >= 0; --s) {
        const int tc = P.time_cell[s];
        if (nodes && tc < base) {
            const int hi = min(base + 2, nt - 1);
            const int lo = max(tc + 3, 0);
            if (base < nt && lo <= hi) flush_rows(s_win, lo, hi, nx, tile, A.node_add);
            base = tc;
        }
        const double fs = valid ? A.tape_f[static_cast<size_t>(s) * ustride + local] : f;
        const double zs = valid ? A.tape_z[static_cast<size_t>(s) * ustride + local] : 0.0;
        const InterpFull in_s = interp_full(g, tc, P.time_weight[s], log(fs / F[s]), hint);
        double sa_cur = obs_seed(static_cast<uint32_t>(s));
        double vs_cur = 0.0;
        BarrierEndpoint node_s{};
        if (endpoints) node_s = barrier_endpoint(up, pp.barrier, lb, h, fs);
        if (bridge_adjoint) {
            const IntervalAdjoint ia = bridge_interval_adjoint(up, h, lsa, node_s, node_next, fs, f_next, in_s.value,
                                                               in_next.value, P.dt[s]);
            sa_next += ia.right_state;
            vs_next += ia.right_var;
            sa_cur += ia.left_state;
            vs_cur += ia.left_var;
        }
        if (barrier && h > 0.0) sa_cur += hit_factor_adjoint(node_s, lsa);
        node_next = node_s;
        // finalise node s + 1: its direct variance seed
        if (vs_next != 0.0) {
            sa_next += vs_next * in_next.dvdx / f_next;
            x_sum += vs_next * in_next.dvdx;
            deposit(in_next, vs_next, s_vol2, nx, vega, s_win, A.node_weight, nodes && valid);
        }
        // transition s -> s + 1 (local_vol.rs:758-789)
        const double lea = sa_next * f_next;
        const double lvol = sqrt(in_s.value);
        const double dt = P.dt[s];
        const double e = ratio[s] * exp(-0.5 * in_s.value * dt + lvol * P.sqrt_dt[s] * zs);
        sa_cur += sa_next * e;
        const double lva = lea * (-0.5 * dt + zs * P.sqrt_dt[s] / (2.0 * lvol));
        sa_cur += lva * (in_s.dvdx / fs);
        x_sum += lva * in_s.dvdx;
        deposit(in_s, lva, s_vol2, nx, vega, s_win, A.node_weight, nodes && valid);
        if (!isfinite(sa_cur) && !fail_code) {
            fail_code = MCG_ERR_NON_FINITE_STATE;
            fail_step = static_cast<uint32_t>(s);
        }
        sa_next = sa_cur;
        vs_next = vs_cur;
        f_next = fs;
        in_next = in_s;
    }
    // node 0
    if (vs_next != 0.0) {
        sa_next += vs_next * in_next.dvdx / f_next;
        x_sum += vs_next * in_next.dvdx;
        deposit(in_next, vs_next, s_vol2, nx, vega, s_win, A.node_weight, nodes && valid);
    }
    if (nodes) flush_rows(s_win, 0, min(base + 2, nt - 1), nx, tile, A.node_add);
    if (failed && !fail_code) fail_code = MCG_ERR_BARRIER_BRIDGE;
    if (valid) {
        if (fail_code) report_error(err, unit, fail_code, fail_step, 0.0, false);
        A.out_vega[local] = vega;
        A.out_delta[local] = sa_next - x_sum / P.spot_variant[which];
    }
}

// Per-unit adjoint components -> CTA records: Vega, adjoint Delta and the
// bumped-adjoint Gamma, antithetic pairs averaged component-wise.
__global__ void __launch_bounds__(kThreads) lv_adjoint_combine_kernel(
    const double* vega, const double* delta, uint64_t units, int pairs, int have_gamma, double h,
    uint32_t tile_offset, StatRecord* partials, uint32_t slots) {
    __shared__ Stat s_red[4 * 3];
    const uint64_t u = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = u < units;
    double vals[3] = {0.0, 0.0, 0.0};
    if (valid) {
        for (int pr = 0; pr < pairs; ++pr) {
            const size_t base = static_cast<size_t>(pr) * 3;
            const double v = vega[(base + 0) * units + u];
            const double d = delta[(base + 0) * units + u];
            const double g = have_gamma ? (delta[(base + 2) * units + u] - delta[(base + 1) * units + u]) / (2.0 * h)
                                        : 0.0;
            if (pr == 0) {
                vals[0] = v;
                vals[1] = d;
                vals[2] = g;
            } else {
                vals[0] = (vals[0] + v) * 0.5;
                vals[1] = (vals[1] + d) * 0.5;
                vals[2] = (vals[2] + g) * 0.5;
            }
        }
    }
    cta_reduce_write<3>(vals, valid, 0x7u, partials + static_cast<size_t>(tile_offset + blockIdx.x) * slots, s_red);
}

// Price (and continuous-barrier diagnostics) of the units of a chunk, taken
// from the adjoint sweeps' forward passes when no separate price pass runs:
// antithetic pairs averaged as the path kernel averages them, one
// kComponents record per CTA tile of the plan's partials.
__global__ void __launch_bounds__(kThreads) lv_adjoint_price_kernel(const double* price, const double* diag,
                                                                    uint64_t units, int pairs, uint32_t tile_offset,
                                                                    uint32_t mask, StatRecord* partials) {
    __shared__ Stat s_red[4 * kComponents];
    const uint64_t u = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = u < units;
    double vals[kComponents];
#pragma unroll
    for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
    if (valid) {
        for (int pr = 0; pr < pairs; ++pr) {
            const double p = price[static_cast<size_t>(pr) * units + u];
            vals[MCG_PRICE] = pr == 0 ? p : (vals[MCG_PRICE] + p) * 0.5;
            if (diag)
                for (int q = 0; q < 8; ++q) {
                    const double d = diag[(static_cast<size_t>(pr) * 8 + q) * units + u];
                    vals[10 + q] = pr == 0 ? d : (vals[10 + q] + d) * 0.5;
                }
        }
    }
    cta_reduce_write<kComponents>(vals, valid, mask,
                                  partials + static_cast<size_t>(tile_offset + blockIdx.x) * kComponents, s_red);
}

// Fixed-policy risk components of a chunk's units: the exercise-value
// prices of the base and bumped spot runtimes (price[(pr * 3 + which) * units + u]),
// the base sweep's Vega; CRN Delta/Gamma as the path kernel forms them,
// antithetic pairs averaged component-wise (average_local_vol_pathwise).
__global__ void __launch_bounds__(kThreads) lv_fixed_policy_combine_kernel(
    const double* price, const double* vega, uint64_t units, int pairs, int crn, int gamma, int want_vega, double h,
    uint32_t tile_offset, StatRecord* partials) {
    __shared__ Stat s_red[4 * kComponents];
    const uint64_t u = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = u < units;
    double vals[kComponents];
#pragma unroll
    for (int c = 0; c < kComponents; ++c) vals[c] = 0.0;
    if (valid) {
        for (int pr = 0; pr < pairs; ++pr) {
            double comp[kComponents];
#pragma unroll
            for (int c = 0; c < kComponents; ++c) comp[c] = 0.0;
            const double base = price[(static_cast<size_t>(pr) * 3 + 0) * units + u];
            comp[MCG_PRICE] = base;
            if (want_vega) comp[MCG_VEGA] = vega[(static_cast<size_t>(pr) * 3 + 0) * units + u];
            if (crn) {
                const double down = price[(static_cast<size_t>(pr) * 3 + 1) * units + u];
                const double up = price[(static_cast<size_t>(pr) * 3 + 2) * units + u];
                const double delta = (up - down) / (2.0 * h);
                comp[MCG_DELTA] = delta;
                comp[MCG_BUMP_DELTA] = delta;
                if (gamma) {
                    const double g = (up - 2.0 * base + down) / (h * h);
                    comp[MCG_GAMMA] = g;
                    comp[MCG_BUMP_GAMMA] = g;
                }
            }
#pragma unroll
            for (int c = 0; c < kComponents; ++c) vals[c] = pr == 0 ? comp[c] : (vals[c] + comp[c]) * 0.5;
        }
    }
    cta_reduce_write<kComponents>(vals, valid, 0x3ffu,
                                  partials + static_cast<size_t>(tile_offset + blockIdx.x) * kComponents, s_red);
}

// Node sums over tiles, per scramble: Neumaier sum in tile order and the
// two-pass second moment of the tile sums (batch means).
__global__ void lv_node_reduce_kernel(const double* node_tiles, uint32_t tiles_per_scramble,
                                      uint32_t scrambles, uint32_t nv, StatRecord* out) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nv * scrambles) return;
    const uint32_t s = idx / nv, k = idx % nv;
    double sum = 0.0, corr = 0.0;
    const size_t base = static_cast<size_t>(s) * tiles_per_scramble;
    for (uint32_t t = 0; t < tiles_per_scramble; ++t) neumaier_add(sum, corr, node_tiles[(base + t) * nv + k]);
    const double mean = (sum + corr) / tiles_per_scramble;
    double q = 0.0, qc = 0.0;
    for (uint32_t t = 0; t < tiles_per_scramble; ++t) {
        const double d = node_tiles[(base + t) * nv + k] - mean;
        neumaier_add(q, qc, d * d);
    }
    out[idx] = {sum, corr, static_cast<double>(tiles_per_scramble), mean, q + qc};
}

size_t lv_adjoint_smem(const DevicePlan& P) {
    return (2 * static_cast<size_t>(P.nx) + 3 * P.nx) * sizeof(double) +
           static_cast<size_t>(P.slot_count) * kAdjThreads * sizeof(double) +
           static_cast<size_t>(z_batch<1>()) * kAdjThreads * sizeof(double) +
           (kAdjThreads / 32) * 32 * static_cast<size_t>(z_batch<1>()) * sizeof(uint16_t);
}

cudaError_t launch_lv_adjoint(const DevicePlan& P, const AdjointArgs& A, ErrorWord* err, cudaStream_t stream) {
    const size_t smem = lv_adjoint_smem(P);
    const unsigned blocks = static_cast<unsigned>((A.units + kAdjThreads - 1) / kAdjThreads);
    auto go = [&](auto kernel) -> cudaError_t {
        const cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<blocks, kAdjThreads, smem, stream>>>(P, A, err);
        return cudaGetLastError();
    };
    if (P.products[0].kind != MCG_PRODUCT_CONTINUOUS_BARRIER) return go(lv_adjoint_kernel<0>);
    if (P.smoothing > 0.0) return go(lv_adjoint_kernel<2>);
    return go(lv_adjoint_kernel<1>);
}

cudaError_t launch_lv_adjoint_combine(const double* vega, const double* delta, uint64_t units, int pairs,
                                      int have_gamma, double h, uint32_t tile_offset, StatRecord* partials,
                                      cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((units + kThreads - 1) / kThreads);
    lv_adjoint_combine_kernel<<<blocks, kThreads, 0, stream>>>(vega, delta, units, pairs, have_gamma, h,
                                                               tile_offset, partials, 3);
    return cudaGetLastError();
}

cudaError_t launch_lv_adjoint_price(const double* price, const double* diag, uint64_t units, int pairs,
                                    uint32_t tile_offset, uint32_t mask, StatRecord* partials, cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((units + kThreads - 1) / kThreads);
    lv_adjoint_price_kernel<<<blocks, kThreads, 0, stream>>>(price, diag, units, pairs, tile_offset, mask, partials);
    return cudaGetLastError();
}

cudaError_t launch_lv_fixed_policy_combine(const double* price, const double* vega, uint64_t units, int pairs,
                                           int crn, int gamma, int want_vega, double h, uint32_t tile_offset,
                                           StatRecord* partials, cudaStream_t stream) {
    const unsigned blocks = static_cast<unsigned>((units + kThreads - 1) / kThreads);
    lv_fixed_policy_combine_kernel<<<blocks, kThreads, 0, stream>>>(price, vega, units, pairs, crn, gamma, want_vega,
                                                                    h, tile_offset, partials);
    return cudaGetLastError();
}

cudaError_t launch_lv_node_reduce(const double* node_tiles, uint32_t tiles_per_scramble, uint32_t scrambles,
                                  uint32_t nv, StatRecord* out, cudaStream_t stream) {
    const uint32_t n = nv * scrambles;
    lv_node_reduce_kernel<<<(n + 127) / 128, 128, 0, stream>>>(node_tiles, tiles_per_scramble, scrambles, nv, out);
    return cudaGetLastError();
}

}  // namespace mcg

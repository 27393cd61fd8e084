// mcg_payoff.cuh -- streaming payoff accumulators and the continuous-barrier
// bridge of the path kernels.
//
// The reference evaluates each product as an opcode tape over stored
// observations (crates/pricing/src/engine/payoff/tape.rs:953-1088, graphs from
// crates/pricing/src/engine/payoff/compile.rs:35-474).  Here each product keeps
// a few registers that are updated as the path reaches an observation, with
// the same arithmetic in the same order, so no observation vector is stored.
#pragma once

#include "mcg_device.cuh"

namespace mcg {

constexpr double kLogMaxExpArgument = 6.564958884017094;  // barrier_bridge.rs:9
constexpr double kLogMinPositive = -744.4400719213812;    // barrier_bridge.rs:10
constexpr double kLn2 = 0.6931471805599453;

// Streaming state of one product on one path.
struct ProductAcc {
    double a;        // Asian weighted sum, lookback extremum, barrier hit state
    double log_sum;  // continuous barrier: sum of interval log survivals
    double hit_log;  // smoothed continuous barrier: sum of log safety weights
    double hit_prod; // smoothed continuous barrier: product of safety weights
    double terminal; // last observed spot
    uint32_t counts; // continuous barrier status counts (10-bit fields); lookback: 1 once `a` holds an extremum
    uint32_t counts2;
    int32_t touched; // exact continuous barrier: an endpoint touched
    int32_t initial_touched;
    // Continuous barrier: the next interval's left-endpoint quantities, carried
    // from this interval's right endpoint (the same values a fresh evaluation
    // of the same state gives): exact -- ln(state) and ln(log-distance);
    // smoothed -- the effective log-distance and its ln.
    double c_end, c_logd;
    uint32_t c_valid;  // bit 0: c_end, bit 1: c_logd
};

MCG_HD void acc_init(ProductAcc& s) {
    s.a = 0.0;
    s.log_sum = 0.0;
    s.hit_log = 0.0;
    s.hit_prod = 1.0;
    s.terminal = 0.0;
    s.counts = 0;
    s.counts2 = 0;
    s.touched = 0;
    s.initial_touched = 0;
    s.c_end = 0.0;
    s.c_logd = 0.0;
    s.c_valid = 0u;
}

// Initial state of a product: the seasoned literals of compile.rs:162-176
// (Asian known fixings), :293-297 (historical barrier hit) and :431-436
// (lookback historical extremum / valuation-date fixing).
MCG_HD void acc_init(ProductAcc& s, const ProductParams& p) {
    acc_init(s);
    if (p.has_initial) {
        s.a = p.initial;
        if (p.kind == MCG_PRODUCT_LOOKBACK) s.counts = 1u;
    }
}

// Whether observation `obs` is a monitoring date of a discrete barrier or a
// lookback (every observation when the product carries no flags).
MCG_HD bool monitored(const ProductParams& p, uint32_t obs) {
    return p.weights == nullptr || p.weights[obs] != 0.0;
}

// Observation update of one product on N paths with one dispatch on the
// product's kind: discrete products (compile.rs:159-202 Asian, :204-403
// discrete barrier, :405-474 lookback, tape.rs:1038-1080 opcode semantics).
// A discrete barrier monitored on an ex-dividend date also sees the spots just
// before the dividend, `pre` (with_pre): its distance is the maximum (smoothed:
// the compact-C2 smooth maximum) of the pre- and post-dividend distances
// (crates/pricing/src/engine/payoff/compile.rs:315-346).
// PRE = false compiles the pre-dividend check out (plans without dividends).
template <int N, bool PRE = true>
MCG_HD void acc_observe_n(const ProductParams& p, ProductAcc (&s)[N], uint32_t obs, const double (&spot)[N],
                          double smoothing, const double (&pre)[N], bool with_pre) {
#pragma unroll
    for (int i = 0; i < N; ++i) s[i].terminal = spot[i];
    switch (p.kind) {
    case MCG_PRODUCT_ASIAN: {
        const double w = p.weights[obs];
#pragma unroll
        for (int i = 0; i < N; ++i) s[i].a = s[i].a + spot[i] * w;
        break;
    }
    case MCG_PRODUCT_LOOKBACK:
        if (!monitored(p, obs)) break;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (s[i].counts == 0u) {
                s[i].a = spot[i];
                s[i].counts = 1u;
            } else if (p.side == MCG_CALL) {
                if (!(s[i].a >= spot[i])) s[i].a = spot[i];
            } else {
                if (!(s[i].a <= spot[i])) s[i].a = spot[i];
            }
        }
        break;
    case MCG_PRODUCT_DISCRETE_BARRIER: {
        if (!monitored(p, obs)) break;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double dist = p.barrier_direction == MCG_BARRIER_UP ? spot[i] - p.barrier : p.barrier - spot[i];
            if (PRE && with_pre) {
                const double pd = p.barrier_direction == MCG_BARRIER_UP ? pre[i] - p.barrier : p.barrier - pre[i];
                if (smoothing > 0.0) {
                    double dl, dr;
                    dist = smooth_maximum(smoothing, pd, dist, dl, dr);
                } else {
                    dist = pd >= dist ? pd : dist;
                }
            }
            double w;
            if (smoothing > 0.0) {
                double comp;
                w = smooth_indicator(smoothing, dist, comp).value;
            } else {
                w = dist >= 0.0 ? 1.0 : 0.0;
            }
            s[i].a = s[i].a + (1.0 - s[i].a) * w;
        }
        break;
    }
    default:
        break;
    }
}

// The same update on one path.
MCG_HD void acc_observe(const ProductParams& p, ProductAcc& s, uint32_t obs,
                                           double spot, double smoothing, bool& failed) {
    (void)failed;
    ProductAcc one[1] = {s};
    const double at[1] = {spot};
    acc_observe_n<1>(p, one, obs, at, smoothing, at, false);
    s = one[0];
}

// ---------------------------------------------- continuous barrier bridge

// log(-expm1(-exp(le))), the ordinary branch's log survival
// (barrier_bridge.rs:341-345, :493-497).
MCG_HD double interval_log_survival(double le) { return log(-expm1(-exp(le))); }

// BarrierBridgeInterval::evaluate (exact), barrier_bridge.rs:446-528, with a
// constant barrier; returns the status and log survival only.
MCG_HD int exact_interval(bool up, double ls, double rs, double barrier,
                                              double lv, double rv, double dt, double& log_surv,
                                              bool& failed) {
    if (!(ls > 0.0) || !isfinite(ls) || !(rs > 0.0) || !isfinite(rs) || !(lv >= 0.0) ||
        !isfinite(lv) || !(rv >= 0.0) || !isfinite(rv)) {
        failed = true;
        log_surv = 0.0;
        return 1;
    }
    const double lb = log(barrier);
    const double ld = up ? lb - log(ls) : log(ls) - lb;
    const double rd = up ? lb - log(rs) : log(rs) - lb;
    if (ld <= 0.0 || rd <= 0.0) {
        log_surv = -INFINITY;
        return 1;  // touched
    }
    const double integrated = (0.5 * lv + 0.5 * rv) * dt;
    if (!isfinite(integrated)) {
        failed = true;
        log_surv = 0.0;
        return 1;
    }
    if (integrated == 0.0) {
        log_surv = 0.0;
        return 2;
    }
    const double le = kLn2 + log(ld) + log(rd) - log(integrated);
    if (le >= kLogMaxExpArgument) {
        log_surv = 0.0;
        return 4;
    }
    if (le <= kLogMinPositive) {
        log_surv = le;
        return 3;
    }
    log_surv = interval_log_survival(le);
    return 0;
}

// SmoothedBarrierBridgeEndpoint::evaluate, barrier_bridge.rs:160-215: the
// safety weight and effective log distance of one endpoint (affine scale 1).
MCG_HD void smooth_endpoint(bool up, double state, double barrier, double h,
                                                double& safety, double& eld, bool& failed) {
    if (!(state > 0.0) || !isfinite(state)) {
        failed = true;
        safety = 1.0;
        eld = 1.0;
        return;
    }
    const double sign = up ? 1.0 : -1.0;
    const double signed_hit = 1.0 * sign * (state - barrier);
    smooth_indicator(h, signed_hit, safety);
    const SmoothD safe = smooth_positive_part(h, -signed_hit);
    const double spot_barrier = 1.0 * barrier;
    const double denominator = up ? spot_barrier - safe.value : spot_barrier + safe.value;
    if (!isfinite(denominator) || denominator <= 0.0) {
        failed = true;
        eld = 1.0;
        return;
    }
    eld = up ? -log1p(-safe.value / spot_barrier) : log1p(safe.value / spot_barrier);
}

// SmoothedBarrierBridgeInterval::evaluate, barrier_bridge.rs:276-357, given
// lld = log(ld) and lrd = log(rd) (a path's consecutive intervals share an
// endpoint and pass its logarithm on); they are read only when ld, rd != 0.
MCG_HD int smooth_interval(double ld, double rd, double lld, double lrd, double lv, double rv,
                           double dt, double& log_surv, bool& failed) {
    if (!(lv >= 0.0) || !isfinite(lv) || !(rv >= 0.0) || !isfinite(rv)) {
        failed = true;
        log_surv = 0.0;
        return 1;
    }
    if (ld == 0.0 || rd == 0.0) {
        log_surv = -INFINITY;
        return 1;
    }
    const double integrated = (0.5 * lv + 0.5 * rv) * dt;
    if (!isfinite(integrated)) {
        failed = true;
        log_surv = 0.0;
        return 1;
    }
    if (integrated == 0.0) {
        log_surv = 0.0;
        return 2;
    }
    const double le = kLn2 + lld + lrd - log(integrated);
    if (le >= kLogMaxExpArgument) {
        log_surv = 0.0;
        return 4;
    }
    if (le <= kLogMinPositive) {
        log_surv = le;
        return 3;
    }
    log_surv = interval_log_survival(le);
    return 0;
}

MCG_HD void count_status(ProductAcc& s, int status) {
    // 16-bit fields: counts = finite | zero << 16, counts2 = underflow | certain << 16.
    if (status == 0) s.counts += 1u;
    else if (status == 2) s.counts += 1u << 16;
    else if (status == 3) s.counts2 += 1u;
    else if (status == 4) s.counts2 += 1u << 16;
}

// One bridge interval of a continuous barrier (exact or smoothed).  Smoothed
// endpoints are recomputed for each interval, as the reference does; the
// smoothed right endpoint's safety weight is a hit factor.
// One interval of a path whose intervals follow one another: the left
// endpoint `ls` is the previous call's right endpoint, whose logarithms (and,
// smoothed, effective log-distance) the accumulator carries, so each interval
// evaluates its right endpoint only.  The arithmetic is exact_interval's and
// smooth_endpoint / smooth_interval's, value for value.
MCG_HD void barrier_interval(const ProductParams& p, ProductAcc& s,
                                                 double h, double ls, double rs, double lv,
                                                 double rv, double dt, bool& failed) {
    const bool up = p.barrier_direction == MCG_BARRIER_UP;
    const uint32_t carried = s.c_valid;
    s.c_valid = 0u;  // the endpoint quantities are set below
    if (!(dt > 0.0)) return;
    double log_surv;
    int status;
    if (h > 0.0) {
        double lsafe, rsafe, ld, rd;
        if (carried & 1u) ld = s.c_end;
        else smooth_endpoint(up, ls, p.barrier, h, lsafe, ld, failed);
        smooth_endpoint(up, rs, p.barrier, h, rsafe, rd, failed);
        s.c_end = rd;
        s.c_valid |= 1u;
        // smooth_interval with ln(ld) carried and ln(rd) kept for the next interval
        if (!(lv >= 0.0) || !isfinite(lv) || !(rv >= 0.0) || !isfinite(rv)) {
            failed = true;
            log_surv = 0.0;
            status = 1;
        } else if (ld == 0.0 || rd == 0.0) {
            log_surv = -INFINITY;
            status = 1;
        } else {
            const double integrated = (0.5 * lv + 0.5 * rv) * dt;
            if (!isfinite(integrated)) {
                failed = true;
                log_surv = 0.0;
                status = 1;
            } else if (integrated == 0.0) {
                log_surv = 0.0;
                status = 2;
            } else {
                const double lld = (carried & 2u) ? s.c_logd : log(ld);
                const double lrd = log(rd);
                s.c_logd = lrd;
                s.c_valid |= 2u;
                const double le = kLn2 + lld + lrd - log(integrated);
                if (le >= kLogMaxExpArgument) {
                    log_surv = 0.0;
                    status = 4;
                } else if (le <= kLogMinPositive) {
                    log_surv = le;
                    status = 3;
                } else {
                    log_surv = interval_log_survival(le);
                    status = 0;
                }
            }
        }
        s.hit_log = s.hit_log + log(rsafe);
        s.hit_prod = s.hit_prod * rsafe;
    } else {
        if (s.initial_touched) return;
        // exact_interval with ln(ls) and ln(ld) carried
        if (!(ls > 0.0) || !isfinite(ls) || !(rs > 0.0) || !isfinite(rs) || !(lv >= 0.0) || !isfinite(lv) ||
            !(rv >= 0.0) || !isfinite(rv)) {
            failed = true;
            log_surv = 0.0;
            status = 1;
        } else {
            const double lb = log(p.barrier);
            const double lls = (carried & 1u) ? s.c_end : log(ls);
            const double lrs = log(rs);
            s.c_end = lrs;
            s.c_valid |= 1u;
            const double ld = up ? lb - lls : lls - lb;
            const double rd = up ? lb - lrs : lrs - lb;
            if (ld <= 0.0 || rd <= 0.0) {
                log_surv = -INFINITY;
                status = 1;  // touched
            } else {
                const double integrated = (0.5 * lv + 0.5 * rv) * dt;
                if (!isfinite(integrated)) {
                    failed = true;
                    log_surv = 0.0;
                    status = 1;
                } else if (integrated == 0.0) {
                    log_surv = 0.0;
                    status = 2;
                } else {
                    const double lld = (carried & 2u) ? s.c_logd : log(ld);
                    const double lrd = log(rd);
                    s.c_logd = lrd;
                    s.c_valid |= 2u;
                    const double le = kLn2 + lld + lrd - log(integrated);
                    if (le >= kLogMaxExpArgument) {
                        log_surv = 0.0;
                        status = 4;
                    } else if (le <= kLogMinPositive) {
                        log_surv = le;
                        status = 3;
                    } else {
                        log_surv = interval_log_survival(le);
                        status = 0;
                    }
                }
            }
        }
        if (status == 1) s.touched = 1;
    }
    s.log_sum += log_surv;
    count_status(s, status);
}

// Start of a continuous-barrier path at the initial state (the spot).
MCG_HD void barrier_begin(const ProductParams& p, ProductAcc& s, double h,
                                              double spot, bool& failed) {
    const bool up = p.barrier_direction == MCG_BARRIER_UP;
    if (h > 0.0) {
        double safety, eld;
        smooth_endpoint(up, spot, p.barrier, h, safety, eld, failed);
        s.hit_log = 0.0 + log(safety);
        s.hit_prod = 1.0 * safety;
    } else {
        s.initial_touched = up ? spot >= p.barrier : spot <= p.barrier;
    }
}

// Final survival and component 10..17 diagnostics,
// crates/pricing/src/engine/payoff/barrier.rs:40-153,204-226.
MCG_HD double barrier_finish(ProductAcc& s, double h, uint32_t intervals,
                                                 double* diag) {
    const double finite = static_cast<double>(s.counts & 0xffffu);
    const double zero = static_cast<double>(s.counts >> 16);
    const double under = static_cast<double>(s.counts2 & 0xffffu);
    const double certain = static_cast<double>(s.counts2 >> 16);
    if (h > 0.0) {
        diag[0] = 1.0 - s.hit_prod;
        diag[1] = 1.0 - 1.0;
        diag[2] = 1.0 - exp(s.log_sum);
        diag[3] = static_cast<double>(intervals);
        diag[4] = finite;
        diag[5] = zero;
        diag[6] = under;
        diag[7] = certain;
        return exp(s.log_sum + s.hit_log);
    }
    const bool endpoint_touched = s.initial_touched || s.touched;
    const double surv = exp(s.log_sum);
    diag[0] = endpoint_touched ? 1.0 : 0.0;
    diag[1] = 0.0;
    diag[2] = endpoint_touched ? 0.0 : 1.0 - surv;
    diag[3] = s.initial_touched ? 0.0 : static_cast<double>(intervals);
    diag[4] = finite;
    diag[5] = zero;
    diag[6] = under;
    diag[7] = certain;
    return endpoint_touched ? 0.0 : surv;
}

// continuous_barrier_payoff_terms, barrier.rs:307-355 (value only).
MCG_HD double barrier_value(const ProductParams& p, double terminal,
                                                double survival) {
    const bool call = p.side == MCG_CALL;
    const double in = call ? terminal - p.strike : p.strike - terminal;
    const double vanilla = fmax(in, 0.0) * p.notional;
    const double rebate = p.has_rebate ? p.rebate : 0.0;
    if (p.barrier_style == MCG_KNOCK_OUT) return rebate + survival * (vanilla - rebate);
    return vanilla + survival * (rebate - vanilla);
}

// Undiscounted payoff of a discrete product from its accumulator.
MCG_HD double acc_payoff(const ProductParams& p, const ProductAcc& s,
                                             double smoothing) {
    const bool call = p.side == MCG_CALL;
    switch (p.kind) {
    case MCG_PRODUCT_EUROPEAN: {
        const double in = call ? s.terminal - p.strike : p.strike - s.terminal;
        return (in >= 0.0 ? in : 0.0) * p.notional;
    }
    case MCG_PRODUCT_DIGITAL: {
        const double dist = call ? s.terminal - p.strike : p.strike - s.terminal;
        double ind;
        if (smoothing > 0.0) {
            double comp;
            ind = smooth_indicator(smoothing, dist, comp).value;
        } else {
            ind = dist >= 0.0 ? 1.0 : 0.0;
        }
        const double base = p.digital_payout == MCG_DIGITAL_ASSET ? s.terminal * p.payout : p.payout;
        return ind * base;
    }
    case MCG_PRODUCT_ASIAN:
    case MCG_PRODUCT_LOOKBACK: {
        const double in = call ? s.a - p.strike : p.strike - s.a;
        return (in >= 0.0 ? in : 0.0) * p.notional;
    }
    case MCG_PRODUCT_DISCRETE_BARRIER: {
        const double in = call ? s.terminal - p.strike : p.strike - s.terminal;
        const double vanilla = (in >= 0.0 ? in : 0.0) * p.notional;
        const double active = p.barrier_style == MCG_KNOCK_OUT ? 1.0 - s.a : s.a;
        double value = vanilla * active;
        if (p.has_rebate) value = value + (1.0 - active) * p.rebate;
        return value;
    }
    default:
        return 0.0;
    }
}

}  // namespace mcg

namespace mcg {

// ------------------------------------------- reverse of the bridge terms

// Log-survival derivatives of one exact interval,
// BarrierBridgeInterval::evaluate, barrier_bridge.rs:446-528 (constant barrier).
struct ExactIntervalDerivs {
    double d_left_state, d_right_state, d_left_var, d_right_var;
};

// ld, rd: the endpoints' signed log distances to the barrier (log(B) - log(state)
// up, log(state) - log(B) down); lld, lrd: their logarithms, read only when
// ld, rd > 0.
MCG_HD ExactIntervalDerivs exact_interval_derivs(bool up, double ls, double rs, double ld, double rd, double lld,
                                                 double lrd, double lv, double rv, double dt) {
    ExactIntervalDerivs d{0.0, 0.0, 0.0, 0.0};
    if (ld <= 0.0 || rd <= 0.0) return d;
    const double average = 0.5 * lv + 0.5 * rv;
    const double integrated = average * dt;
    if (!isfinite(integrated) || integrated == 0.0) return d;
    const double le = kLn2 + lld + lrd - log(integrated);
    if (le >= kLogMaxExpArgument) return d;
    double led;
    if (le <= kLogMinPositive) {
        led = 1.0;
    } else {
        const double e = exp(le);
        led = e / expm1(e);
    }
    const double ldd = led / ld;
    const double rdd = led / rd;
    const double ivd = -led / integrated;
    const double sign = up ? 1.0 : -1.0;
    const double avd = ivd * dt;
    d.d_left_state = -sign * ldd / ls;
    d.d_right_state = -sign * rdd / rs;
    d.d_left_var = 0.5 * avd;
    d.d_right_var = 0.5 * avd;
    return d;
}

// Smoothed endpoint with its derivatives (barrier_bridge.rs:160-249, affine
// scale 1): safety weight, effective log distance, d(hit weight)/d(state) and
// d(effective log distance)/d(state).
struct SmoothEndpointFull {
    double safety, eld, hit_d_state, eld_d_state;
};

MCG_HD SmoothEndpointFull smooth_endpoint_full(bool up, double state, double barrier, double h) {
    SmoothEndpointFull e{1.0, 1.0, 0.0, 0.0};
    const double sign = up ? 1.0 : -1.0;
    const double signed_hit = 1.0 * sign * (state - barrier);
    const SmoothD hit = smooth_indicator(h, signed_hit, e.safety);
    const SmoothD safe = smooth_positive_part(h, -signed_hit);
    const double spot_barrier = 1.0 * barrier;
    const double denominator = up ? spot_barrier - safe.value : spot_barrier + safe.value;
    e.eld = up ? -log1p(-safe.value / spot_barrier) : log1p(safe.value / spot_barrier);
    const double hit_x = hit.first;
    const double safe_x = -safe.first;
    const double distance_safe = 1.0 / denominator;
    const double distance_x = distance_safe * safe_x;
    const double x_state = 1.0 * sign;
    e.hit_d_state = hit_x * x_state;
    e.eld_d_state = distance_x * x_state;
    return e;
}

// Log-survival derivatives of one smoothed interval with respect to the two
// effective log distances and the two local variances (barrier_bridge.rs:276-357),
// given lld = log(ld) and lrd = log(rd).
struct SmoothIntervalDerivs {
    double d_left_distance, d_right_distance, d_left_var, d_right_var;
};

MCG_HD SmoothIntervalDerivs smooth_interval_derivs(double ld, double rd, double lld, double lrd, double lv,
                                                   double rv, double dt) {
    SmoothIntervalDerivs d{0.0, 0.0, 0.0, 0.0};
    if (ld == 0.0 || rd == 0.0) return d;
    const double average = 0.5 * lv + 0.5 * rv;
    const double integrated = average * dt;
    if (!isfinite(integrated) || integrated == 0.0) return d;
    const double le = kLn2 + lld + lrd - log(integrated);
    if (le >= kLogMaxExpArgument) return d;
    double led;
    if (le <= kLogMinPositive) {
        led = 1.0;
    } else {
        const double e = exp(le);
        led = e / expm1(e);
    }
    const double ivd = -led / integrated;
    const double avd = ivd * dt;
    d.d_left_distance = led / ld;
    d.d_right_distance = led / rd;
    d.d_left_var = 0.5 * avd;
    d.d_right_var = 0.5 * avd;
    return d;
}

// One observation node of a continuous-barrier path as the bridge adjoint
// reads it: computed once per node and shared by the two intervals that meet
// there (and by the node's smoothed hit factor).
struct BarrierEndpoint {
    double d;      // smoothed: effective log distance; exact: signed log distance to the barrier
    double log_d;  // log(d)
    double d_state, hit_d_state, safety;  // smoothed: d(d)/d(state), d(hit weight)/d(state), safety weight
};

// lb = log(barrier).
MCG_HD BarrierEndpoint barrier_endpoint(bool up, double barrier, double lb, double h, double state) {
    BarrierEndpoint n{1.0, 0.0, 0.0, 0.0, 1.0};
    if (h > 0.0) {
        const SmoothEndpointFull e = smooth_endpoint_full(up, state, barrier, h);
        n.d = e.eld;
        n.d_state = e.eld_d_state;
        n.hit_d_state = e.hit_d_state;
        n.safety = e.safety;
    } else {
        const double ls = log(state);
        n.d = up ? lb - ls : ls - lb;
    }
    n.log_d = log(n.d);
    return n;
}

// Adjoint of the continuous-barrier bridge for one interval [k-1, k]:
// contributions to the state seeds and the direct variance seeds of both
// nodes, given the log-survival adjoint lsa
// (pathwise_local_vol.rs:219-271; barrier.rs:82-118 for the smoothed reverse).
struct IntervalAdjoint {
    double left_state, right_state, left_var, right_var;
};

MCG_HD IntervalAdjoint bridge_interval_adjoint(bool up, double h, double lsa, const BarrierEndpoint& L,
                                               const BarrierEndpoint& R, double ls, double rs, double lv, double rv,
                                               double dt) {
    IntervalAdjoint a{0.0, 0.0, 0.0, 0.0};
    if (!(dt > 0.0)) return a;
    if (h > 0.0) {
        const SmoothIntervalDerivs d = smooth_interval_derivs(L.d, R.d, L.log_d, R.log_d, lv, rv, dt);
        a.left_state = 0.0 * L.hit_d_state + (lsa * d.d_left_distance) * L.d_state;
        a.right_state = 0.0 * R.hit_d_state + (lsa * d.d_right_distance) * R.d_state;
        a.left_var = lsa * d.d_left_var;
        a.right_var = lsa * d.d_right_var;
        return a;
    }
    const ExactIntervalDerivs d =
        exact_interval_derivs(up, ls, rs, L.d, R.d, L.log_d, R.log_d, lv, rv, dt);
    a.left_state = lsa * d.d_left_state;
    a.right_state = lsa * d.d_right_state;
    a.left_var = lsa * d.d_left_var;
    a.right_var = lsa * d.d_right_var;
    return a;
}

// The same for a lone interval.
MCG_HD IntervalAdjoint barrier_interval_adjoint(bool up, double barrier, double h, double lsa,
                                                double ls, double rs, double lv, double rv,
                                                double dt) {
    if (!(dt > 0.0)) return IntervalAdjoint{0.0, 0.0, 0.0, 0.0};
    const double lb = log(barrier);
    const BarrierEndpoint L = barrier_endpoint(up, barrier, lb, h, ls);
    const BarrierEndpoint R = barrier_endpoint(up, barrier, lb, h, rs);
    return bridge_interval_adjoint(up, h, lsa, L, R, ls, rs, lv, rv, dt);
}

// Adjoint of a smoothed hit factor at one node: -lsa * d(hit)/d(state) / safety.
MCG_HD double hit_factor_adjoint(const BarrierEndpoint& n, double lsa) {
    return n.safety == 0.0 ? 0.0 : -lsa * n.hit_d_state / n.safety;
}

MCG_HD double hit_factor_adjoint(bool up, double barrier, double h, double lsa, double state) {
    const SmoothEndpointFull e = smooth_endpoint_full(up, state, barrier, h);
    return e.safety == 0.0 ? 0.0 : -lsa * e.hit_d_state / e.safety;
}

}  // namespace mcg

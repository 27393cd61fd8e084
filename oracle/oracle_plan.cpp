// oracle_plan.cpp -- plan compile and execute of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY: the oracle the CUDA engine is compared against.
// It restates SimulationPlan::execute and the per-unit closures of
// msfmfjt/rust-pricing-library (paths relative to that project) and evaluates
// the same `mcg_plan_desc` the engine takes.  Fixed reduction blocks are run on
// a thread pool and merged in the reference's fixed tree, so the result does not
// depend on the thread count (crates/pricing/src/engine/mc/execution.rs:334-744).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../include/mcg.h"
#include "oracle_core.h"

namespace oracle {
namespace {

constexpr int kComponents = MCG_PATHWISE_COMPONENTS;
// Per-unit values: the reference's 18 components plus the adjoint Delta and
// the bumped-adjoint Gamma of the local-volatility adjoint.
constexpr int kWidth = kComponents + 2;
constexpr double kNormal95 = 1.959963984540054;  // plan/simulation.rs:24
constexpr double kLogMaxExpArgument = 6.564958884017094;   // barrier_bridge.rs:9
constexpr double kLogMinPositive = -744.4400719213812;     // barrier_bridge.rs:10
constexpr double kLn2 = 0.6931471805599453;

thread_local std::string g_error;

struct Failure {
    int code = MCG_OK;
    uint32_t step = 0;
    double value = 0.0;
};

uint64_t bits_of(double v) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
}

// ----------------------------------------------------------- smoothing

// CompactC2Smoothing, crates/pricing/src/product/smoothing.rs:29-198.
struct Deriv {
    double value, first, second;
};
struct BinaryDeriv {
    double value, left_first, right_first;
};

double transition_coordinate(double input, double h) {
    const double full = 2.0 * h;
    if (std::isfinite(full)) return (input + h) / full;
    if (input < 0.0) return 0.5 * ((input + h) / h);
    return 0.5 * (input / h + 1.0);
}

double quintic(double u) { return u * u * u * (10.0 + u * (-15.0 + 6.0 * u)); }

void interior_indicator(double input, double h, double u, Deriv& d, double& complement) {
    const double hit = quintic(u);
    const double safety = 1.0 - hit;
    double z, value, comp, sign;
    if (safety <= 32.0 * 2.220446049250313e-16) {
        z = transition_coordinate(-input, h);
        const double tail = quintic(z);
        value = 1.0 - tail;
        comp = tail;
        sign = -1.0;
    } else {
        z = u;
        value = hit;
        comp = safety;
        sign = 1.0;
    }
    const double z2 = z * z;
    const double z3 = z2 * z;
    const double omz = 1.0 - z;
    const double first = 15.0 * z2 * omz * omz / h;
    const double numerator = sign * (120.0 * z3 - 180.0 * z2 + 60.0 * z);
    const double denominator = 4.0 * h * h;
    const double second = std::isnormal(denominator) ? numerator / denominator
                                                     : ((0.25 * numerator) / h) / h;
    d = {value, first, second};
    complement = comp;
}

void indicator_with_complement(double h, double input, Deriv& d, double& complement) {
    if (input <= -h) {
        d = {0.0, 0.0, 0.0};
        complement = 1.0;
        return;
    }
    if (input >= h) {
        d = {1.0, 0.0, 0.0};
        complement = 0.0;
        return;
    }
    interior_indicator(input, h, transition_coordinate(input, h), d, complement);
}

Deriv indicator(double h, double input) {
    Deriv d;
    double c;
    indicator_with_complement(h, input, d, c);
    return d;
}

void positive_part_with_complement(double h, double input, Deriv& d, double& complement) {
    if (input <= -h) {
        d = {0.0, 0.0, 0.0};
        complement = 1.0;
        return;
    }
    if (input >= h) {
        d = {input, 1.0, 0.0};
        complement = 0.0;
        return;
    }
    const double u = transition_coordinate(input, h);
    const double u2 = u * u;
    const double u4 = u2 * u2;
    Deriv ind;
    double comp;
    interior_indicator(input, h, u, ind, comp);
    const double scaled_u4 = 2.0 * h * u4;
    const double poly = 2.5 + u * (-3.0 + u);
    const double value = std::isnormal(scaled_u4) ? scaled_u4 * poly : (2.0 * u4 * poly) * h;
    d = {value, ind.value, ind.first};
    complement = comp;
}

Deriv positive_part(double h, double input) {
    Deriv d;
    double c;
    positive_part_with_complement(h, input, d, c);
    return d;
}

BinaryDeriv smooth_maximum(double h, double left, double right) {
    const double diff = left - right;
    if (diff >= h) return {left, 1.0, 0.0};
    if (diff <= -h) return {right, 0.0, 1.0};
    Deriv p;
    double rf;
    positive_part_with_complement(h, diff, p, rf);
    return {right + p.value, p.first, rf};
}

BinaryDeriv smooth_minimum(double h, double left, double right) {
    const double diff = left - right;
    if (diff >= h) return {right, 0.0, 1.0};
    if (diff <= -h) return {left, 1.0, 0.0};
    Deriv p;
    double lf;
    positive_part_with_complement(h, diff, p, lf);
    return {left - p.value, lf, p.first};
}

// ------------------------------------------------------ barrier bridge

// Status of one bridge interval, barrier_bridge.rs:18-25.
enum BridgeStatus { kFinite = 0, kTouched = 1, kZeroVariance = 2, kUnderflow = 3, kCertain = 4 };

struct ExactInterval {
    int status;
    double log_survival;
    double d_left_state, d_right_state, d_left_var, d_right_var;
};

// BarrierBridgeInterval::evaluate, barrier_bridge.rs:446-528 (constant barrier, B = 1).
bool exact_interval(bool up, double ls, double rs, double lb, double rb, double lv, double rv,
                    double dt, ExactInterval& out, Failure& f) {
    if (!(ls > 0.0) || !std::isfinite(ls) || !(rs > 0.0) || !std::isfinite(rs)) {
        f = {MCG_ERR_BARRIER_BRIDGE, 0, ls};
        return false;
    }
    if (!(lv >= 0.0) || !std::isfinite(lv) || !(rv >= 0.0) || !std::isfinite(rv) ||
        !(dt > 0.0) || !std::isfinite(dt)) {
        f = {MCG_ERR_BARRIER_BRIDGE, 0, lv};
        return false;
    }
    const double left_distance = up ? std::log(lb) - std::log(ls) : std::log(ls) - std::log(lb);
    const double right_distance = up ? std::log(rb) - std::log(rs) : std::log(rs) - std::log(rb);
    out = {kTouched, -INFINITY, 0, 0, 0, 0};
    if (left_distance <= 0.0 || right_distance <= 0.0) return true;
    const double average = 0.5 * lv + 0.5 * rv;
    const double integrated = average * dt;
    if (!std::isfinite(integrated)) {
        f = {MCG_ERR_BARRIER_BRIDGE, 0, integrated};
        return false;
    }
    if (integrated == 0.0) {
        out = {kZeroVariance, 0.0, 0, 0, 0, 0};
        return true;
    }
    const double log_exponent =
        kLn2 + std::log(left_distance) + std::log(right_distance) - std::log(integrated);
    if (log_exponent >= kLogMaxExpArgument) {
        out = {kCertain, 0.0, 0, 0, 0, 0};
        return true;
    }
    int status;
    double log_survival, led;
    if (log_exponent <= kLogMinPositive) {
        status = kUnderflow;
        log_survival = log_exponent;
        led = 1.0;
    } else {
        const double exponent = std::exp(log_exponent);
        const double survival = -std::expm1(-exponent);
        status = kFinite;
        log_survival = std::log(survival);
        led = exponent / std::expm1(exponent);
    }
    const double ldd = led / left_distance;
    const double rdd = led / right_distance;
    const double ivd = -led / integrated;
    const double sign = up ? 1.0 : -1.0;
    const double avd = ivd * dt;
    out.status = status;
    out.log_survival = log_survival;
    out.d_left_state = -sign * ldd / ls;
    out.d_right_state = -sign * rdd / rs;
    out.d_left_var = 0.5 * avd;
    out.d_right_var = 0.5 * avd;
    return true;
}

// SmoothedBarrierBridgeEndpoint, barrier_bridge.rs:160-249 (affine scale 1 here
// generalised to the coordinate's B).
struct SmoothEndpoint {
    double hit_weight, safety_weight, eld;
    double hit_d_state, eld_d_state;
};

bool smooth_endpoint(bool up, double state, double barrier, double scale, double h,
                     SmoothEndpoint& e, Failure& f) {
    if (!(state > 0.0) || !std::isfinite(state)) {
        f = {MCG_ERR_BARRIER_BRIDGE, 0, state};
        return false;
    }
    const double sign = up ? 1.0 : -1.0;
    const double diff = state - barrier;
    const double signed_hit = scale * sign * diff;
    Deriv hit;
    double safety;
    indicator_with_complement(h, signed_hit, hit, safety);
    const Deriv safe = positive_part(h, -signed_hit);
    const double spot_barrier = scale * barrier;
    const double denominator = up ? spot_barrier - safe.value : spot_barrier + safe.value;
    if (!std::isfinite(denominator) || denominator <= 0.0) {
        f = {MCG_ERR_BARRIER_BRIDGE, 0, safe.value};
        return false;
    }
    const double eld = up ? -std::log1p(-safe.value / spot_barrier)
                          : std::log1p(safe.value / spot_barrier);
    const double hit_x = hit.first;
    const double safe_x = -safe.first;
    const double distance_safe = 1.0 / denominator;
    const double distance_x = distance_safe * safe_x;
    const double x_state = scale * sign;
    e.hit_weight = hit.value;
    e.safety_weight = safety;
    e.eld = eld;
    e.hit_d_state = hit_x * x_state;
    e.eld_d_state = distance_x * x_state;
    return true;
}

struct SmoothInterval {
    int status;
    double log_survival;
    SmoothEndpoint left, right;
    double d_left_distance, d_right_distance, d_left_var, d_right_var;
};

// SmoothedBarrierBridgeInterval::evaluate, barrier_bridge.rs:276-357.
bool smooth_interval(bool up, double ls, double rs, double lb, double rb, double lscale,
                     double rscale, double lv, double rv, double dt, double h, SmoothInterval& out,
                     Failure& f) {
    if (!smooth_endpoint(up, ls, lb, lscale, h, out.left, f)) return false;
    if (!smooth_endpoint(up, rs, rb, rscale, h, out.right, f)) return false;
    if (!(lv >= 0.0) || !std::isfinite(lv) || !(rv >= 0.0) || !std::isfinite(rv) ||
        !(dt > 0.0) || !std::isfinite(dt)) {
        f = {MCG_ERR_BARRIER_BRIDGE, 0, lv};
        return false;
    }
    out.d_left_distance = out.d_right_distance = out.d_left_var = out.d_right_var = 0.0;
    const double ld = out.left.eld, rd = out.right.eld;
    if (ld == 0.0 || rd == 0.0) {
        out.status = kTouched;
        out.log_survival = -INFINITY;
        return true;
    }
    const double average = 0.5 * lv + 0.5 * rv;
    const double integrated = average * dt;
    if (!std::isfinite(integrated)) {
        f = {MCG_ERR_BARRIER_BRIDGE, 0, integrated};
        return false;
    }
    if (integrated == 0.0) {
        out.status = kZeroVariance;
        out.log_survival = 0.0;
        return true;
    }
    const double log_exponent = kLn2 + std::log(ld) + std::log(rd) - std::log(integrated);
    if (log_exponent >= kLogMaxExpArgument) {
        out.status = kCertain;
        out.log_survival = 0.0;
        return true;
    }
    double led;
    if (log_exponent <= kLogMinPositive) {
        out.status = kUnderflow;
        out.log_survival = log_exponent;
        led = 1.0;
    } else {
        const double exponent = std::exp(log_exponent);
        const double survival = -std::expm1(-exponent);
        out.status = kFinite;
        out.log_survival = std::log(survival);
        led = exponent / std::expm1(exponent);
    }
    const double ivd = -led / integrated;
    const double avd = ivd * dt;
    out.d_left_distance = led / ld;
    out.d_right_distance = led / rd;
    out.d_left_var = 0.5 * avd;
    out.d_right_var = 0.5 * avd;
    return true;
}

// ------------------------------------------------------------- dividends

// AffineDividendCoordinate, crates/pricing/src/market/dividend.rs:137-208:
// the observed spot is a S0 + b f of the canonical state f; spot_scale is its
// derivative scale under a spot bump with the cash held fixed.
struct Coord {
    double a = 0.0, b = 1.0, spot_scale = 1.0;
    // at_spot, dividend.rs:170-181.
    Coord at_spot(double original, double spot) const {
        if (original == spot) return *this;
        return {a * original / spot, spot_scale - (spot_scale - b) * original / spot, spot_scale};
    }
    double spot_of(double s0, double f) const { return a * s0 + b * f; }
};

struct DividendEvent {
    double t, cash, alpha, beta;
};

// AffineDividendTransform::new_with_carry_curves and its coordinates,
// dividend.rs:283-491 (compile_event :622-642, validation :644-690).
struct Dividends {
    std::vector<DividendEvent> ev;
    double spot = 0.0, reserve = 0.0;
    const Curve* rc = nullptr;
    const Curve* qc = nullptr;

    bool compile(const mcg_dividends& d, double s0, const Curve& r, const Curve& q) {
        ev.clear();
        spot = s0;
        rc = &r;
        qc = &q;
        for (uint32_t i = 0; i < d.count; ++i) {
            const double t = d.ex_times[i], cash = d.fixed_cash[i], beta = d.proportional[i];
            if (!std::isfinite(t) || t < 0.0) return false;
            if (!(std::isfinite(cash) && cash >= 0.0)) return false;
            if (!(std::isfinite(beta) && beta >= 0.0 && beta < 1.0)) return false;
            if (i && !(t > d.ex_times[i - 1])) return false;
            const double alpha = cash / s0;
            if (!std::isfinite(alpha)) return false;
            ev.push_back({t, cash, alpha, beta});
        }
        // compile_reserve, dividend.rs:332-354
        double proportional = 1.0, res = 0.0;
        for (const auto& e : ev) {
            proportional *= 1.0 - e.beta;
            const double discount = std::exp(rc->log_discount(e.t)) / std::exp(qc->log_discount(e.t));
            res += e.cash / proportional * discount;
        }
        const double residual = s0 - res;
        if (!std::isfinite(res) || !std::isfinite(residual) || residual <= 0.0) return false;
        reserve = res;
        return true;
    }
    Coord initial() const { return {reserve / spot, (spot - reserve) / spot, 1.0}; }
    // carry, dividend.rs:366-392
    Coord carry(Coord c, double start, double end) const {
        if (c.a == 0.0 || start == end) return c;
        const double g = qc->log_discount(end) - rc->log_discount(end) - qc->log_discount(start) +
                         rc->log_discount(start);
        c.a *= std::exp(g);
        return c;
    }
    // after, dividend.rs:187-208
    static Coord after(Coord c, const DividendEvent& e) {
        return {(1.0 - e.beta) * c.a - e.alpha, (1.0 - e.beta) * c.b, (1.0 - e.beta) * c.spot_scale};
    }
    // coordinate_after_time, dividend.rs:434-460
    Coord after_time(double time) const {
        if (ev.empty()) return Coord{};  // no dividends: the identity
        Coord c = initial();
        double prev = 0.0;
        for (const auto& e : ev) {
            if (!(e.t <= time)) break;
            c = carry(c, prev, e.t);
            c = after(c, e);
            prev = e.t;
        }
        c = carry(c, prev, time);
        bool settled = true;
        for (const auto& e : ev) settled = settled && (e.t <= time || e.cash == 0.0);
        if (settled) c.a = 0.0;
        return c;
    }
    // event_timeline's `before` entry of event i, dividend.rs:492-518
    Coord before_event(size_t i) const {
        if (ev.empty()) return Coord{};
        Coord c = initial();
        double prev = 0.0;
        size_t last_cash = ev.size();
        for (size_t k = ev.size(); k-- > 0;)
            if (ev[k].cash != 0.0) {
                last_cash = k;
                break;
            }
        for (size_t k = 0; k < ev.size(); ++k) {
            const Coord before = carry(c, prev, ev[k].t);
            if (k == i) return before;
            Coord aft = after(before, ev[k]);
            if (last_cash == ev.size() || k >= last_cash) aft.a = 0.0;
            c = aft;
            prev = ev[k].t;
        }
        return c;
    }
    // index of the event at exactly `time`, or -1
    long event_at(double time) const {
        for (size_t k = 0; k < ev.size(); ++k)
            if (bits_of(ev[k].t) == bits_of(time)) return static_cast<long>(k);
        return -1;
    }
};

// ------------------------------------------------------------- the plan

struct Product {
    mcg_product_desc d;
    std::vector<double> weights;
    // Discrete barrier / lookback monitoring flags (every observation without flags).
    bool monitored(size_t i) const {
        return (d.kind != MCG_PRODUCT_DISCRETE_BARRIER && d.kind != MCG_PRODUCT_LOOKBACK) ||
               weights.empty() || weights[i] != 0.0;
    }
};

struct Plan {
    int model, engine;
    uint64_t seed, units;
    uint32_t scrambles;
    bool antithetic, bridge_flag;
    uint64_t block;
    double spot, vol, discount, expiry, total_variance;
    Curve rc, qc;
    std::vector<double> obs_t, obs_fwd;
    std::vector<Product> products;
    bool req_delta, req_gamma, req_vega, req_nodes;
    double gamma_bump, spot_bump, vol_bump, smoothing;
    // local volatility
    Grid grid;
    std::vector<double> nodes, fwd[3];  // base, down, up
    double bump_spot[3];
    std::vector<uint32_t> obs_node;
    BridgePlan bridge;
    bool use_bridge = false;
    // rqmc
    std::vector<uint32_t> dirs;
    std::vector<Scramble> scr;  // scramble-major, dimension-minor
    uint32_t dimension = 0;
    uint32_t domain = 0;  // RandomDomain of the pseudo stream: Valuation 0, LsmTrain 1
    // discrete dividends: observation coordinates after (and, on an ex-date,
    // before) the dividend; local volatility per spot runtime and node, and the
    // post-dividend spot checks of the ex-date nodes
    Dividends div;
    double residual_spot = 0.0;
    std::vector<Coord> obs_post, obs_pre;
    std::vector<char> obs_has_pre;
    std::vector<Coord> node_post[3], node_pre[3];
    std::vector<char> node_has_pre;
    std::vector<std::pair<size_t, Coord>> checks[3];
    bool risk_enabled() const { return req_delta || req_gamma || req_vega; }
    bool has_continuous_barrier() const {
        for (const auto& p : products)
            if (p.d.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) return true;
        return false;
    }
};

double forward_at(const Plan& p, double spot, double t) {
    return spot * std::exp(p.qc.log_discount(t) - p.rc.log_discount(t));
}

bool fail(const char* msg) {
    g_error = msg;
    return false;
}

// LocalVolTimeGrid::compile, crates/pricing/src/engine/processes/local_vol.rs:167-237.
bool compile_time_grid(std::vector<double> events, double maximum_step,
                       std::vector<double>& nodes) {
    std::sort(events.begin(), events.end(),
              [](double a, double b) { return total_key(a) < total_key(b); });
    events.erase(std::unique(events.begin(), events.end(),
                             [](double a, double b) { return bits_of(a) == bits_of(b); }),
                 events.end());
    if (bits_of(events[0]) != 0) events.insert(events.begin(), 0.0);
    nodes.clear();
    nodes.push_back(0.0);
    for (size_t i = 0; i + 1 < events.size(); ++i) {
        const double left = events[i], right = events[i + 1];
        if (right <= left) continue;
        const double interval = right - left;
        double steps_f = std::ceil(interval / maximum_step);
        size_t steps = steps_f < 1.0 ? 1 : static_cast<size_t>(steps_f);
        const double sub = interval / static_cast<double>(steps);
        for (size_t k = 1; k < steps; ++k) nodes.push_back(left + sub * static_cast<double>(k));
        nodes.push_back(right);
    }
    return true;
}

bool build_plan(const mcg_plan_desc* d, Plan& p) {
    if (!d || d->abi_version != MCG_ABI_VERSION) return fail("abi_version");
    p.model = d->model;
    p.engine = d->engine;
    p.seed = d->master_seed;
    p.units = d->sampling_units;
    p.scrambles = d->scramble_count;
    p.antithetic = d->antithetic != 0;
    p.bridge_flag = d->brownian_bridge != 0;
    p.block = d->reduction_block_size ? d->reduction_block_size : 4096;
    p.spot = d->spot;
    p.vol = d->volatility;
    p.rc.set(d->discount_curve.times, d->discount_curve.discount_factors,
             d->discount_curve.pillar_count);
    p.qc.set(d->dividend_curve.times, d->dividend_curve.discount_factors,
             d->dividend_curve.pillar_count);
    p.discount = std::exp(p.rc.log_discount(d->payment_time));
    p.obs_t.assign(d->observation_times, d->observation_times + d->observation_count);
    p.expiry = p.obs_t.back();
    p.residual_spot = p.spot;
    if (d->discrete_dividends.count) {
        if (!p.div.compile(d->discrete_dividends, p.spot, p.rc, p.qc)) return fail("dividends");
        p.residual_spot = p.spot - p.div.reserve;
        for (uint32_t i = 0; i < d->product_count; ++i)
            if (d->products[i].kind == MCG_PRODUCT_CONTINUOUS_BARRIER || d->products[i].kind == MCG_PRODUCT_AMERICAN)
                return fail("dividends with a continuous barrier or early exercise");
        if (d->model == MCG_MODEL_LOCAL_VOLATILITY && (d->request_vega || d->request_local_vega_nodes))
            return fail("local-volatility Vega with dividends");
    }
    for (double t : p.obs_t) {
        p.obs_post.push_back(p.div.after_time(t));
        const long k = p.div.event_at(t);
        p.obs_has_pre.push_back(k >= 0);
        p.obs_pre.push_back(k >= 0 ? p.div.before_event(static_cast<size_t>(k)) : Coord{});
    }
    for (double t : p.obs_t) p.obs_fwd.push_back(forward_at(p, p.spot, t));
    for (uint32_t i = 0; i < d->product_count; ++i) {
        Product pr;
        pr.d = d->products[i];
        if (pr.d.observation_weights)
            pr.weights.assign(pr.d.observation_weights,
                              pr.d.observation_weights + d->observation_count);
        pr.d.observation_weights = nullptr;
        p.products.push_back(pr);
    }
    p.req_delta = d->request_delta != 0;
    p.req_gamma = d->request_gamma != 0;
    p.req_vega = d->request_vega != 0;
    p.req_nodes = d->request_local_vega_nodes != 0;
    p.smoothing = d->smoothing_half_width;
    // Validation bumps, crates/pricing/src/engine/compile/simulation.rs:481-502.
    p.gamma_bump = d->gamma_bump_relative ? p.spot * d->gamma_bump : d->gamma_bump;
    p.spot_bump = p.req_gamma ? p.gamma_bump : std::min(p.spot * 1.0e-4, 0.5 * p.residual_spot);
    if (p.model == MCG_MODEL_BLACK_SCHOLES) {
        p.total_variance = p.vol * p.vol * p.expiry;
        p.vol_bump = p.vol == 0.0 ? 0.0 : std::min(1.0e-4, p.vol * 0.5);
    } else {
        const auto& g = d->local_variance;
        p.grid.t.assign(g.time_nodes, g.time_nodes + g.time_count);
        p.grid.x.assign(g.log_moneyness_nodes, g.log_moneyness_nodes + g.log_moneyness_count);
        p.grid.v.assign(g.values, g.values + static_cast<size_t>(g.time_count) * g.log_moneyness_count);
        p.grid.floor = g.floor;
        p.grid.cap = g.cap;
        double maximum_step = 0.0;
        for (size_t i = 0; i + 1 < p.grid.t.size(); ++i)
            maximum_step = std::max(maximum_step, p.grid.t[i + 1] - p.grid.t[i]);
        std::vector<double> events = p.grid.t;
        events.insert(events.end(), p.obs_t.begin(), p.obs_t.end());
        // ex-dividend times up to expiry are grid events (compile/local_vol.rs:38-52)
        for (const auto& e : p.div.ev)
            if (e.t <= p.expiry) events.push_back(e.t);
        compile_time_grid(events, maximum_step, p.nodes);
        p.bump_spot[0] = p.spot;
        p.bump_spot[1] = p.spot - p.spot_bump;
        p.bump_spot[2] = p.spot + p.spot_bump;
        for (int k = 0; k < 3; ++k)
            for (double t : p.nodes) p.fwd[k].push_back(forward_at(p, p.bump_spot[k], t));
        // node coordinates of each spot runtime, the transform recompiled at
        // that spot (local_vol_runtime_for_spot, risk/pathwise_local_vol.rs:51-69)
        p.node_has_pre.clear();
        for (double t : p.nodes) p.node_has_pre.push_back(p.div.event_at(t) >= 0);
        for (int k = 0; k < 3; ++k) {
            Dividends dk;
            if (d->discrete_dividends.count &&
                !dk.compile(d->discrete_dividends, p.bump_spot[k], p.rc, p.qc))
                return fail("dividends at a bumped spot");
            for (double t : p.nodes) {
                p.node_post[k].push_back(dk.after_time(t));
                const long e = dk.event_at(t);
                p.node_pre[k].push_back(e >= 0 ? dk.before_event(static_cast<size_t>(e)) : Coord{});
            }
            // dividend checkpoints through the horizon (local_vol.rs:326-345)
            for (const auto& e : dk.ev) {
                if (!(e.t <= p.nodes.back())) continue;
                size_t node = 0;
                while (node < p.nodes.size() && bits_of(p.nodes[node]) != bits_of(e.t)) ++node;
                p.checks[k].push_back({node, dk.after_time(e.t)});
            }
        }
        for (double t : p.obs_t) {
            uint32_t idx = 0;
            for (; idx < p.nodes.size(); ++idx)
                if (bits_of(p.nodes[idx]) == bits_of(t)) break;
            p.obs_node.push_back(idx);
        }
        p.total_variance = p.nodes.back() * p.grid.cap;  // maximum_total_variance
        p.vol_bump = 0.0;
    }
    const bool lv = p.model == MCG_MODEL_LOCAL_VOLATILITY;
    const uint32_t steps = lv ? static_cast<uint32_t>(p.nodes.size() - 1)
                              : static_cast<uint32_t>(p.obs_t.size());
    if (lv && (p.bridge_flag)) {
        if (!p.bridge.compile(p.nodes)) return fail("bridge");
        p.use_bridge = true;
    }
    p.dimension = steps;
    if (p.engine == MCG_ENGINE_RQMC) {
        if (steps > d->sobol_dimension_count) return fail("sobol dimension");
        p.dirs.assign(d->sobol_directions,
                      d->sobol_directions + static_cast<size_t>(steps) * 32u);
        for (uint32_t s = 0; s < p.scrambles; ++s)
            for (uint32_t dim = 0; dim < steps; ++dim)
                p.scr.push_back(compile_scramble(p.seed, d->scramble_begin + s, dim));
    }
    return true;
}

// ------------------------------------------------------ BS observations

struct Obs {
    double post_spot, f, w;
    double pre_spot;   // the ex-date spot before the dividend (has_pre)
    bool has_pre;
    Coord post, pre;   // coordinates at the observation's spot runtime
};

// path_observation, black_scholes.rs:335-354: S = a S0 + b f after (and
// before) an ex-date's dividend, at the runtime's spot.
void bs_observe(const Plan& p, size_t i, double f, double w, double spot, Obs& o) {
    o.f = f;
    o.w = w;
    o.post = p.obs_post[i].at_spot(p.spot, spot);
    o.post_spot = o.post.a * spot + o.post.b * f;
    o.has_pre = p.obs_has_pre[i] != 0;
    o.pre = o.has_pre ? p.obs_pre[i].at_spot(p.spot, spot) : o.post;
    o.pre_spot = o.has_pre ? o.pre.a * spot + o.pre.b * f : o.post_spot;
}

// path_observations_from_normals, crates/pricing/src/engine/processes/black_scholes.rs:297-331.
void bs_observations(const Plan& p, const double* z, double spot, double vol, Obs* out) {
    const double spot_scale = spot / p.spot;
    const size_t n = p.obs_t.size();
    if (n == 1) {
        const double t = p.obs_t[0];
        const double tv = vol * vol * t;
        const double sd = std::sqrt(tv);
        const double w = std::sqrt(t) * z[0];
        const double lr = -0.5 * tv + sd * z[0];
        const double f = p.obs_fwd[0] * spot_scale * std::exp(lr);
        bs_observe(p, 0, f, w, spot, out[0]);
        return;
    }
    double prev = 0.0, w = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double t = p.obs_t[i];
        const double step = std::max(t - prev, 0.0);
        w += std::sqrt(step) * z[i];
        prev = t;
        const double tv = vol * vol * t;
        const double f = p.obs_fwd[i] * spot_scale * std::exp(-0.5 * tv + vol * w);
        bs_observe(p, i, f, w, spot, out[i]);
    }
}

// ------------------------------------------------------ payoff programs

// Hand-lowered payoff graphs of crates/pricing/src/engine/payoff/compile.rs:35-474
// with the forward/reverse opcode semantics of crates/pricing/src/engine/payoff/tape.rs:594-781,953-1088.
// `spots` are the observation spots; `adj` (may be null) receives dPayoff/dSpot.
// A discrete barrier monitored on an ex-dividend date (has_pre[i]) also sees the
// spot before the dividend: its distance is the maximum (smoothed: the compact-C2
// smooth maximum) of the pre- and post-dividend distances
// (crates/pricing/src/engine/payoff/compile.rs:315-346); pre_adj receives
// dPayoff/dPreSpot.
double payoff_eval(const Product& pr, const double* spots, size_t n, double h, double* adj,
                   const double* pre_spots = nullptr, const char* has_pre = nullptr, double* pre_adj = nullptr) {
    const mcg_product_desc& d = pr.d;
    const bool call = d.side == MCG_CALL;
    if (adj)
        for (size_t i = 0; i < n; ++i) adj[i] = 0.0;
    if (pre_adj)
        for (size_t i = 0; i < n; ++i) pre_adj[i] = 0.0;
    switch (d.kind) {
    case MCG_PRODUCT_EUROPEAN: {
        const double s = spots[n - 1];
        const double in = call ? s - d.strike : d.strike - s;
        const double pos = in >= 0.0 ? in : 0.0;
        if (adj) adj[n - 1] = (in >= 0.0 ? d.notional : 0.0) * (call ? 1.0 : -1.0);
        return pos * d.notional;
    }
    case MCG_PRODUCT_DIGITAL: {
        const double s = spots[n - 1];
        const double dist = call ? s - d.strike : d.strike - s;
        double ind, ind_first = 0.0;
        if (h > 0.0) {
            const Deriv dd = indicator(h, dist);
            ind = dd.value;
            ind_first = dd.first;
        } else {
            ind = dist >= 0.0 ? 1.0 : 0.0;
        }
        const bool asset = d.digital_payout == MCG_DIGITAL_ASSET;
        const double base = asset ? s * d.payout : d.payout;
        if (adj) {
            double a = 0.0;
            if (asset) a += ind * d.payout;
            if (h > 0.0) a += (call ? 1.0 : -1.0) * (base * ind_first);
            adj[n - 1] = a;
        }
        return ind * base;
    }
    case MCG_PRODUCT_ASIAN: {
        // Known fixings first (compile.rs:162-176), then the simulated observations.
        double sum = d.has_initial_state ? d.initial_state : 0.0;
        for (size_t i = 0; i < n; ++i) sum = sum + spots[i] * pr.weights[i];
        const double in = call ? sum - d.strike : d.strike - sum;
        const double pos = in >= 0.0 ? in : 0.0;
        if (adj) {
            const double g = (in >= 0.0 ? d.notional : 0.0) * (call ? 1.0 : -1.0);
            for (size_t i = 0; i < n; ++i) adj[i] = g * pr.weights[i];
        }
        return pos * d.notional;
    }
    case MCG_PRODUCT_LOOKBACK: {
        // The historical extremum (or valuation-date fixing) is a literal, the
        // first simulated monitoring date otherwise (compile.rs:426-452).
        bool seeded = d.has_initial_state != 0;
        double ext = seeded ? d.initial_state : 0.0;
        size_t arg = n;  // n: the literal holds the extremum
        for (size_t i = 0; i < n; ++i) {
            if (!pr.monitored(i)) continue;
            if (!seeded) {
                ext = spots[i];
                arg = i;
                seeded = true;
            } else if (call) {
                if (!(ext >= spots[i])) { ext = spots[i]; arg = i; }
            } else {
                if (!(ext <= spots[i])) { ext = spots[i]; arg = i; }
            }
        }
        const double in = call ? ext - d.strike : d.strike - ext;
        const double pos = in >= 0.0 ? in : 0.0;
        if (adj && arg < n) adj[arg] = (in >= 0.0 ? d.notional : 0.0) * (call ? 1.0 : -1.0);
        return pos * d.notional;
    }
    case MCG_PRODUCT_DISCRETE_BARRIER: {
        const double s = spots[n - 1];
        const double in = call ? s - d.strike : d.strike - s;
        const double pos = in >= 0.0 ? in : 0.0;
        const double vanilla = pos * d.notional;
        const bool up = d.barrier_direction == MCG_BARRIER_UP;
        double hit = d.has_initial_state ? d.initial_state : 0.0;  // historical hit, compile.rs:293-297
        std::vector<double> hist, weights, firsts, pre_share, post_share;
        if (adj && h > 0.0) {
            hist.resize(n);
            weights.resize(n);
            firsts.resize(n);
            pre_share.assign(n, 0.0);
            post_share.assign(n, 1.0);
        }
        for (size_t i = 0; i < n; ++i) {
            if (!pr.monitored(i)) {
                if (adj && h > 0.0) {
                    hist[i] = hit;
                    weights[i] = 0.0;
                    firsts[i] = 0.0;
                }
                continue;
            }
            double dist = up ? spots[i] - d.barrier : d.barrier - spots[i];
            if (has_pre && has_pre[i]) {
                const double pre = up ? pre_spots[i] - d.barrier : d.barrier - pre_spots[i];
                if (h > 0.0) {
                    const BinaryDeriv m = smooth_maximum(h, pre, dist);
                    if (adj) {
                        pre_share[i] = m.left_first;
                        post_share[i] = m.right_first;
                    }
                    dist = m.value;
                } else {
                    dist = pre >= dist ? pre : dist;
                }
            }
            double wgt;
            if (h > 0.0) {
                const Deriv dd = indicator(h, dist);
                wgt = dd.value;
                if (adj) {
                    hist[i] = hit;
                    weights[i] = wgt;
                    firsts[i] = dd.first;
                }
            } else {
                wgt = dist >= 0.0 ? 1.0 : 0.0;
            }
            hit = hit + (1.0 - hit) * wgt;
        }
        const bool ko = d.barrier_style == MCG_KNOCK_OUT;
        const double active = ko ? 1.0 - hit : hit;
        double value = vanilla * active;
        if (d.has_rebate) value = value + (1.0 - active) * d.rebate;
        if (adj) {
            // reverse sweep: d value / d active and / d vanilla
            double a_active = vanilla;
            if (d.has_rebate) a_active = a_active + (-d.rebate);
            const double a_vanilla = active;
            if (h > 0.0) {
                double a_hit = ko ? -a_active : a_active;
                for (size_t k = n; k-- > 0;) {
                    const double a_w = a_hit * (1.0 - hist[k]);
                    a_hit = a_hit * (1.0 - weights[k]);
                    const double a_dist = a_w * firsts[k];
                    adj[k] += (up ? 1.0 : -1.0) * (a_dist * post_share[k]);
                    if (pre_adj && pre_share[k] != 0.0) pre_adj[k] += (up ? 1.0 : -1.0) * (a_dist * pre_share[k]);
                }
            }
            adj[n - 1] += (in >= 0.0 ? a_vanilla * d.notional : 0.0) * (call ? 1.0 : -1.0);
        }
        return value;
    }
    default:
        return 0.0;
    }
}

// ------------------------------------------------- continuous barrier

struct BarrierEval {
    double survival;
    double diag[8];  // components 10..17
    // reverse data
    bool exact_active;  // exact, not touched: interval adjoints flow
    std::vector<ExactInterval> ex;
    std::vector<SmoothInterval> sm;
    std::vector<double> hit_safety, hit_dstate;  // smoothed hit factors, index 0 = initial
    double log_survival_total;
};

void diag_from_exact(const std::vector<ExactInterval>& iv, bool endpoint_touched, double surv,
                     double* diag) {
    uint32_t fin = 0, tch = 0, zv = 0, un = 0, ce = 0;
    for (const auto& i : iv) {
        if (i.status == kFinite) ++fin;
        else if (i.status == kTouched) ++tch;
        else if (i.status == kZeroVariance) ++zv;
        else if (i.status == kUnderflow) ++un;
        else ++ce;
    }
    diag[0] = endpoint_touched ? 1.0 : 0.0;
    diag[1] = 0.0;
    diag[2] = endpoint_touched ? 0.0 : 1.0 - surv;
    diag[3] = static_cast<double>(iv.size());
    diag[4] = fin;
    diag[5] = zv;
    diag[6] = un;
    diag[7] = ce;
}

// Continuous barrier survival over a sequence of states, exact or smoothed:
// BS crates/pricing/src/engine/processes/black_scholes.rs:94-293 and
// LV crates/pricing/src/engine/processes/local_vol_valuation.rs:251-434.
// states[0] is the initial spot/state; variances per state.
bool barrier_bridge(const Plan& p, const mcg_product_desc& d, const double* states,
                    const double* variances, const double* times, size_t count, BarrierEval& be,
                    Failure& f) {
    const bool up = d.barrier_direction == MCG_BARRIER_UP;
    const double B = d.barrier;
    const double h = p.smoothing;
    be.ex.clear();
    be.sm.clear();
    be.hit_safety.clear();
    be.hit_dstate.clear();
    if (h > 0.0) {
        SmoothEndpoint e0;
        if (!smooth_endpoint(up, states[0], B, 1.0, h, e0, f)) return false;
        be.hit_safety.push_back(e0.safety_weight);
        be.hit_dstate.push_back(1.0 * e0.hit_d_state + 0.0 * e0.eld_d_state);
        double log_bridge = 0.0;
        uint32_t fin = 0, zv = 0, un = 0, ce = 0;
        for (size_t k = 1; k < count; ++k) {
            const double dt = times[k] - times[k - 1];
            if (!(dt > 0.0)) continue;
            SmoothInterval si;
            if (!smooth_interval(up, states[k - 1], states[k], B, B, 1.0, 1.0, variances[k - 1],
                                 variances[k], dt, h, si, f))
                return false;
            be.hit_safety.push_back(si.right.safety_weight);
            be.hit_dstate.push_back(1.0 * si.right.hit_d_state + 0.0 * si.right.eld_d_state);
            be.sm.push_back(si);
        }
        for (const auto& si : be.sm) {
            log_bridge += si.log_survival;
            if (si.status == kFinite) ++fin;
            else if (si.status == kZeroVariance) ++zv;
            else if (si.status == kUnderflow) ++un;
            else if (si.status == kCertain) ++ce;
        }
        double log_hit = 0.0;
        for (double s : be.hit_safety) log_hit = log_hit + std::log(s);
        be.log_survival_total = log_bridge + log_hit;
        be.survival = std::exp(be.log_survival_total);
        double prod = 1.0;
        for (double s : be.hit_safety) prod = prod * s;
        be.diag[0] = 1.0 - prod;
        be.diag[1] = 1.0 - 1.0;
        be.diag[2] = 1.0 - std::exp(log_bridge);
        be.diag[3] = static_cast<double>(be.sm.size());
        be.diag[4] = fin;
        be.diag[5] = zv;
        be.diag[6] = un;
        be.diag[7] = ce;
        be.exact_active = false;
        return true;
    }
    const bool initial_touched = up ? states[0] >= B : states[0] <= B;
    double log_survival = 0.0;
    if (!initial_touched) {
        for (size_t k = 1; k < count; ++k) {
            const double dt = times[k] - times[k - 1];
            if (!(dt > 0.0)) continue;
            ExactInterval iv;
            if (!exact_interval(up, states[k - 1], states[k], B, B, variances[k - 1], variances[k],
                                dt, iv, f))
                return false;
            be.ex.push_back(iv);
        }
    }
    uint32_t touched = 0;
    for (const auto& iv : be.ex) {
        log_survival += iv.log_survival;
        if (iv.status == kTouched) ++touched;
    }
    const bool endpoint_touched = initial_touched || touched != 0;
    const double path_surv = std::exp(log_survival);
    be.survival = endpoint_touched ? 0.0 : path_surv;
    be.exact_active = !endpoint_touched;
    diag_from_exact(be.ex, endpoint_touched, path_surv, be.diag);
    return true;
}

struct BarrierTerms {
    double value, terminal_derivative, survival_derivative;
};

// continuous_barrier_payoff_terms, crates/pricing/src/engine/payoff/barrier.rs:307-355.
BarrierTerms barrier_terms(const mcg_product_desc& d, double terminal, double survival) {
    const bool call = d.side == MCG_CALL;
    const double in = call ? terminal - d.strike : d.strike - terminal;
    const double vanilla = std::max(in, 0.0) * d.notional;
    const double vd = in >= 0.0 ? (call ? 1.0 : -1.0) * d.notional : 0.0;
    const double rebate = d.has_rebate ? d.rebate : 0.0;
    if (d.barrier_style == MCG_KNOCK_OUT)
        return {rebate + survival * (vanilla - rebate), survival * vd, vanilla - rebate};
    return {vanilla + survival * (rebate - vanilla), (1.0 - survival) * vd, rebate - vanilla};
}

// ------------------------------------------------------- BS pathwise

struct Aad {
    double price, delta, vega;
    double diag[8];
    bool has_diag;
};

// pathwise_aad, black_scholes.rs:476-563,648-793.
bool bs_pathwise(const Plan& p, const Product& pr, const double* z, double spot, double vol,
                 Aad& out, Failure& f, std::vector<Obs>& obs, std::vector<double>& tmp) {
    const size_t n = p.obs_t.size();
    out.has_diag = false;
    const mcg_product_desc& d = pr.d;
    if (d.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
        obs.resize(n);
        bs_observations(p, z, spot, vol, obs.data());
        std::vector<double> st(n + 1), var(n + 1, vol * vol), tt(n + 1);
        st[0] = spot;
        tt[0] = 0.0;
        for (size_t i = 0; i < n; ++i) {
            st[i + 1] = obs[i].f;
            tt[i + 1] = p.obs_t[i];
        }
        BarrierEval be;
        if (!barrier_bridge(p, d, st.data(), var.data(), tt.data(), n + 1, be, f)) return false;
        const BarrierTerms terms = barrier_terms(d, obs[n - 1].post_spot, be.survival);
        std::vector<double> sa(n + 1, 0.0);  // index 0 = initial state
        sa[n] += terms.terminal_derivative * 1.0;
        double var_adj = 0.0;
        if (p.smoothing > 0.0) {
            const double lsa = terms.survival_derivative * be.survival;
            for (size_t k = 0; k < be.sm.size(); ++k) {
                const auto& si = be.sm[k];
                const double ea_l = lsa * si.d_left_distance;
                const double ea_r = lsa * si.d_right_distance;
                sa[k] += 0.0 * si.left.hit_d_state + ea_l * si.left.eld_d_state;
                sa[k + 1] += 0.0 * si.right.hit_d_state + ea_r * si.right.eld_d_state;
                var_adj += (lsa * si.d_left_var) + (lsa * si.d_right_var);
            }
            for (size_t k = 0; k < be.hit_safety.size(); ++k) {
                const double der = be.hit_safety[k] == 0.0
                                       ? 0.0
                                       : -lsa * be.hit_dstate[k] / be.hit_safety[k];
                sa[k] += der;
            }
        } else if (be.exact_active) {
            const double lsa = terms.survival_derivative * be.survival;
            for (size_t k = 0; k < be.ex.size(); ++k) {
                sa[k] += lsa * be.ex[k].d_left_state;
                sa[k + 1] += lsa * be.ex[k].d_right_state;
                var_adj += (lsa * be.ex[k].d_left_var) + (lsa * be.ex[k].d_right_var);
            }
        }
        double delta = sa[0];
        double vega = 2.0 * vol * var_adj;
        for (size_t i = 0; i < n; ++i) {
            delta += sa[i + 1] * obs[i].f / spot;
            vega += sa[i + 1] * obs[i].f * (-vol * p.obs_t[i] + obs[i].w);
        }
        out.price = p.discount * terms.value;
        out.delta = p.discount * delta;
        out.vega = p.discount * vega;
        std::memcpy(out.diag, be.diag, sizeof(out.diag));
        out.has_diag = true;
        return true;
    }
    if (n == 1) {
        // pathwise_aad_single_terminal, black_scholes.rs:757-793
        const double t = p.obs_t[0];
        const double tv = vol * vol * t;
        const double sd = std::sqrt(tv);
        const double lr = -0.5 * tv + sd * z[0];
        const double bf = p.obs_fwd[0] * (spot / p.spot);
        const double f = bf * std::exp(lr);
        const Coord c = p.obs_post[0].at_spot(p.spot, spot);
        const double terminal = c.a * spot + c.b * f;
        double a;
        const double value = payoff_eval(pr, &terminal, 1, p.smoothing, &a);
        out.price = p.discount * value;
        out.delta = p.discount * a * c.spot_scale * f / spot;
        const double tvega = c.b * f * (-vol * t + std::sqrt(t) * z[0]);
        out.vega = p.discount * a * tvega;
        return true;
    }
    obs.resize(n);
    bs_observations(p, z, spot, vol, obs.data());
    tmp.resize(4 * n);
    double* spots = tmp.data();
    double* adj = tmp.data() + n;
    double* pre_spots = tmp.data() + 2 * n;
    double* pre_adj = tmp.data() + 3 * n;
    for (size_t i = 0; i < n; ++i) {
        spots[i] = obs[i].post_spot;
        pre_spots[i] = obs[i].pre_spot;
    }
    const double value = payoff_eval(pr, spots, n, p.smoothing, adj, pre_spots, p.obs_has_pre.data(), pre_adj);
    // terminal adjoints, then the pre-dividend ones (black_scholes.rs:525-562)
    double delta = 0.0, vega = 0.0;
    for (size_t k = n; k-- > 0;) {
        if (adj[k] == 0.0) continue;
        delta += adj[k] * obs[k].post.spot_scale * obs[k].f / spot;
        vega += adj[k] * obs[k].post.b * obs[k].f * (-vol * p.obs_t[k] + obs[k].w);
    }
    for (size_t k = n; k-- > 0;) {
        if (pre_adj[k] == 0.0 || !obs[k].has_pre) continue;
        delta += pre_adj[k] * obs[k].pre.spot_scale * obs[k].f / spot;
        vega += pre_adj[k] * obs[k].pre.b * obs[k].f * (-vol * p.obs_t[k] + obs[k].w);
    }
    out.price = p.discount * value;
    out.delta = p.discount * delta;
    out.vega = p.discount * vega;
    return true;
}

// pathwise_values, black_scholes.rs:417-472.
bool bs_unit_product(const Plan& p, const Product& pr, const double* z, double* values,
                     Failure& f, std::vector<Obs>& obs, std::vector<double>& tmp) {
    for (int c = 0; c < kComponents; ++c) values[c] = 0.0;
    if (p.risk_enabled()) {
        Aad base, dn, up, a, b;
        if (!bs_pathwise(p, pr, z, p.spot, p.vol, base, f, obs, tmp)) return false;
        double gamma = 0.0;
        if (p.req_gamma) {
            const double bump = p.gamma_bump;
            if (!bs_pathwise(p, pr, z, p.spot - bump, p.vol, a, f, obs, tmp)) return false;
            if (!bs_pathwise(p, pr, z, p.spot + bump, p.vol, b, f, obs, tmp)) return false;
            gamma = (b.delta - a.delta) / (2.0 * bump);
        }
        const double sb = p.spot_bump;
        if (!bs_pathwise(p, pr, z, p.spot - sb, p.vol, dn, f, obs, tmp)) return false;
        if (!bs_pathwise(p, pr, z, p.spot + sb, p.vol, up, f, obs, tmp)) return false;
        const double bump_delta = (up.price - dn.price) / (2.0 * sb);
        const double bump_gamma = (up.price - 2.0 * base.price + dn.price) / (sb * sb);
        double bump_vega = 0.0;
        if (p.vol_bump != 0.0) {
            const double vb = p.vol_bump;
            if (!bs_pathwise(p, pr, z, p.spot, p.vol - vb, a, f, obs, tmp)) return false;
            if (!bs_pathwise(p, pr, z, p.spot, p.vol + vb, b, f, obs, tmp)) return false;
            bump_vega = (b.price - a.price) / (2.0 * vb);
        }
        values[MCG_PRICE] = base.price;
        values[MCG_DELTA] = base.delta;
        values[MCG_VEGA] = base.vega;
        values[MCG_GAMMA] = gamma;
        values[MCG_BUMP_DELTA] = bump_delta;
        values[MCG_DELTA_DIFFERENCE] = bump_delta - base.delta;
        values[MCG_BUMP_VEGA] = bump_vega;
        values[MCG_VEGA_DIFFERENCE] = bump_vega - base.vega;
        values[MCG_BUMP_GAMMA] = bump_gamma;
        values[MCG_GAMMA_DIFFERENCE] = bump_gamma - gamma;
        if (base.has_diag)
            for (int k = 0; k < 8; ++k) values[10 + k] = base.diag[k];
        return true;
    }
    const size_t n = p.obs_t.size();
    obs.resize(n);
    bs_observations(p, z, p.spot, p.vol, obs.data());
    if (pr.d.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
        Aad base;
        if (!bs_pathwise(p, pr, z, p.spot, p.vol, base, f, obs, tmp)) return false;
        values[MCG_PRICE] = base.price;
        for (int k = 0; k < 8; ++k) values[10 + k] = base.diag[k];
        return true;
    }
    tmp.resize(2 * n);
    for (size_t i = 0; i < n; ++i) {
        tmp[i] = obs[i].post_spot;
        tmp[n + i] = obs[i].pre_spot;
    }
    values[MCG_PRICE] = p.discount * payoff_eval(pr, tmp.data(), n, p.smoothing, nullptr, tmp.data() + n,
                                                 p.obs_has_pre.data());
    return true;
}


// ---------------------------------------------------------- local vol

struct LvPath {
    std::vector<double> state;          // per node
    std::vector<double> var;            // per step: local variance used
    std::vector<Interpolation> interp;  // per step
    std::vector<double> expo;           // per step: exponential factor
    std::vector<double> shock;          // per step
};

// LocalVolLogEulerPlan::evolve_path_inner, crates/pricing/src/engine/processes/local_vol.rs:459-559.
bool lv_evolve(const Plan& p, int which, const double* shocks, LvPath& path, Failure& f) {
    const size_t steps = p.nodes.size() - 1;
    const std::vector<double>& F = p.fwd[which];
    path.state.resize(steps + 1);
    path.var.resize(steps);
    path.interp.resize(steps);
    path.expo.resize(steps);
    path.shock.assign(shocks, shocks + steps);
    double state = p.bump_spot[which];
    path.state[0] = state;
    for (size_t s = 0; s < steps; ++s) {
        const double time = p.nodes[s];
        const double dt = p.nodes[s + 1] - time;
        const double x = std::log(state / F[s]);
        Interpolation in;
        if (!p.grid.interpolate(time, x, in)) {
            f = {MCG_ERR_INVALID_SURFACE_QUERY, static_cast<uint32_t>(s), x};
            return false;
        }
        const double lvol = std::sqrt(in.value);
        const double ratio = F[s + 1] / F[s];
        const double e = ratio * std::exp(-0.5 * in.value * dt + lvol * std::sqrt(dt) * shocks[s]);
        state *= e;
        if (!std::isfinite(state) || state <= 0.0) {
            f = {MCG_ERR_NON_FINITE_STATE, static_cast<uint32_t>(s + 1), state};
            return false;
        }
        // post-dividend spot of an ex-date node (validate_post_event_f_state,
        // dividend.rs:557-583, at local_vol.rs:520-545)
        for (const auto& ck : p.checks[which])
            if (ck.first == s + 1) {
                const double post = ck.second.spot_of(p.bump_spot[which], state);
                if (!std::isfinite(post) || post <= 0.0) {
                    f = {MCG_ERR_MARKET, static_cast<uint32_t>(s + 1), post};
                    return false;
                }
            }
        path.state[s + 1] = state;
        path.var[s] = in.value;
        path.interp[s] = in;
        path.expo[s] = e;
    }
    return true;
}

// Node variances for the continuous-barrier bridge, local_vol_valuation.rs:262-279.
bool lv_node_variances(const Plan& p, int which, const LvPath& path, std::vector<double>& nv,
                       Failure& f) {
    const size_t count = p.nodes.size();
    nv.resize(count);
    for (size_t k = 0; k < count; ++k) {
        Interpolation in;
        const double x = std::log(path.state[k] / p.fwd[which][k]);
        if (!p.grid.interpolate(p.nodes[k], x, in)) {
            f = {MCG_ERR_INVALID_SURFACE_QUERY, static_cast<uint32_t>(k), x};
            return false;
        }
        nv[k] = in.value;
    }
    return true;
}

// Discounted payoff of one LV path at one spot runtime,
// local_vol_discounted_payoff_at_spot_inner, local_vol_valuation.rs:161-206.
bool lv_payoff(const Plan& p, const Product& pr, int which, const LvPath& path, double& value,
               BarrierEval* be_out, BarrierTerms* terms_out, std::vector<double>& nv,
               Failure& f) {
    const size_t n = p.obs_t.size();
    const double spot = p.bump_spot[which];
    if (pr.d.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) {
        if (!lv_node_variances(p, which, path, nv, f)) return false;
        BarrierEval be;
        if (!barrier_bridge(p, pr.d, path.state.data(), nv.data(), p.nodes.data(),
                            p.nodes.size(), be, f))
            return false;
        const double terminal = 0.0 * spot + 1.0 * path.state[p.obs_node[n - 1]];
        const BarrierTerms t = barrier_terms(pr.d, terminal, be.survival);
        value = p.discount * t.value;
        if (be_out) *be_out = std::move(be);
        if (terms_out) *terms_out = t;
        return true;
    }
    // local_vol_state_observations, local_vol_valuation.rs:221-247
    std::vector<double> spots(2 * n);
    std::vector<char> has_pre(n);
    for (size_t i = 0; i < n; ++i) {
        const size_t node = p.obs_node[i];
        spots[i] = p.node_post[which][node].spot_of(spot, path.state[node]);
        has_pre[i] = p.node_has_pre[node];
        spots[n + i] = has_pre[i] ? p.node_pre[which][node].spot_of(spot, path.state[node]) : spots[i];
    }
    value = p.discount * payoff_eval(pr, spots.data(), n, p.smoothing, nullptr, spots.data() + n, has_pre.data());
    return true;
}

// reverse_path_with_variance_seeds and LocalVolPath::reverse_state_adjoints,
// local_vol/direct_adjoints.rs:97-159 and local_vol.rs:723-803, for the spot
// runtime `which`.  Returns the combined grid-value adjoints, the adjoint of the
// initial state and x_sum = sum over nodes of dPayoff/dx_i, the sensitivity to
// the forward normalisers (every F_i is proportional to the spot).
bool lv_reverse(const Plan& p, int which, const LvPath& path, std::vector<double> seeds,
                const std::vector<double>& var_seeds, std::vector<double>& grid_adj,
                double& initial_adjoint, double& x_sum, Failure& f) {
    const size_t count = p.nodes.size();
    const size_t steps = count - 1;
    grid_adj.assign(p.grid.v.size(), 0.0);
    x_sum = 0.0;
    for (size_t i = 0; i < count; ++i) {
        Interpolation in;
        if (!p.grid.interpolate(p.nodes[i], std::log(path.state[i] / p.fwd[which][i]), in)) {
            f = {MCG_ERR_INVALID_SURFACE_QUERY, static_cast<uint32_t>(i), 0.0};
            return false;
        }
        const double seed = var_seeds[i];
        const double dvdx = p.grid.x_derivative(in);
        seeds[i] += seed * dvdx / path.state[i];
        x_sum += seed * dvdx;
        p.grid.transpose_accumulate(in, seed, grid_adj.data());
    }
    std::vector<double> trans(p.grid.v.size(), 0.0);
    for (size_t s = steps; s-- > 0;) {
        const double nsa = seeds[s + 1];
        const double ns = path.state[s + 1];
        const double lea = nsa * ns;
        const double lvol = std::sqrt(path.var[s]);
        const double dt = p.nodes[s + 1] - p.nodes[s];
        const double sqdt = std::sqrt(dt);
        seeds[s] += nsa * path.expo[s];
        const double lva = lea * (-0.5 * dt + path.shock[s] * sqdt / (2.0 * lvol));
        const double dvdx = p.grid.x_derivative(path.interp[s]);
        seeds[s] += lva * (dvdx / path.state[s]);
        x_sum += lva * dvdx;
        if (!std::isfinite(seeds[s]) || !std::isfinite(lva)) {
            f = {MCG_ERR_NON_FINITE_STATE, static_cast<uint32_t>(s), seeds[s]};
            return false;
        }
        p.grid.transpose_accumulate(path.interp[s], lva, trans.data());
    }
    for (size_t k = 0; k < grid_adj.size(); ++k) grid_adj[k] += trans[k];
    initial_adjoint = seeds[0];
    return true;
}

// Payoff seeds of one LV path (pathwise_local_vol.rs:206-303) and the reverse
// sweep: Vega = sum of 2 sqrt(v) x node adjoint (:310-321), node values, and
// the adjoint spot Delta dP/dS0 = lambda_0 - x_sum / S0 (holding the dynamics
// in forward-normalised log-moneyness, as the bumped runtimes do).
bool lv_adjoint(const Plan& p, const Product& pr, int which, const double* shocks, double& price,
                double& vega, double& adjoint_delta, double* node_values, double* diag, Failure& f) {
    LvPath path;
    if (!lv_evolve(p, which, shocks, path, f)) return false;
    BarrierEval be;
    BarrierTerms terms{};
    std::vector<double> nv;
    const bool cb = pr.d.kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
    if (!lv_payoff(p, pr, which, path, price, cb ? &be : nullptr, cb ? &terms : nullptr, nv, f))
        return false;
    if (cb && diag)
        for (int k = 0; k < 8; ++k) diag[k] = be.diag[k];
    const size_t count = p.nodes.size();
    const size_t n = p.obs_t.size();
    std::vector<double> seeds(count, 0.0), vseeds(count, 0.0);
    if (cb) {
        const uint32_t tn = p.obs_node[n - 1];
        seeds[tn] += p.discount * terms.terminal_derivative * 1.0;
        if (p.smoothing > 0.0) {
            const double lsa = (p.discount * terms.survival_derivative) * be.survival;
            for (size_t k = 0; k < be.sm.size(); ++k) {
                const auto& si = be.sm[k];
                seeds[k] += 0.0 * si.left.hit_d_state + (lsa * si.d_left_distance) * si.left.eld_d_state;
                seeds[k + 1] += 0.0 * si.right.hit_d_state + (lsa * si.d_right_distance) * si.right.eld_d_state;
                vseeds[k] += lsa * si.d_left_var;
                vseeds[k + 1] += lsa * si.d_right_var;
            }
            for (size_t k = 0; k < be.hit_safety.size(); ++k) {
                const double der = be.hit_safety[k] == 0.0
                                       ? 0.0
                                       : -lsa * be.hit_dstate[k] / be.hit_safety[k];
                seeds[k] += der;
            }
        } else if (be.exact_active) {
            const double lsa = p.discount * terms.survival_derivative * be.survival;
            for (size_t k = 0; k < be.ex.size(); ++k) {
                seeds[k] += lsa * be.ex[k].d_left_state;
                seeds[k + 1] += lsa * be.ex[k].d_right_state;
                vseeds[k] += lsa * be.ex[k].d_left_var;
                vseeds[k + 1] += lsa * be.ex[k].d_right_var;
            }
        }
    } else {
        std::vector<double> spots(n), adj(n);
        for (size_t i = 0; i < n; ++i) spots[i] = path.state[p.obs_node[i]];
        payoff_eval(pr, spots.data(), n, p.smoothing, adj.data());
        for (size_t k = n; k-- > 0;)
            if (adj[k] != 0.0) seeds[p.obs_node[k]] += p.discount * adj[k] * 1.0;
    }
    std::vector<double> grid_adj;
    double lambda0, x_sum;
    if (!lv_reverse(p, which, path, seeds, vseeds, grid_adj, lambda0, x_sum, f)) return false;
    NeumaierSum v;
    for (size_t k = 0; k < grid_adj.size(); ++k) {
        const double node = grid_adj[k] * 2.0 * std::sqrt(p.grid.v[k]);
        v.add(node);
        if (node_values) node_values[k] = node;
    }
    vega = v.total();
    adjoint_delta = lambda0 - x_sum / p.bump_spot[which];
    return true;
}

// local_vol_pathwise_values_and_buckets_inner,
// crates/pricing/src/engine/risk/pathwise_local_vol.rs:127-361.  Values 18 and
// 19 (beyond the reference's 18) hold the adjoint Delta and the bumped-adjoint
// Gamma when Vega and Delta (and Gamma) are requested.
bool lv_unit_product(const Plan& p, const Product& pr, const double* shocks, double* values,
                     double* node_values, Failure& f) {
    for (int c = 0; c < kComponents + 2; ++c) values[c] = 0.0;
    double price;
    if (p.req_vega || p.req_nodes) {
        double vega, adelta, diag[8];
        if (!lv_adjoint(p, pr, 0, shocks, price, vega, adelta, node_values, diag, f)) return false;
        values[MCG_VEGA] = vega;
        if (pr.d.kind == MCG_PRODUCT_CONTINUOUS_BARRIER)
            for (int k = 0; k < 8; ++k) values[10 + k] = diag[k];
        if (p.req_delta) values[kComponents] = adelta;
        if (p.req_delta && p.req_gamma) {
            double pd, pu, vd, vu, dd, du;
            if (!lv_adjoint(p, pr, 1, shocks, pd, vd, dd, nullptr, nullptr, f)) return false;
            if (!lv_adjoint(p, pr, 2, shocks, pu, vu, du, nullptr, nullptr, f)) return false;
            values[kComponents + 1] = (du - dd) / (2.0 * p.spot_bump);
        }
    } else {
        LvPath path;
        if (!lv_evolve(p, 0, shocks, path, f)) return false;
        BarrierEval be;
        BarrierTerms terms{};
        std::vector<double> nv;
        const bool cb = pr.d.kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
        if (!lv_payoff(p, pr, 0, path, price, cb ? &be : nullptr, cb ? &terms : nullptr, nv, f))
            return false;
        if (cb)
            for (int k = 0; k < 8; ++k) values[10 + k] = be.diag[k];
    }
    values[MCG_PRICE] = price;
    if (p.req_delta || p.req_gamma) {
        double down, up;
        LvPath bumped;
        std::vector<double> nv;
        if (!lv_evolve(p, 1, shocks, bumped, f)) return false;
        if (!lv_payoff(p, pr, 1, bumped, down, nullptr, nullptr, nv, f)) return false;
        if (!lv_evolve(p, 2, shocks, bumped, f)) return false;
        if (!lv_payoff(p, pr, 2, bumped, up, nullptr, nullptr, nv, f)) return false;
        const double h = p.spot_bump;
        const double delta = (up - down) / (2.0 * h);
        values[MCG_DELTA] = delta;
        values[MCG_BUMP_DELTA] = delta;
        if (p.req_gamma) {
            const double gamma = (up - 2.0 * price + down) / (h * h);
            values[MCG_GAMMA] = gamma;
            values[MCG_BUMP_GAMMA] = gamma;
        }
    }
    return true;
}

// -------------------------------------------------------------- shocks

// Normals of one unit: pseudo (Philox, dimension = step or bridge rank) or
// RQMC (scrambled Sobol), crates/pricing/src/engine/sampling/path_normals.rs:11-83
// and crates/pricing/src/engine/processes/local_vol.rs:621-668.
void unit_shocks(const Plan& p, uint32_t scramble, uint64_t unit, double* out,
                 std::vector<double>& normals, std::vector<double>& scratch) {
    const uint32_t dims = p.dimension;
    normals.resize(dims);
    const bool lv = p.model == MCG_MODEL_LOCAL_VOLATILITY;
    if (!lv && p.total_variance == 0.0) {
        for (uint32_t d = 0; d < dims; ++d) out[d] = 0.0;
        return;
    }
    for (uint32_t d = 0; d < dims; ++d) {
        if (p.engine == MCG_ENGINE_PSEUDO) {
            normals[d] = philox_normal(p.seed, unit, d, p.domain);
        } else {
            const uint32_t w = sobol_word(&p.dirs[static_cast<size_t>(d) * 32u], static_cast<uint32_t>(unit));
            const uint32_t x = p.scr[static_cast<size_t>(scramble) * dims + d].apply(w);
            normals[d] = inverse_standard_normal(open_unit_interval(x));
        }
    }
    if (lv && p.use_bridge) {
        p.bridge.apply(normals.data(), out, scratch);
    } else {
        for (uint32_t d = 0; d < dims; ++d) out[d] = normals[d];
    }
}

// One sampling unit, every product: primary path and (antithetic) its mate,
// crates/pricing/src/engine/risk/valuation.rs:138-149.
bool unit_values(const Plan& p, uint32_t scramble, uint64_t unit, std::vector<double>& out,
                 std::vector<double>& nodes_out, Failure& f) {
    const size_t P = p.products.size();
    const uint32_t dims = p.dimension;
    std::vector<double> z(dims), mate(dims), normals, scratch, tmp;
    std::vector<Obs> obs;
    unit_shocks(p, scramble, unit, z.data(), normals, scratch);
    out.assign(P * kWidth, 0.0);
    const size_t gv = p.grid.v.size();
    const bool want_nodes = p.model == MCG_MODEL_LOCAL_VOLATILITY && p.req_nodes;
    if (want_nodes) nodes_out.assign(P * gv, 0.0);
    std::vector<double> a(kWidth, 0.0), b(kWidth, 0.0), na(gv), nb(gv);
    for (size_t k = 0; k < P; ++k) {
        const Product& pr = p.products[k];
        bool ok;
        if (p.model == MCG_MODEL_BLACK_SCHOLES)
            ok = bs_unit_product(p, pr, z.data(), a.data(), f, obs, tmp);
        else
            ok = lv_unit_product(p, pr, z.data(), a.data(), want_nodes ? na.data() : nullptr, f);
        if (!ok) return false;
        if (p.antithetic) {
            for (uint32_t d = 0; d < dims; ++d) mate[d] = -z[d];
            if (p.model == MCG_MODEL_BLACK_SCHOLES)
                ok = bs_unit_product(p, pr, mate.data(), b.data(), f, obs, tmp);
            else
                ok = lv_unit_product(p, pr, mate.data(), b.data(), want_nodes ? nb.data() : nullptr, f);
            if (!ok) return false;
            for (int c = 0; c < kWidth; ++c) a[c] = (a[c] + b[c]) * 0.5;
            if (want_nodes)
                for (size_t g = 0; g < gv; ++g) na[g] = (na[g] + nb[g]) * 0.5;
        }
        std::copy(a.begin(), a.end(), out.begin() + k * kWidth);
        if (want_nodes) std::copy(na.begin(), na.end(), nodes_out.begin() + k * gv);
    }
    return true;
}

// --------------------------------------------------------------- driver

struct BlockResult {
    std::vector<Statistics> stats;  // products x components (+ nodes)
    Failure failure;
    uint64_t failed_unit = 0;
};

// Fixed-block map-reduce over [0, units) for one scramble,
// DeterministicExecutor::try_map_reduce_statistics_array_*, execution.rs:550-744.
bool map_reduce(const Plan& p, uint32_t scramble, uint64_t units, int threads,
                std::vector<Statistics>& total, mcg_error_record& err) {
    const size_t P = p.products.size();
    const size_t gv = (p.model == MCG_MODEL_LOCAL_VOLATILITY && p.req_nodes) ? p.grid.v.size() : 0;
    const size_t width = P * kWidth + P * gv;
    const uint64_t block = p.block;
    const uint64_t nblocks = (units + block - 1) / block;
    std::vector<BlockResult> results(nblocks);
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        std::vector<double> vals, nodes;
        for (;;) {
            const uint64_t b = next.fetch_add(1);
            if (b >= nblocks) break;
            BlockResult& r = results[b];
            r.stats.assign(width, Statistics{});
            const uint64_t begin = b * block, end = std::min(units, begin + block);
            for (uint64_t u = begin; u < end; ++u) {
                if (!unit_values(p, scramble, u, vals, nodes, r.failure)) {
                    r.failed_unit = u;
                    break;
                }
                for (size_t i = 0; i < P * kWidth; ++i) r.stats[i].add(vals[i]);
                for (size_t i = 0; i < P * gv; ++i) r.stats[P * kWidth + i].add(nodes[i]);
            }
        }
    };
    std::vector<std::thread> pool;
    const int nt = std::max(1, threads);
    for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    for (uint64_t b = 0; b < nblocks; ++b) {
        if (results[b].failure.code != MCG_OK) {
            err.code = results[b].failure.code;
            err.step = results[b].failure.step;
            err.sampling_unit = results[b].failed_unit;
            err.value_bits = bits_of(results[b].failure.value);
            return false;
        }
    }
    total.assign(width, Statistics{});
    for (size_t i = 0; i < width; ++i) {
        std::vector<NeumaierSum> sums;
        std::vector<CenteredMoment> moms;
        sums.reserve(nblocks);
        moms.reserve(nblocks);
        for (uint64_t b = 0; b < nblocks; ++b) {
            sums.push_back(results[b].stats[i].sum);
            moms.push_back(results[b].stats[i].moments);
        }
        total[i].sum = fixed_tree_reduce(sums, NeumaierSum::merged);
        total[i].moments = fixed_tree_reduce(moms, CenteredMoment::merged);
    }
    return true;
}

mcg_statistics to_c(const Statistics& s) {
    return {s.sum.sum, s.sum.correction, s.moments.count, s.moments.mean, s.moments.second_moment};
}

// estimate_from_statistics, crates/pricing/src/engine/risk/report.rs:454-473.
mcg_estimate estimate(const Statistics& s, uint64_t units, double scale) {
    const double inv = 1.0 / static_cast<double>(units);
    const double value = s.sum.total() * inv * scale;
    const double var = s.moments.count > 1
                           ? s.moments.second_moment / static_cast<double>(s.moments.count - 1)
                           : 0.0;
    const double se = std::sqrt(var * inv) * std::fabs(scale);
    const double hw = kNormal95 * se;
    return {value, se, value - hw, value + hw, units};
}

}  // namespace

// Full execute: SimulationPlan::execute, crates/pricing/src/engine/risk/valuation.rs:19-437
// and crates/pricing/src/engine/risk/local_vol.rs:24-420.
int evaluate(const mcg_plan_desc* desc, mcg_result* result, int threads) {
    Plan p;
    if (!build_plan(desc, p)) return MCG_ERR_INVALID_ARGUMENT;
    const size_t P = p.products.size();
    if (!result || result->product_capacity < P) return MCG_ERR_INVALID_ARGUMENT;
    std::memset(&result->error, 0, sizeof(result->error));
    const size_t gv = (p.model == MCG_MODEL_LOCAL_VOLATILITY && p.req_nodes) ? p.grid.v.size() : 0;
    std::vector<Statistics> stats;
    uint64_t independent;
    if (p.engine == MCG_ENGINE_PSEUDO) {
        if (!map_reduce(p, 0, p.units, threads, stats, result->error)) return result->error.code;
        independent = p.units;
        result->evaluated_paths = p.units * (p.antithetic ? 2 : 1);
    } else {
        const size_t width = P * kWidth + P * gv;
        std::vector<std::vector<double>> replicate(width);
        for (uint32_t s = 0; s < p.scrambles; ++s) {
            std::vector<Statistics> within;
            if (!map_reduce(p, s, p.units, threads, within, result->error)) return result->error.code;
            for (size_t i = 0; i < width; ++i)
                replicate[i].push_back(within[i].sum.total() / static_cast<double>(p.units));
        }
        stats.assign(width, Statistics{});
        for (size_t i = 0; i < width; ++i) {
            stats[i].moments = CenteredMoment::two_pass(replicate[i]);
            for (double v : replicate[i]) stats[i].sum.add(v);
        }
        if (result->replicate_means && result->replicate_capacity >= uint64_t{p.scrambles} * P * kComponents)
            for (uint32_t s = 0; s < p.scrambles; ++s)
                for (size_t k = 0; k < P; ++k)
                    for (int c = 0; c < kComponents; ++c)
                        result->replicate_means[(s * P + k) * kComponents + c] = replicate[k * kWidth + c][s];
        independent = p.scrambles;
        result->evaluated_paths = p.units * p.scrambles * (p.antithetic ? 2 : 1);
    }
    result->independent_sampling_units = independent;
    result->time_steps = p.dimension;
    result->effective_dimension = p.dimension;
    for (size_t k = 0; k < P; ++k) {
        mcg_product_result& r = result->products[k];
        for (int c = 0; c < kComponents; ++c) r.components[c] = to_c(stats[k * kWidth + c]);
        for (int c = 0; c < 2; ++c) r.adjoint_components[c] = to_c(stats[k * kWidth + kComponents + c]);
        const Statistics& price = stats[k * kWidth + MCG_PRICE];
        r.price = estimate(price, independent, 1.0);
        r.delta = estimate(stats[k * kWidth + MCG_DELTA], independent, 1.0);
        r.gamma = estimate(stats[k * kWidth + MCG_GAMMA], independent, 1.0);
        r.vega = estimate(stats[k * kWidth + MCG_VEGA], independent, 1.0);
        r.bump_delta = estimate(stats[k * kWidth + MCG_BUMP_DELTA], independent, 1.0);
        r.bump_gamma = estimate(stats[k * kWidth + MCG_BUMP_GAMMA], independent, 1.0);
        r.bump_vega = estimate(stats[k * kWidth + MCG_BUMP_VEGA], independent, 1.0);
        r.adjoint_delta = estimate(stats[k * kWidth + kComponents], independent, 1.0);
        r.adjoint_gamma = estimate(stats[k * kWidth + kComponents + 1], independent, 1.0);
        const double sv = price.moments.count > 1
                              ? price.moments.second_moment /
                                    static_cast<double>(price.moments.count - 1)
                              : 0.0;
        r.sampling_variance = p.total_variance == 0.0 ? 0.0 : sv;
        r.estimator_variance = r.sampling_variance / static_cast<double>(independent);
    }
    if (gv && result->local_vega_nodes && result->node_capacity >= P * gv) {
        for (size_t i = 0; i < P * gv; ++i) {
            const Statistics& s = stats[P * kWidth + i];
            result->local_vega_nodes[i] = to_c(s);
            if (result->local_vega_node_estimates)
                result->local_vega_node_estimates[i] = estimate(s, independent, 1.0);
        }
    }
    return MCG_OK;
}

const char* last_error() { return g_error.c_str(); }

// Exposed for the sampling tests: the increments of one unit.
int unit_shocks_api(const mcg_plan_desc* desc, uint32_t scramble, uint64_t unit, double* out) {
    Plan p;
    if (!build_plan(desc, p)) return MCG_ERR_INVALID_ARGUMENT;
    std::vector<double> normals, scratch;
    unit_shocks(p, scramble, unit, out, normals, scratch);
    return MCG_OK;
}

int unit_values_api(const mcg_plan_desc* desc, uint32_t scramble, uint64_t unit, double* out) {
    Plan p;
    if (!build_plan(desc, p)) return MCG_ERR_INVALID_ARGUMENT;
    std::vector<double> vals, nodes;
    Failure f;
    if (!unit_values(p, scramble, unit, vals, nodes, f)) return f.code;
    std::copy(vals.begin(), vals.end(), out);
    return MCG_OK;
}

// Bump-and-revalue on common random numbers: PricingSource::scenarios
// (crates/pricing/src/engine/risk/bump.rs:384-462) for spot and constant-
// volatility moves, CompiledScenarios::compile / evaluate (:568-690): every
// side is the plan with one input moved, on the same seeds; its sampling units
// (units_from_recorded, :490-523) are the unit values (pseudo-MC, antithetic
// pairs averaged) or the scramble means (RQMC); each estimate is paired(),
// the ordered two-pass statistics of the per-unit differences (:556-566).
int bump_evaluate_api(const mcg_plan_desc* desc, const mcg_bump_request* req, uint32_t count,
                      mcg_bump_estimate* est, mcg_bump_report* rep, int threads) {
    if (!desc || !req || !est || count == 0) return MCG_ERR_INVALID_ARGUMENT;
    if (rep) std::memset(rep, 0, sizeof(*rep));
    if (desc->product_count != 1) return MCG_ERR_UNSUPPORTED;
    struct Sc {
        int target;
        double amount;
    };
    std::vector<Sc> sc;
    std::vector<uint32_t> sc_of(count);
    bool gamma = false;
    for (uint32_t i = 0; i < count; ++i) {
        const int target = req[i].measure == MCG_BUMP_VOLATILITY_VEGA ? 1 : 0;
        if (!(req[i].size > 0.0)) return MCG_ERR_INVALID_ARGUMENT;
        if (target == 1 && desc->model != MCG_MODEL_BLACK_SCHOLES) return MCG_ERR_INVALID_ARGUMENT;
        const double level = target == 0 ? desc->spot : desc->volatility;
        const double amount = req[i].relative ? req[i].size * level : req[i].size;
        uint32_t j = 0;
        while (j < sc.size() && !(sc[j].target == target && sc[j].amount == amount)) ++j;
        if (j == sc.size()) sc.push_back({target, amount});
        sc_of[i] = j;
        gamma |= req[i].measure == MCG_BUMP_SPOT_GAMMA;
    }
    const uint32_t ns = static_cast<uint32_t>(sc.size());
    const uint32_t sides = 2 * ns + (gamma ? 1u : 0u);
    std::vector<std::vector<double>> units_of(sides);
    std::vector<double> side_price(sides);
    uint64_t independent = 0;
    for (uint32_t k = 0; k < sides; ++k) {
        mcg_plan_desc s = *desc;
        if (k < 2 * ns) {
            const double sign = k % 2 == 0 ? 1.0 : -1.0;
            if (sc[k / 2].target == 0) s.spot = desc->spot + sign * sc[k / 2].amount;
            else s.volatility = desc->volatility + sign * sc[k / 2].amount;
            if (!(s.spot > 0.0) || (sc[k / 2].target == 1 && !(s.volatility > 0.0))) return MCG_ERR_INVALID_ARGUMENT;
        }
        Plan p;
        if (!build_plan(&s, p)) return MCG_ERR_INVALID_ARGUMENT;
        mcg_error_record err{};
        if (p.engine == MCG_ENGINE_PSEUDO) {
            std::vector<Statistics> stats;
            if (!map_reduce(p, 0, p.units, threads, stats, err)) return err.code;
            side_price[k] = stats[MCG_PRICE].sum.total() / static_cast<double>(p.units);
            std::vector<double>& u = units_of[k];
            u.assign(p.units, 0.0);
            std::atomic<uint64_t> next{0};
            std::atomic<int> failed{0};
            auto worker = [&]() {
                std::vector<double> vals, nodes;
                Failure f;
                for (;;) {
                    const uint64_t b = next.fetch_add(4096);
                    if (b >= p.units) break;
                    for (uint64_t i = b; i < std::min<uint64_t>(p.units, b + 4096); ++i) {
                        if (!unit_values(p, 0, i, vals, nodes, f)) {
                            failed = f.code;
                            return;
                        }
                        u[i] = vals[MCG_PRICE];
                    }
                }
            };
            std::vector<std::thread> pool;
            for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(worker);
            for (auto& t : pool) t.join();
            if (failed) return failed;
            independent = p.units;
        } else {
            std::vector<double>& u = units_of[k];
            NeumaierSum total;
            for (uint32_t sidx = 0; sidx < p.scrambles; ++sidx) {
                std::vector<Statistics> within;
                if (!map_reduce(p, sidx, p.units, threads, within, err)) return err.code;
                u.push_back(within[MCG_PRICE].sum.total() / static_cast<double>(p.units));
                total.add(u.back());
            }
            side_price[k] = total.total() / static_cast<double>(p.scrambles);
            independent = p.scrambles;
        }
    }
    const uint32_t base = 2 * ns;
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t j = sc_of[i];
        const double h = sc[j].amount;
        const bool second = req[i].measure == MCG_BUMP_SPOT_GAMMA;
        const std::vector<double>& up = units_of[2 * j];
        const std::vector<double>& down = units_of[2 * j + 1];
        std::vector<double> diff(up.size());
        for (size_t q = 0; q < up.size(); ++q)
            diff[q] = second ? ((up[q] - units_of[base][q]) + (down[q] - units_of[base][q])) / (h * h)
                             : (up[q] - down[q]) / (2.0 * h);
        if (diff.size() < 2) return MCG_ERR_INVALID_ARGUMENT;
        NeumaierSum sum;
        for (double v : diff) sum.add(v);
        const CenteredMoment m = CenteredMoment::two_pass(diff);
        const double n = static_cast<double>(diff.size());
        const double value = sum.total() / n;
        const double se = std::sqrt(m.second_moment / (n - 1.0) / n);
        est[i] = mcg_bump_estimate{req[i].measure, j, h, value, se, static_cast<uint64_t>(diff.size()),
                                   side_price[2 * j], side_price[2 * j + 1]};
    }
    if (rep) {
        rep->scenarios = ns;
        rep->sides = sides;
        rep->evaluations = 2ull * ns + (gamma ? 1u : 0u);
        if (gamma) rep->base_price.value = side_price[base];
        rep->base_price.effective_sampling_units = independent;
    }
    return MCG_OK;
}

// One Log-Euler path on given nodes, forwards, grid and shocks, and its
// reverse sweep for given dPayoff/dS_k seeds (the equation-(10) step
// adjoints of the reference's local-vol fixtures): the path's states and the
// grid-value adjoints.
int lv_step_adjoints_api(const double* times, uint32_t n_times, const double* forwards, const double* grid_t,
                         uint32_t nt, const double* grid_x, uint32_t nx, const double* values, double initial,
                         const double* shocks, const double* state_seeds, double* states_out,
                         double* grid_adj_out) {
    Plan p;
    p.nodes.assign(times, times + n_times);
    p.fwd[0].assign(forwards, forwards + n_times);
    p.bump_spot[0] = initial;
    p.grid.t.assign(grid_t, grid_t + nt);
    p.grid.x.assign(grid_x, grid_x + nx);
    p.grid.v.assign(values, values + static_cast<size_t>(nt) * nx);
    p.grid.floor = 1e-8;
    p.grid.cap = 4.0;
    LvPath path;
    Failure f;
    if (!lv_evolve(p, 0, shocks, path, f)) return f.code;
    std::vector<double> seeds(state_seeds, state_seeds + n_times), var_seeds(n_times, 0.0), grid_adj;
    double initial_adjoint = 0.0, x_sum = 0.0;
    if (!lv_reverse(p, 0, path, seeds, var_seeds, grid_adj, initial_adjoint, x_sum, f)) return f.code;
    for (uint32_t i = 0; i < n_times; ++i) states_out[i] = path.state[i];
    for (size_t i = 0; i < grid_adj.size(); ++i) grid_adj_out[i] = grid_adj[i];
    return MCG_OK;
}

// A continuous barrier on one Log-Euler path (the reference's direct-variance
// fixture): exact bridge survival over the first `monitor_end` intervals with
// node variances at the path's states, a knock-out/in payoff of the vanilla
// q S_T^2 with a rebate, discounted; the price and the grid-value adjoints of
// the reverse sweep with the bridge's state and direct-variance seeds.
int lv_barrier_adjoints_api(const double* times, uint32_t n_times, const double* forwards, const double* grid_t,
                            uint32_t nt, const double* grid_x, uint32_t nx, const double* values, double initial,
                            const double* shocks, double barrier, int up, int knock_out, uint32_t monitor_end,
                            double quadratic, double rebate, double discount, double* price_out,
                            double* grid_adj_out) {
    Plan p;
    p.nodes.assign(times, times + n_times);
    p.fwd[0].assign(forwards, forwards + n_times);
    p.bump_spot[0] = initial;
    p.grid.t.assign(grid_t, grid_t + nt);
    p.grid.x.assign(grid_x, grid_x + nx);
    p.grid.v.assign(values, values + static_cast<size_t>(nt) * nx);
    p.grid.floor = 1e-8;
    p.grid.cap = 4.0;
    p.smoothing = 0.0;
    LvPath path;
    Failure f;
    if (!lv_evolve(p, 0, shocks, path, f)) return f.code;
    std::vector<double> nv;
    if (!lv_node_variances(p, 0, path, nv, f)) return f.code;
    mcg_product_desc d{};
    d.kind = MCG_PRODUCT_CONTINUOUS_BARRIER;
    d.barrier = barrier;
    d.barrier_direction = up ? MCG_BARRIER_UP : MCG_BARRIER_DOWN;
    d.barrier_style = knock_out ? MCG_KNOCK_OUT : MCG_KNOCK_IN;
    BarrierEval be;
    if (!barrier_bridge(p, d, path.state.data(), nv.data(), p.nodes.data(), monitor_end + 1, be, f)) return f.code;
    const double st = path.state[n_times - 1];
    const double vanilla = quadratic * st * st;
    const double surv = be.survival;
    const double value = knock_out ? rebate + surv * (vanilla - rebate) : vanilla + surv * (rebate - vanilla);
    *price_out = discount * value;
    std::vector<double> seeds(n_times, 0.0), var_seeds(n_times, 0.0), grid_adj;
    seeds[n_times - 1] = discount * (knock_out ? surv : 1.0 - surv) * 2.0 * quadratic * st;
    if (be.exact_active) {
        const double lsa = discount * (knock_out ? vanilla - rebate : rebate - vanilla) * surv;
        for (size_t k = 0; k < be.ex.size(); ++k) {
            seeds[k] += lsa * be.ex[k].d_left_state;
            seeds[k + 1] += lsa * be.ex[k].d_right_state;
            var_seeds[k] += lsa * be.ex[k].d_left_var;
            var_seeds[k + 1] += lsa * be.ex[k].d_right_var;
        }
    }
    double initial_adjoint = 0.0, x_sum = 0.0;
    if (!lv_reverse(p, 0, path, seeds, var_seeds, grid_adj, initial_adjoint, x_sum, f)) return f.code;
    for (size_t i = 0; i < grid_adj.size(); ++i) grid_adj_out[i] = grid_adj[i];
    return MCG_OK;
}

int time_grid_api(const mcg_plan_desc* desc, double* nodes_out, uint32_t capacity,
                  uint32_t* count) {
    Plan p;
    if (!build_plan(desc, p)) return MCG_ERR_INVALID_ARGUMENT;
    *count = static_cast<uint32_t>(p.nodes.size());
    for (size_t i = 0; i < p.nodes.size() && i < capacity; ++i) nodes_out[i] = p.nodes[i];
    return MCG_OK;
}

// Path matrix of an early-exercise plan: the spot at every observation
// (exercise) date, spots[date * paths + path], for the plan's engine under the
// random domain `domain`.  Path order and mates follow pseudo_lsm_path_matrices
// and rqmc_lsm_path_matrices (crates/pricing/src/engine/mc/early_exercise.rs:28-175,
// 177-320): path = unit * 2 (+1 for the antithetic mate), RQMC units numbered
// scramble-major.  Spots are post_spot of write_lsm_trajectory and
// write_local_vol_lsm_trajectory (early_exercise.rs:330-450).
int lsm_spots(const mcg_plan_desc* desc, uint32_t domain, int threads, std::vector<double>& spots,
              uint64_t& path_count, mcg_error_record& err, std::vector<double>* brownians) {
    Plan p;
    if (!build_plan(desc, p)) return MCG_ERR_INVALID_ARGUMENT;
    p.domain = domain;
    const bool rqmc = p.engine == MCG_ENGINE_RQMC;
    const uint64_t mult = p.antithetic ? 2 : 1;
    const uint64_t units = p.units * (rqmc ? p.scrambles : 1);
    const size_t dates = p.obs_t.size();
    path_count = units * mult;
    spots.assign(dates * path_count, 0.0);
    if (brownians) brownians->assign(dates * path_count, 0.0);
    const bool lv = p.model == MCG_MODEL_LOCAL_VOLATILITY;
    std::vector<Failure> failures(static_cast<size_t>(std::max(1, threads)));
    std::vector<uint64_t> failed_unit(failures.size(), ~0ull);
    std::atomic<uint64_t> next{0};
    constexpr uint64_t kChunk = 1024;
    auto worker = [&](size_t t) {
        std::vector<double> z(p.dimension), normals, scratch;
        std::vector<Obs> obs(dates);
        LvPath path;
        for (;;) {
            const uint64_t begin = next.fetch_add(kChunk);
            if (begin >= units || failures[t].code != MCG_OK) break;
            const uint64_t end = std::min(units, begin + kChunk);
            for (uint64_t u = begin; u < end; ++u) {
                const uint32_t scramble = rqmc ? static_cast<uint32_t>(u / p.units) : 0u;
                const uint64_t local = rqmc ? u % p.units : u;
                unit_shocks(p, scramble, local, z.data(), normals, scratch);
                for (uint64_t m = 0; m < mult; ++m) {
                    if (m == 1)
                        for (double& v : z) v = -v;
                    const uint64_t col = u * mult + m;
                    if (lv) {
                        if (!lv_evolve(p, 0, z.data(), path, failures[t])) {
                            failed_unit[t] = u;
                            return;
                        }
                        for (size_t d = 0; d < dates; ++d)
                            spots[d * path_count + col] = 0.0 * p.spot + 1.0 * path.state[p.obs_node[d]];
                    } else {
                        bs_observations(p, z.data(), p.spot, p.vol, obs.data());
                        for (size_t d = 0; d < dates; ++d) spots[d * path_count + col] = obs[d].post_spot;
                        if (brownians)
                            for (size_t d = 0; d < dates; ++d) (*brownians)[d * path_count + col] = obs[d].w;
                    }
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (size_t t = 0; t < failures.size(); ++t) pool.emplace_back(worker, t);
    for (auto& t : pool) t.join();
    uint64_t first = ~0ull;
    size_t which = 0;
    for (size_t t = 0; t < failures.size(); ++t)
        if (failures[t].code != MCG_OK && failed_unit[t] < first) {
            first = failed_unit[t];
            which = t;
        }
    if (first != ~0ull) {
        err.code = failures[which].code;
        err.step = failures[which].step;
        err.sampling_unit = first;
        err.value_bits = bits_of(failures[which].value);
        return err.code;
    }
    return MCG_OK;
}

// Fixed-policy pathwise risk of an early-exercise plan under Black--Scholes:
// per sampling unit, the 18 components of fixed_policy_pathwise_values
// (crates/pricing/src/engine/processes/black_scholes.rs:358-415) for the
// discounted exercise value at each path's stopping date (its
// pathwise_aad_for_output, :567-643), antithetic mates averaged, reduced as
// constant_vol_fixed_policy_pseudo/rqmc_statistics
// (crates/pricing/src/engine/mc/early_exercise.rs:454-600) do.
int lsm_fixed_policy_risk(const mcg_plan_desc* desc, const uint32_t* stops, const double* df, int threads,
                          mcg_lsm_result* result) {
    Plan p;
    if (!build_plan(desc, p)) return MCG_ERR_INVALID_ARGUMENT;
    const bool rqmc = p.engine == MCG_ENGINE_RQMC;
    const uint64_t mult = p.antithetic ? 2 : 1;
    const mcg_product_desc& pr = desc->products[0];
    const bool call = pr.side == MCG_CALL;
    const size_t n = p.obs_t.size();
    auto eval = [&](const double* z, uint32_t k, double spot, double vol, std::vector<Obs>& obs, double& price,
                    double& delta, double& vega) {
        bs_observations(p, z, spot, vol, obs.data());
        const double s = obs[k].post_spot;
        const double in = call ? s - pr.strike : pr.strike - s;
        const double value = (in >= 0.0 ? in : 0.0) * pr.notional;
        const double adj = (in >= 0.0 ? pr.notional : 0.0) * (call ? 1.0 : -1.0);
        double d = 0.0, v = 0.0;
        if (adj != 0.0) {
            d += adj * 1.0 * obs[k].f / spot;
            v += adj * 1.0 * obs[k].f * (-vol * p.obs_t[k] + obs[k].w);
        }
        price = df[k] * value;
        delta = df[k] * d;
        vega = df[k] * v;
    };
    auto unit_components = [&](const double* z, uint32_t k, std::vector<Obs>& obs, double* values) {
        double bp, bd, bv, dp, dd, dv, up, ud, uv, x, y, w;
        eval(z, k, p.spot, p.vol, obs, bp, bd, bv);
        double gamma = 0.0;
        if (p.req_gamma) {
            const double bump = p.gamma_bump;
            eval(z, k, p.spot - bump, p.vol, obs, x, dd, w);
            eval(z, k, p.spot + bump, p.vol, obs, x, ud, w);
            gamma = (ud - dd) / (2.0 * bump);
        }
        const double sb = p.spot_bump;
        eval(z, k, p.spot - sb, p.vol, obs, dp, dd, dv);
        eval(z, k, p.spot + sb, p.vol, obs, up, ud, uv);
        const double bump_delta = (up - dp) / (2.0 * sb);
        const double bump_gamma = (up - 2.0 * bp + dp) / (sb * sb);
        double bump_vega = 0.0;
        if (p.vol_bump != 0.0) {
            const double vb = p.vol_bump;
            eval(z, k, p.spot, p.vol - vb, obs, x, y, w);
            double hi;
            eval(z, k, p.spot, p.vol + vb, obs, hi, y, w);
            bump_vega = (hi - x) / (2.0 * vb);
        }
        for (int c = 0; c < kComponents; ++c) values[c] = 0.0;
        values[MCG_PRICE] = bp;
        values[MCG_DELTA] = bd;
        values[MCG_VEGA] = bv;
        values[MCG_GAMMA] = gamma;
        values[MCG_BUMP_DELTA] = bump_delta;
        values[MCG_DELTA_DIFFERENCE] = bump_delta - bd;
        values[MCG_BUMP_VEGA] = bump_vega;
        values[MCG_VEGA_DIFFERENCE] = bump_vega - bv;
        values[MCG_BUMP_GAMMA] = bump_gamma;
        values[MCG_GAMMA_DIFFERENCE] = bump_gamma - gamma;
    };
    // One scramble (RQMC) or the whole pseudo run: fixed blocks, fixed tree.
    auto reduce = [&](uint32_t scramble, std::vector<Statistics>& out) {
        const uint64_t units = p.units;
        const uint64_t nblocks = (units + p.block - 1) / p.block;
        std::vector<std::vector<Statistics>> blocks(nblocks, std::vector<Statistics>(kComponents));
        std::atomic<uint64_t> next{0};
        auto worker = [&]() {
            std::vector<double> z(p.dimension), mate(p.dimension), normals, scratch;
            std::vector<Obs> obs(n);
            double a[kComponents], b[kComponents];
            for (;;) {
                const uint64_t blk = next.fetch_add(1);
                if (blk >= nblocks) break;
                for (uint64_t u = blk * p.block; u < std::min(units, (blk + 1) * p.block); ++u) {
                    unit_shocks(p, scramble, u, z.data(), normals, scratch);
                    const uint64_t base = ((rqmc ? static_cast<uint64_t>(scramble) * units : 0) + u) * mult;
                    unit_components(z.data(), stops[base], obs, a);
                    if (mult == 2) {
                        for (size_t i = 0; i < z.size(); ++i) mate[i] = -z[i];
                        unit_components(mate.data(), stops[base + 1], obs, b);
                        for (int c = 0; c < kComponents; ++c) a[c] = (a[c] + b[c]) * 0.5;
                    }
                    for (int c = 0; c < kComponents; ++c) blocks[blk][c].add(a[c]);
                }
            }
        };
        std::vector<std::thread> pool;
        for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
        out.assign(kComponents, Statistics{});
        for (int c = 0; c < kComponents; ++c) {
            std::vector<NeumaierSum> sums;
            std::vector<CenteredMoment> moms;
            for (uint64_t b = 0; b < nblocks; ++b) {
                sums.push_back(blocks[b][c].sum);
                moms.push_back(blocks[b][c].moments);
            }
            out[c].sum = fixed_tree_reduce(sums, NeumaierSum::merged);
            out[c].moments = fixed_tree_reduce(moms, CenteredMoment::merged);
        }
    };
    std::vector<Statistics> total;
    uint64_t independent;
    if (!rqmc) {
        reduce(0, total);
        independent = p.units;
    } else {
        std::vector<std::vector<double>> reps(kComponents);
        for (uint32_t s = 0; s < p.scrambles; ++s) {
            std::vector<Statistics> within;
            reduce(s, within);
            for (int c = 0; c < kComponents; ++c)
                reps[c].push_back(within[c].sum.total() / static_cast<double>(p.units));
        }
        total.assign(kComponents, Statistics{});
        for (int c = 0; c < kComponents; ++c) {
            total[c].moments = CenteredMoment::two_pass(reps[c]);
            for (double v : reps[c]) total[c].sum.add(v);
        }
        independent = p.scrambles;
    }
    for (int c = 0; c < kComponents; ++c) result->risk_components[c] = to_c(total[c]);
    result->delta = estimate(total[MCG_DELTA], independent, 1.0);
    result->gamma = estimate(total[MCG_GAMMA], independent, 1.0);
    result->vega = estimate(total[MCG_VEGA], independent, 1.0);
    result->bump_delta = estimate(total[MCG_BUMP_DELTA], independent, 1.0);
    result->bump_gamma = estimate(total[MCG_BUMP_GAMMA], independent, 1.0);
    result->bump_vega = estimate(total[MCG_BUMP_VEGA], independent, 1.0);
    return MCG_OK;
}

// One LV valuation path's fixed-policy values: the discounted exercise value
// at its stopping date k (the American payoff graph's output k,
// local_vol_pathwise_values_and_buckets_inner with a cash-flow selection,
// crates/pricing/src/engine/risk/pathwise_local_vol.rs:127-361): price,
// reverse-sweep Vega and node values (seed at the stop node), CRN Delta and
// Gamma from the bumped spot runtimes.
bool lv_fixed_values(const Plan& p, const mcg_product_desc& pd, const double* shocks, uint32_t k, double dfk,
                     double* values, double* nodes, Failure& f) {
    for (int c = 0; c < kComponents; ++c) values[c] = 0.0;
    const bool call = pd.side == MCG_CALL;
    auto exercise = [&](int which, const LvPath& path, double& adj) {
        const double s = 0.0 * p.bump_spot[which] + 1.0 * path.state[p.obs_node[k]];
        const double in = call ? s - pd.strike : pd.strike - s;
        adj = (in >= 0.0 ? pd.notional : 0.0) * (call ? 1.0 : -1.0);
        return dfk * ((in >= 0.0 ? in : 0.0) * pd.notional);
    };
    LvPath path;
    if (!lv_evolve(p, 0, shocks, path, f)) return false;
    double adj;
    const double price = exercise(0, path, adj);
    values[MCG_PRICE] = price;
    if (p.req_vega || p.req_nodes) {
        const size_t count = p.nodes.size();
        std::vector<double> seeds(count, 0.0), vseeds(count, 0.0), grid_adj;
        seeds[p.obs_node[k]] += dfk * adj * 1.0;
        double lambda0, x_sum;
        if (!lv_reverse(p, 0, path, seeds, vseeds, grid_adj, lambda0, x_sum, f)) return false;
        NeumaierSum v;
        for (size_t j = 0; j < grid_adj.size(); ++j) {
            const double node = grid_adj[j] * 2.0 * std::sqrt(p.grid.v[j]);
            v.add(node);
            if (nodes) nodes[j] = node;
        }
        values[MCG_VEGA] = v.total();
    }
    if (p.req_delta || p.req_gamma) {
        LvPath bumped;
        double a;
        if (!lv_evolve(p, 1, shocks, bumped, f)) return false;
        const double down = exercise(1, bumped, a);
        if (!lv_evolve(p, 2, shocks, bumped, f)) return false;
        const double up = exercise(2, bumped, a);
        const double h = p.spot_bump;
        const double delta = (up - down) / (2.0 * h);
        values[MCG_DELTA] = delta;
        values[MCG_BUMP_DELTA] = delta;
        if (p.req_gamma) {
            const double gamma = (up - 2.0 * price + down) / (h * h);
            values[MCG_GAMMA] = gamma;
            values[MCG_BUMP_GAMMA] = gamma;
        }
    }
    return true;
}

// Fixed-policy risk of an early-exercise plan under local volatility,
// local_vol_fixed_policy_pseudo/rqmc_statistics_with_vega_kt
// (crates/pricing/src/engine/risk/early_exercise.rs:465-700): per unit the
// pair-averaged values (average_local_vol_pathwise), pseudo: a two-pass over
// the units' values in order; RQMC: per-scramble means of Neumaier sums, then
// a two-pass over the scramble means.  Node values are reduced the same way.
int lsm_lv_fixed_policy_risk(const mcg_plan_desc* desc, const uint32_t* stops, const double* df, int threads,
                             mcg_lsm_result* result) {
    Plan p;
    if (!build_plan(desc, p)) return MCG_ERR_INVALID_ARGUMENT;
    const bool rqmc = p.engine == MCG_ENGINE_RQMC;
    const uint64_t mult = p.antithetic ? 2 : 1;
    const uint64_t units = p.units * (rqmc ? p.scrambles : 1);
    const mcg_product_desc& pd = desc->products[0];
    const size_t nv = p.grid.v.size();
    const bool want_nodes = p.req_nodes && result->local_vega_nodes && result->node_capacity >= nv;
    const size_t width = kComponents + (want_nodes ? nv : 0);
    std::vector<double> vals(units * width, 0.0);
    std::vector<Failure> failures(static_cast<size_t>(std::max(1, threads)));
    std::vector<uint64_t> failed(failures.size(), ~0ull);
    std::atomic<uint64_t> next{0};
    auto worker = [&](size_t t) {
        std::vector<double> z(p.dimension), mate(p.dimension), normals, scratch, a(kComponents), b(kComponents);
        std::vector<double> na(nv), nb(nv);
        for (;;) {
            const uint64_t u = next.fetch_add(1);
            if (u >= units || failures[t].code != MCG_OK) break;
            const uint32_t scramble = rqmc ? static_cast<uint32_t>(u / p.units) : 0u;
            const uint64_t local = rqmc ? u % p.units : u;
            unit_shocks(p, scramble, local, z.data(), normals, scratch);
            const uint32_t k0 = stops[u * mult];
            if (!lv_fixed_values(p, pd, z.data(), k0, df[k0], a.data(), want_nodes ? na.data() : nullptr,
                                 failures[t])) {
                failed[t] = u;
                return;
            }
            double* out = vals.data() + u * width;
            if (mult == 2) {
                for (size_t i = 0; i < z.size(); ++i) mate[i] = -z[i];
                const uint32_t k1 = stops[u * mult + 1];
                if (!lv_fixed_values(p, pd, mate.data(), k1, df[k1], b.data(), want_nodes ? nb.data() : nullptr,
                                     failures[t])) {
                    failed[t] = u;
                    return;
                }
                for (int c = 0; c < kComponents; ++c) out[c] = (a[c] + b[c]) * 0.5;
                if (want_nodes)
                    for (size_t j = 0; j < nv; ++j) out[kComponents + j] = (na[j] + nb[j]) * 0.5;
            } else {
                for (int c = 0; c < kComponents; ++c) out[c] = a[c];
                if (want_nodes)
                    for (size_t j = 0; j < nv; ++j) out[kComponents + j] = na[j];
            }
        }
    };
    std::vector<std::thread> pool;
    for (size_t t = 0; t < failures.size(); ++t) pool.emplace_back(worker, t);
    for (auto& t : pool) t.join();
    for (size_t t = 0; t < failures.size(); ++t)
        if (failures[t].code != MCG_OK) {
            result->error.code = failures[t].code;
            result->error.step = failures[t].step;
            result->error.sampling_unit = failed[t];
            return failures[t].code;
        }
    // ordered reduction of one column
    auto reduce = [&](size_t col, Statistics& st) {
        std::vector<double> column;
        if (!rqmc) {
            column.resize(units);
            for (uint64_t u = 0; u < units; ++u) column[u] = vals[u * width + col];
        } else {
            for (uint32_t s = 0; s < p.scrambles; ++s) {
                NeumaierSum sum;
                for (uint64_t i = 0; i < p.units; ++i) sum.add(vals[(s * p.units + i) * width + col]);
                column.push_back(sum.total() / static_cast<double>(p.units));
            }
        }
        st = Statistics{};
        for (double v : column) st.sum.add(v);
        st.moments = CenteredMoment::two_pass(column);
    };
    const uint64_t independent = rqmc ? p.scrambles : p.units;
    std::vector<Statistics> total(kComponents);
    for (int c = 0; c < kComponents; ++c) {
        reduce(static_cast<size_t>(c), total[c]);
        result->risk_components[c] = to_c(total[c]);
    }
    result->delta = estimate(total[MCG_DELTA], independent, 1.0);
    result->gamma = estimate(total[MCG_GAMMA], independent, 1.0);
    result->vega = estimate(total[MCG_VEGA], independent, 1.0);
    result->bump_delta = estimate(total[MCG_BUMP_DELTA], independent, 1.0);
    result->bump_gamma = estimate(total[MCG_BUMP_GAMMA], independent, 1.0);
    result->bump_vega = estimate(total[MCG_BUMP_VEGA], independent, 1.0);
    if (want_nodes)
        for (size_t j = 0; j < nv; ++j) {
            Statistics st;
            reduce(kComponents + j, st);
            result->local_vega_nodes[j] = to_c(st);
            if (result->local_vega_node_estimates) result->local_vega_node_estimates[j] = estimate(st, independent, 1.0);
        }
    return MCG_OK;
}

double plan_discount(const mcg_plan_desc* desc, double t) {
    Curve c;
    c.set(desc->discount_curve.times, desc->discount_curve.discount_factors,
          desc->discount_curve.pillar_count);
    return std::exp(c.log_discount(t));
}

// The forward of the plan's spot at t (forward_at, as the path store uses it).
double plan_forward(const mcg_plan_desc* desc, double t) {
    Plan p;
    p.spot = desc->spot;
    p.rc.set(desc->discount_curve.times, desc->discount_curve.discount_factors,
             desc->discount_curve.pillar_count);
    p.qc.set(desc->dividend_curve.times, desc->dividend_curve.discount_factors,
             desc->dividend_curve.pillar_count);
    return forward_at(p, p.spot, t);
}

}  // namespace oracle

namespace oracle {
// Continuous-barrier bridge over one state sequence (test entry point).
int barrier_path_api(int up, double barrier, double h, const double* states,
                     const double* variances, const double* times, size_t count, double* survival,
                     double* diag) {
    Plan p;
    p.smoothing = h;
    mcg_product_desc d{};
    d.kind = MCG_PRODUCT_CONTINUOUS_BARRIER;
    d.barrier_direction = up ? MCG_BARRIER_UP : MCG_BARRIER_DOWN;
    d.barrier = barrier;
    BarrierEval be;
    Failure f;
    if (!barrier_bridge(p, d, states, variances, times, count, be, f)) return f.code;
    *survival = be.survival;
    for (int k = 0; k < 8; ++k) diag[k] = be.diag[k];
    return 0;
}
}  // namespace oracle

namespace oracle {
// Smoothing and bridge primitives for the fixture tests.
void smoothing_api(double h, double input, double* out) {
    Deriv ind, pos;
    double c;
    indicator_with_complement(h, input, ind, c);
    positive_part_with_complement(h, input, pos, c);
    out[0] = ind.value; out[1] = ind.first; out[2] = ind.second;
    out[3] = pos.value; out[4] = pos.first; out[5] = pos.second;
}
void extrema_api(double h, double left, double right, double* out) {
    out[0] = smooth_maximum(h, left, right).value;
    out[1] = smooth_minimum(h, left, right).value;
}
int exact_bridge_api(int up, double barrier, double s0, double s1, double integrated, double* survival) {
    ExactInterval iv;
    Failure f;
    if (!exact_interval(up != 0, s0, s1, barrier, barrier, integrated, integrated, 1.0, iv, f)) return f.code;
    *survival = std::exp(iv.log_survival);
    return 0;
}
int smoothed_bridge_api(int up, double barrier, double s0, double s1, double h, double integrated,
                        double* out) {
    SmoothInterval si;
    Failure f;
    if (!smooth_interval(up != 0, s0, s1, barrier, barrier, 1.0, 1.0, integrated, integrated, 1.0, h, si, f))
        return f.code;
    out[0] = si.left.hit_weight;
    out[1] = si.right.hit_weight;
    out[2] = si.left.eld;
    out[3] = si.right.eld;
    out[4] = std::exp(si.log_survival);
    out[5] = si.left.safety_weight * si.right.safety_weight;
    return 0;
}
}  // namespace oracle

namespace oracle {
// Adjoint of one continuous-barrier interval (test entry point): state and
// direct-variance seeds of the two nodes for a log-survival adjoint lsa.
int interval_adjoint_api(int up, double barrier, double h, double lsa, double ls, double rs, double lv,
                         double rv, double dt, double* out) {
    Failure f;
    if (h > 0.0) {
        SmoothInterval si;
        if (!smooth_interval(up != 0, ls, rs, barrier, barrier, 1.0, 1.0, lv, rv, dt, h, si, f)) return f.code;
        out[0] = 0.0 * si.left.hit_d_state + (lsa * si.d_left_distance) * si.left.eld_d_state;
        out[1] = 0.0 * si.right.hit_d_state + (lsa * si.d_right_distance) * si.right.eld_d_state;
        out[2] = lsa * si.d_left_var;
        out[3] = lsa * si.d_right_var;
        return 0;
    }
    ExactInterval iv;
    if (!exact_interval(up != 0, ls, rs, barrier, barrier, lv, rv, dt, iv, f)) return f.code;
    out[0] = lsa * iv.d_left_state;
    out[1] = lsa * iv.d_right_state;
    out[2] = lsa * iv.d_left_var;
    out[3] = lsa * iv.d_right_var;
    return 0;
}
}  // namespace oracle

// oracle_core.cpp -- sampling, bridge, statistics, curve and grid primitives of
// the CPU oracle.  TEST INFRASTRUCTURE ONLY (see oracle_core.h).
#include "../include/mcg.h"
#include "oracle_core.h"

#include <algorithm>
#include <queue>

namespace oracle {

namespace {

double polynomial(double argument, const double* c) {
    double value = c[7];
    for (int i = 6; i >= 0; --i) value = value * argument + c[i];
    return value;
}

// Wichura AS241 coefficient table (Applied Statistics 37(3), 1988), as the
// binary64 values of crates/pricing/src/engine/sampling/random.rs:181-240,
// written as exact hexadecimal literals.
const double kA[8] = {0x1.b18d91e9eef75p+1, 0x1.0a4888b1a436ep+7, 0x1.ece5d2213c0ccp+10, 0x1.ad1d8cd4ee71dp+13,
                      0x1.66c3e869b752ap+15, 0x1.06c1c55b78f20p+16, 0x1.052d26b2e4604p+15, 0x1.39a296f7d925ep+11};
const double kB[8] = {0x1.0000000000000p+0, 0x1.5281b386e1ab5p+5, 0x1.5797efdc8b3f7p+9, 0x1.512322e75c89fp+12,
                      0x1.4b772d5d65266p+14, 0x1.3317caa64f4bep+15, 0x1.c0e457cb1ae76p+14, 0x1.46a7eca984b6ap+12};
const double kC[8] = {0x1.6c665fde9526ap+0, 0x1.2857748cab19bp+2, 0x1.713f71462256ap+2, 0x1.d2ecb1a3d02c4p+1,
                      0x1.453cc085375b2p+0, 0x1.ef2abb9b85c37p-3, 0x1.744eb6c45ec67p-6, 0x1.9615ac0b7ace9p-11};
const double kD[8] = {0x1.0000000000000p+0, 0x1.06cefbb46a449p+1, 0x1.ad278e6526633p+0, 0x1.61292f23385c9p-1,
                      0x1.2f5123394f040p-3, 0x1.f207a7eab17bfp-7, 0x1.1f18cbfdf2728p-11, 0x1.20d3f686439e4p-30};
const double kE[8] = {0x1.aa1b1c13ee527p+2, 0x1.5daea6e875003p+2, 0x1.c8ea6461fa445p+0, 0x1.2fad9315255d0p-2,
                      0x1.b2b41193b4ee7p-6, 0x1.45c1908425345p-10, 0x1.c6ec6cc59e02ap-16, 0x1.afb74d693bf93p-23};
const double kF[8] = {0x1.0000000000000p+0, 0x1.331d34fc7d77ep-1, 0x1.186eb183443fbp-3, 0x1.e76f93215462ap-7,
                      0x1.9c8bc979dc5d7p-11, 0x1.35c2c494cf5d0p-16, 0x1.31446f740bfc3p-23, 0x1.269bff1f8c190p-49};

}  // namespace

// random.rs:176-277.
double inverse_standard_normal(double probability) {
    if (!(probability > 0.0 && probability < 1.0)) return std::nan("");
    const double centered = probability - 0.5;
    if (std::fabs(centered) <= 0.425) {
        const double argument = 0.180625 - centered * centered;
        return centered * polynomial(argument, kA) / polynomial(argument, kB);
    }
    const double tail = centered < 0.0 ? probability : 1.0 - probability;
    const double radius = std::sqrt(-std::log(tail));
    double magnitude;
    if (radius <= 5.0) {
        const double argument = radius - 1.6;
        magnitude = polynomial(argument, kC) / polynomial(argument, kD);
    } else {
        const double argument = radius - 5.0;
        magnitude = polynomial(argument, kE) / polynomial(argument, kF);
    }
    return centered < 0.0 ? -magnitude : magnitude;
}

// compile_scramble, crates/pricing/src/engine/sampling/qmc.rs:348-369: row 0 is
// the MSB unit row; row r keeps the raw Philox bits left of the diagonal.
Scramble compile_scramble(uint64_t seed, uint64_t scramble, uint32_t dimension) {
    Scramble s;
    const uint32_t block = dimension * 32u;
    s.shift = philox_word(seed, scramble, block, 2u);
    s.rows[0] = 0x80000000u;
    for (uint32_t row = 1; row < 32; ++row) {
        const uint32_t raw = philox_word(seed, scramble, block + row, 2u);
        const uint32_t before = 0xffffffffu << (32u - row);
        s.rows[row] = (raw & before) | (1u << (31u - row));
    }
    return s;
}

// ---------------------------------------------------------------- bridge

namespace {

struct Candidate {
    double variance, time;
    uint32_t node, left, right;
};

// IntervalCandidate ordering, bridge.rs:149-160: larger variance first, then
// earlier time, then smaller node.  Returns true when a < b.
bool candidate_less(const Candidate& a, const Candidate& b) {
    const int64_t va = total_key(a.variance), vb = total_key(b.variance);
    if (va != vb) return va < vb;
    const int64_t ta = total_key(a.time), tb = total_key(b.time);
    if (ta != tb) return ta > tb;
    return a.node > b.node;
}

bool interval_candidate(const std::vector<double>& t, uint32_t left, uint32_t right,
                        Candidate& best, bool& any) {
    any = false;
    if (right <= left + 1) return true;
    const double denominator = t[right] - t[left];
    for (uint32_t node = left + 1; node < right; ++node) {
        const double variance = ((t[node] - t[left]) * (t[right] - t[node])) / denominator;
        if (!std::isfinite(variance) || variance <= 0.0) return false;
        Candidate c{variance, t[node], node, left, right};
        if (!any || candidate_less(best, c)) best = c;
        any = true;
    }
    return true;
}

}  // namespace

// BrownianBridgePlan::compile, bridge.rs:177-208,395-467.
bool BridgePlan::compile(const std::vector<double>& node_times) {
    times = node_times;
    instructions.clear();
    inverse_sqrt_dt.clear();
    if (times.size() < 2) return false;
    for (double t : times)
        if (!std::isfinite(t)) return false;
    if (total_key(times[0]) != 0) return false;
    for (size_t i = 0; i + 1 < times.size(); ++i)
        if (!(times[i + 1] > times[i])) return false;
    for (size_t i = 0; i + 1 < times.size(); ++i)
        inverse_sqrt_dt.push_back(1.0 / std::sqrt(times[i + 1] - times[i]));
    const uint32_t terminal = static_cast<uint32_t>(times.size() - 1);
    BridgeInstruction first{};
    first.terminal = true;
    first.node = terminal;
    first.rank = 0;
    first.standard_deviation = std::sqrt(times[terminal]);
    instructions.push_back(first);
    auto cmp = [](const Candidate& a, const Candidate& b) { return candidate_less(a, b); };
    std::priority_queue<Candidate, std::vector<Candidate>, decltype(cmp)> heap(cmp);
    Candidate c;
    bool any;
    if (!interval_candidate(times, 0, terminal, c, any)) return false;
    if (any) heap.push(c);
    uint32_t rank = 1;
    while (!heap.empty()) {
        const Candidate top = heap.top();
        heap.pop();
        const double denominator = times[top.right] - times[top.left];
        BridgeInstruction ins{};
        ins.terminal = false;
        ins.node = top.node;
        ins.left = top.left;
        ins.right = top.right;
        ins.rank = rank++;
        ins.left_weight = (times[top.right] - times[top.node]) / denominator;
        ins.right_weight = (times[top.node] - times[top.left]) / denominator;
        ins.standard_deviation = std::sqrt(top.variance);
        instructions.push_back(ins);
        if (!interval_candidate(times, top.left, top.node, c, any)) return false;
        if (any) heap.push(c);
        if (!interval_candidate(times, top.node, top.right, c, any)) return false;
        if (any) heap.push(c);
    }
    return true;
}

// apply_one_factor, bridge.rs:272-311.
void BridgePlan::apply(const double* normals, double* increments,
                       std::vector<double>& w) const {
    w.assign(times.size(), 0.0);
    for (const auto& ins : instructions) {
        if (ins.terminal) {
            w[ins.node] = ins.standard_deviation * normals[ins.rank];
        } else {
            w[ins.node] = ins.left_weight * w[ins.left] + ins.right_weight * w[ins.right] +
                          ins.standard_deviation * normals[ins.rank];
        }
    }
    for (size_t i = 0; i + 1 < times.size(); ++i)
        increments[i] = (w[i + 1] - w[i]) * inverse_sqrt_dt[i];
}

// reverse_one_factor, bridge.rs:314-363.
void BridgePlan::reverse(const double* increment_adjoints, double* normal_adjoints,
                         std::vector<double>& va) const {
    const size_t n = inverse_sqrt_dt.size();
    va.assign(times.size(), 0.0);
    for (size_t i = 0; i < n; ++i) {
        const double scaled = increment_adjoints[i] * inverse_sqrt_dt[i];
        va[i] -= scaled;
        va[i + 1] += scaled;
    }
    for (size_t i = 0; i < n; ++i) normal_adjoints[i] = 0.0;
    for (auto it = instructions.rbegin(); it != instructions.rend(); ++it) {
        if (it->terminal) {
            normal_adjoints[it->rank] += va[it->node] * it->standard_deviation;
        } else {
            const double adjoint = va[it->node];
            normal_adjoints[it->rank] += adjoint * it->standard_deviation;
            va[it->left] += adjoint * it->left_weight;
            va[it->right] += adjoint * it->right_weight;
        }
    }
}

// --------------------------------------------------------------- moments

// CenteredMoment::from_ordered_values_two_pass, reduction.rs:99-122.
CenteredMoment CenteredMoment::two_pass(const std::vector<double>& values) {
    CenteredMoment m;
    if (values.empty()) return m;
    NeumaierSum s;
    for (double v : values) s.add(v);
    const double mean = s.total() / static_cast<double>(values.size());
    NeumaierSum sq;
    for (double v : values) {
        const double d = v - mean;
        sq.add(d * d);
    }
    m.count = values.size();
    m.mean = mean;
    m.second_moment = sq.total();
    return m;
}

// ----------------------------------------------------------------- curve

// LogLinearDiscountCurve::evaluate, curve.rs:163-200 (binary search under total_cmp).
double Curve::log_discount(double time) const {
    if (time == 0.0) time = 0.0;
    const int64_t key = total_key(time);
    size_t lo = 0, hi = times.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (total_key(times[mid]) < key) lo = mid + 1; else hi = mid;
    }
    if (lo < times.size() && total_key(times[lo]) == key) return logs[lo];
    size_t right = lo < times.size() ? lo : times.size() - 1;
    size_t left = right - 1;
    const double weight = (time - times[left]) / (times[right] - times[left]);
    return logs[left] + weight * (logs[right] - logs[left]);
}

// ------------------------------------------------------------------ grid

// lower_cell, local_variance.rs:629-634.
uint32_t lower_cell(const std::vector<double>& nodes, double value) {
    const int64_t key = total_key(value);
    size_t lo = 0, hi = nodes.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (total_key(nodes[mid]) < key) lo = mid + 1; else hi = mid;
    }
    size_t index;
    if (lo < nodes.size() && total_key(nodes[lo]) == key) index = lo;
    else index = lo == 0 ? 0 : lo - 1;
    return static_cast<uint32_t>(std::min(index, nodes.size() - 2));
}

// interpolate + interpolate_in_cells, local_variance.rs:273-383.
bool Grid::interpolate(double time, double log_moneyness, Interpolation& out) const {
    if (!std::isfinite(time) || time < t[0] || time > t.back()) return false;
    if (!std::isfinite(log_moneyness)) return false;
    double xv = log_moneyness;
    out.in_range = true;
    if (log_moneyness < x[0]) {
        xv = x[0];
        out.in_range = false;
    } else if (log_moneyness > x.back()) {
        xv = x.back();
        out.in_range = false;
    }
    const uint32_t tc = lower_cell(t, time);
    const uint32_t xc = lower_cell(x, xv);
    const double tw = (time - t[tc]) / (t[tc + 1] - t[tc]);
    const double xw = (xv - x[xc]) / (x[xc + 1] - x[xc]);
    const uint32_t n = nx();
    const size_t row = static_cast<size_t>(tc) * n;
    const size_t next = row + n;
    const double lower = v[row + xc] * (1.0 - xw) + v[row + xc + 1] * xw;
    const double upper = v[next + xc] * (1.0 - xw) + v[next + xc + 1] * xw;
    out.value = lower * (1.0 - tw) + upper * tw;
    out.time_cell = tc;
    out.x_cell = xc;
    out.time_weight = tw;
    out.x_weight = xw;
    return true;
}

// interpolation_log_moneyness_derivative, local_variance.rs:398-414.
double Grid::x_derivative(const Interpolation& in) const {
    if (!in.in_range) return 0.0;
    const uint32_t n = nx();
    const size_t row = static_cast<size_t>(in.time_cell) * n;
    const size_t next = row + n;
    const uint32_t l = in.x_cell;
    const double width = x[l + 1] - x[l];
    const double lower_slope = (v[row + l + 1] - v[row + l]) / width;
    const double upper_slope = (v[next + l + 1] - v[next + l]) / width;
    return lower_slope * (1.0 - in.time_weight) + upper_slope * in.time_weight;
}

// LocalVarianceInterpolation::transpose_accumulate, local_variance.rs:109-124.
void Grid::transpose_accumulate(const Interpolation& in, double seed, double* adjoints) const {
    const uint32_t n = nx();
    const size_t row = static_cast<size_t>(in.time_cell) * n;
    const size_t next = row + n;
    const uint32_t left = in.x_cell;
    const uint32_t right = std::min(left + 1, n - 1);
    const double tl = 1.0 - in.time_weight, tr = in.time_weight;
    const double xl = 1.0 - in.x_weight, xr = in.x_weight;
    adjoints[row + left] += seed * tl * xl;
    adjoints[row + right] += seed * tl * xr;
    adjoints[next + left] += seed * tr * xl;
    adjoints[next + right] += seed * tr * xr;
}

}  // namespace oracle

namespace oracle {

// ------------------------------------------------- SSVI -> Dupire grid

namespace {

double endpoint_derivative(double aw, double nw, double as, double ns) {
    double d = ((2.0 * aw + nw) * as - aw * ns) / (aw + nw);
    auto sg = [](double v) { return std::signbit(v) ? -1.0 : 1.0; };  // f64::signum (non-NaN)
    if (sg(d) != sg(as)) {
        d = 0.0;
    } else if (sg(as) != sg(ns) && std::fabs(d) > 3.0 * std::fabs(as)) {
        d = 3.0 * as;
    }
    return d;
}

}  // namespace

// pchip_derivatives, crates/pricing/src/market/pchip.rs:178-237.
std::vector<double> pchip_derivatives(const std::vector<double>& t, const std::vector<double>& v) {
    const size_t n = t.size();
    std::vector<double> h(n - 1), s(n - 1), d(n, 0.0);
    for (size_t i = 0; i + 1 < n; ++i) {
        h[i] = t[i + 1] - t[i];
        s[i] = (v[i + 1] - v[i]) / h[i];
    }
    if (n == 2) return {s[0], s[0]};
    auto sg = [](double x) { return std::signbit(x) ? -1.0 : 1.0; };
    d[0] = endpoint_derivative(h[0], h[1], s[0], s[1]);
    for (size_t i = 1; i + 1 < n; ++i) {
        const double l = s[i - 1], r = s[i];
        if (l == 0.0 || r == 0.0 || sg(l) != sg(r)) {
            d[i] = 0.0;
        } else {
            const double lw = h[i - 1], rw = h[i];
            const double w1 = 2.0 * rw + lw;
            const double w2 = rw + 2.0 * lw;
            d[i] = (w1 + w2) / (w1 / l + w2 / r);
        }
    }
    const size_t last = n - 2;
    d[n - 1] = endpoint_derivative(h[last], h[last - 1], s[last], s[last - 1]);
    return d;
}

// ThetaPchip::evaluate, crates/pricing/src/market/pchip.rs:111-176.
void pchip_evaluate(const std::vector<double>& t, const std::vector<double>& v,
                    const std::vector<double>& d, double slope, double time, double& theta,
                    double& derivative) {
    if (time == 0.0) time = 0.0;
    if (time < t[0]) {
        derivative = v[0] / t[0];
        theta = time * derivative;
        return;
    }
    const int64_t key = total_key(time);
    size_t lo = 0, hi = t.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (total_key(t[mid]) < key) lo = mid + 1; else hi = mid;
    }
    if (lo < t.size() && total_key(t[lo]) == key) {
        theta = v[lo];
        derivative = d[lo];
        return;
    }
    if (lo < t.size()) {
        const size_t right = lo, left = lo - 1;
        const double width = t[right] - t[left];
        const double sc = (time - t[left]) / width;
        const double sc2 = sc * sc;
        const double sc3 = sc2 * sc;
        const double h00 = 2.0 * sc3 - 3.0 * sc2 + 1.0;
        const double h10 = sc3 - 2.0 * sc2 + sc;
        const double h01 = -2.0 * sc3 + 3.0 * sc2;
        const double h11 = sc3 - sc2;
        theta = h00 * v[left] + h10 * width * d[left] + h01 * v[right] + h11 * width * d[right];
        const double d00 = (6.0 * sc2 - 6.0 * sc) / width;
        const double d10 = 3.0 * sc2 - 4.0 * sc + 1.0;
        const double d01 = (-6.0 * sc2 + 6.0 * sc) / width;
        const double d11 = 3.0 * sc2 - 2.0 * sc;
        derivative = d00 * v[left] + d10 * d[left] + d01 * v[right] + d11 * d[right];
        return;
    }
    const size_t last = t.size() - 1;
    theta = v[last] + slope * (time - t[last]);
    derivative = slope;
}

// LocalVarianceGrid::from_surface over a StandardSsvi power-law surface,
// crates/pricing/src/market/local_variance.rs:149-206 with
// crates/pricing/src/market/ssvi.rs:121-176,226-273,410-479.
// Returns the repair count, or -1 on a surface error.
int ssvi_grid(const std::vector<double>& theta_t, const std::vector<double>& theta_v,
              double slope, double rho, double eta, double gamma, const std::vector<double>& tn,
              const std::vector<double>& xn, double floor, double cap, std::vector<double>& out) {
    const std::vector<double> pd = pchip_derivatives(theta_t, theta_v);
    out.assign(tn.size() * xn.size(), 0.0);
    int repairs = 0;
    for (size_t i = 0; i < tn.size(); ++i) {
        const double st = tn[i] == 0.0 ? tn[1] : tn[i];
        double theta, dtheta;
        pchip_evaluate(theta_t, theta_v, pd, slope, st, theta, dtheta);
        const double phi = eta / (std::pow(theta, gamma) * std::pow(1.0 + theta, 1.0 - gamma));
        const double phi_td = -phi * (gamma / theta + (1.0 - gamma) / (1.0 + theta));
        for (size_t j = 0; j < xn.size(); ++j) {
            const double x = xn[j];
            const double y = phi * x;
            const double a = y + rho;
            const double q = std::sqrt(a * a + 1.0 - rho * rho);
            const double shape = 1.0 + rho * y + q;
            const double w = theta * shape / 2.0;
            const double common = rho + a / q;
            const double wk = theta * phi * common / 2.0;
            const double wkk = theta * phi * phi * (1.0 - rho * rho) / (2.0 * q * q * q);
            const double partial = shape / 2.0 + theta * x * phi_td * common / 2.0;
            const double wt = partial * dtheta;
            if (!(w > 0.0) || !std::isfinite(w)) return -1;
            const double u = 1.0 - x * wk / (2.0 * w);
            const double density = u * u - (wk * wk / 4.0) * (1.0 / w + 1.0 / 4.0) + wkk / 2.0;
            if (!std::isfinite(density) || density <= 0.0) return -1;
            const double raw = wt / density;
            double value = raw;
            if (std::isnan(raw)) { value = floor; ++repairs; }
            else if (raw == -INFINITY) { value = floor; ++repairs; }
            else if (raw == INFINITY) { value = cap; ++repairs; }
            else if (raw <= 0.0) { value = floor; ++repairs; }
            else if (raw < floor) { value = floor; ++repairs; }
            else if (raw > cap) { value = cap; ++repairs; }
            out[i * xn.size() + j] = value;
        }
    }
    return repairs;
}

// ---------------------------------------------------------------- surfaces

// PhiSpec::evaluate, crates/pricing/src/market/ssvi.rs:121-176 (power law and
// Heston-like with its small-z series below |z| = 1e-4).
void phi_of(const mcg_surface_desc& d, double theta, double& phi, double& dphi) {
    if (d.kind == MCG_SURFACE_SSVI_POWER_LAW) {
        phi = d.eta / (std::pow(theta, d.gamma) * std::pow(1.0 + theta, 1.0 - d.gamma));
        dphi = -phi * (d.gamma / theta + (1.0 - d.gamma) / (1.0 + theta));
        return;
    }
    const double z = d.lambda * theta;
    if (std::fabs(z) <= 1.0e-4) {
        phi = 0.5 + z * (-1.0 / 6.0 + z * (1.0 / 24.0 + z * (-1.0 / 120.0 +
                                                               z * (1.0 / 720.0 + z * (-1.0 / 5040.0 + z / 40320.0)))));
        const double dz = -1.0 / 6.0 + z * (1.0 / 12.0 + z * (-1.0 / 40.0 + z * (1.0 / 180.0 +
                                                                                  z * (-1.0 / 1008.0 + z / 6720.0))));
        dphi = d.lambda * dz;
        return;
    }
    const double e = std::exp(-z);
    phi = (z - 1.0 + e) / (z * z);
    dphi = d.lambda * (2.0 - z - (z + 2.0) * e) / (z * z * z);
}

// EssviSurface::parameters with interpolate / long_parameters,
// crates/pricing/src/market/essvi.rs:192-240,299-340.
void essvi_parameters(const mcg_surface_desc& d, double time, double p[6]) {
    const double* T = d.slice_times;
    const double* TH = d.slice_thetas;
    const double* PS = d.slice_psis;
    const double* RP = d.slice_rho_psis;
    const size_t n = d.slice_count;
    if (time < T[0]) {
        const double inv = 1.0 / T[0];
        const double scale = time * inv;
        const double q[6] = {scale * TH[0], scale * PS[0], scale * RP[0], TH[0] * inv, PS[0] * inv, RP[0] * inv};
        std::memcpy(p, q, sizeof(q));
        return;
    }
    auto interp = [&](size_t l, size_t r) {
        const double width = T[r] - T[l];
        const double weight = (time - T[l]) / width;
        p[0] = TH[l] + weight * (TH[r] - TH[l]);
        p[1] = PS[l] + weight * (PS[r] - PS[l]);
        p[2] = RP[l] + weight * (RP[r] - RP[l]);
        p[3] = (TH[r] - TH[l]) / width;
        p[4] = (PS[r] - PS[l]) / width;
        p[5] = (RP[r] - RP[l]) / width;
    };
    auto long_end = [&](size_t last) {
        p[0] = TH[last] + d.terminal_theta_slope * (time - T[last]);
        p[1] = PS[last];
        p[2] = RP[last];
        p[3] = d.terminal_theta_slope;
        p[4] = 0.0;
        p[5] = 0.0;
    };
    const int64_t key = total_key(time);
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (total_key(T[mid]) < key) lo = mid + 1; else hi = mid;
    }
    if (lo < n && total_key(T[lo]) == key) {
        if (lo + 1 < n) interp(lo, lo + 1); else long_end(lo);
    } else if (lo < n) {
        interp(lo - 1, lo);
    } else {
        long_end(n - 1);
    }
}

// ImpliedVarianceSurface::total_variance_derivatives of both surfaces:
// StandardSsvi (ssvi.rs:410-479) and evaluate_total_variance (essvi.rs:342-396).
// out = {w, w_k, w_kk, w_t}; false on a non-finite or non-positive result.
bool surface_derivatives(const mcg_surface_desc& d, const std::vector<double>& pd, double time, double k,
                         double out[4]) {
    if (d.kind == MCG_SURFACE_ESSVI) {
        double p[6];
        essvi_parameters(d, time, p);
        const double theta = p[0], psi = p[1], rho_psi = p[2], dtheta = p[3], dpsi = p[4], drho_psi = p[5];
        const double phi = psi / theta;
        const double rho = rho_psi / psi;
        const double rho_d = (drho_psi * psi - rho_psi * dpsi) / (psi * psi);
        const double phi_d = (dpsi * theta - psi * dtheta) / (theta * theta);
        const double y = phi * k;
        const double y_d = k * phi_d;
        const double a = y + rho;
        const double q = std::sqrt(a * a + 1.0 - rho * rho);
        const double q_d = (a * (y_d + rho_d) - rho * rho_d) / q;
        const double shape = 1.0 + rho * y + q;
        const double shape_d = rho_d * y + rho * y_d + q_d;
        out[0] = theta * shape / 2.0;
        out[1] = theta * phi * (rho + a / q) / 2.0;
        out[2] = theta * phi * phi * (1.0 - rho * rho) / (2.0 * q * q * q);
        out[3] = dtheta * shape / 2.0 + theta * shape_d / 2.0;
    } else {
        const std::vector<double> t(d.theta_times, d.theta_times + d.theta_count);
        const std::vector<double> v(d.theta_values, d.theta_values + d.theta_count);
        double theta, dtheta, phi, dphi;
        pchip_evaluate(t, v, pd, d.terminal_theta_slope, time, theta, dtheta);
        phi_of(d, theta, phi, dphi);
        const double rho = d.rho;
        const double y = phi * k;
        const double a = y + rho;
        const double q = std::sqrt(a * a + 1.0 - rho * rho);
        const double shape = 1.0 + rho * y + q;
        const double common = rho + a / q;
        out[0] = theta * shape / 2.0;
        out[1] = theta * phi * common / 2.0;
        out[2] = theta * phi * phi * (1.0 - rho * rho) / (2.0 * q * q * q);
        out[3] = (shape / 2.0 + theta * k * dphi * common / 2.0) * dtheta;
    }
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(out[i])) return false;
    return out[0] > 0.0;
}

// LocalVarianceGrid::from_surface (local_variance.rs:149-206) over any surface
// kind.  Returns the repair count, or -1 on a surface error.
int surface_grid(const mcg_surface_desc& d, const std::vector<double>& tn, const std::vector<double>& xn,
                 double floor, double cap, std::vector<double>& out) {
    std::vector<double> pd;
    if (d.kind != MCG_SURFACE_ESSVI)
        pd = pchip_derivatives(std::vector<double>(d.theta_times, d.theta_times + d.theta_count),
                               std::vector<double>(d.theta_values, d.theta_values + d.theta_count));
    out.assign(tn.size() * xn.size(), 0.0);
    int repairs = 0;
    for (size_t i = 0; i < tn.size(); ++i) {
        const double st = tn[i] == 0.0 ? tn[1] : tn[i];
        for (size_t j = 0; j < xn.size(); ++j) {
            const double x = xn[j];
            double w[4];
            if (!surface_derivatives(d, pd, st, x, w)) return -1;
            // durrleman_density_factor, ssvi.rs:226-273
            const double u = 1.0 - x * w[1] / (2.0 * w[0]);
            const double density = u * u - (w[1] * w[1] / 4.0) * (1.0 / w[0] + 1.0 / 4.0) + w[2] / 2.0;
            if (!std::isfinite(density) || density <= 0.0) return -1;
            const double raw = w[3] / density;
            // classify_local_variance, local_variance.rs:607-627
            double value = raw;
            if (std::isnan(raw) || raw == -INFINITY || raw <= 0.0 || raw < floor) value = floor;
            else if (raw == INFINITY || raw > cap) value = cap;
            if (value != raw || std::isnan(raw)) ++repairs;
            out[i * xn.size() + j] = value;
        }
    }
    return repairs;
}

// piecewise_sinh_log_moneyness_nodes, crates/pricing/src/market/local_variance.rs:417-478.
std::vector<double> piecewise_sinh_nodes(double left, double right, size_t nl, size_t nr,
                                         double ls, double rs) {
    auto ratio = [](double shape, double fraction) {
        return shape == 0.0 ? fraction : std::sinh(shape * fraction) / std::sinh(shape);
    };
    std::vector<double> nodes;
    for (size_t i = 0; i <= nl; ++i) {
        const double fr = static_cast<double>(i) / static_cast<double>(nl);
        nodes.push_back(i == nl ? 0.0 : left * ratio(ls, 1.0 - fr));
    }
    for (size_t i = 1; i <= nr; ++i) {
        const double fr = static_cast<double>(i) / static_cast<double>(nr);
        nodes.push_back(right * ratio(rs, fr));
    }
    return nodes;
}

}  // namespace oracle

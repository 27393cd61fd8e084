// oracle_vegakt.cpp -- test infrastructure: CPU restatement of the VegaKT
// node allocation the engine exports as mcg_vega_kt_project.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU baseline load the oracle.
//
// Follows, from msfmfjt/rust-pricing-library:
//   allocate_local_vol_nodes        crates/pricing/src/engine/risk/local_vol_allocation.rs:108-163
//   project_local_vega_nodes_to_reporting_iv, active_density_domain
//                                   crates/pricing/src/engine/risk/vegakt.rs:856-948
//   ReportingIvBasis::interpolate / project_weight / transpose_accumulate
//                                   vegakt.rs:364-377,512-570, reporting_*_interval :1523-1556
//   analytic_call_density_row_from_surface  vegakt.rs:90-123
//   ReportingIvSurface::total_variance_derivatives, lower_cell, interpolation_weight
//                                   crates/pricing/src/engine/processes/local_vol_valuation.rs:56-138
//   evaluate_forward_call / durrleman_density_factor
//                                   crates/pricing/src/market/ssvi.rs:226-320
//   standard_normal_pdf             crates/pricing-numerics/src/normal.rs:4-6
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/mcg.h"
#include "oracle_core.h"

namespace oracle {
namespace {

constexpr double kPi = 3.141592653589793;

uint64_t bits_of(double v) {
    uint64_t b;
    std::memcpy(&b, &v, sizeof(b));
    return b;
}

// lower_cell: binary search under total_cmp; Ok(i) -> min(i, n - 2), Err(i) -> min(max(i - 1, 0), n - 2).
size_t lower_cell(const double* nodes, size_t n, double value) {
    const int64_t key = total_key(value);
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (total_key(nodes[mid]) < key) lo = mid + 1; else hi = mid;
    }
    if (lo < n && total_key(nodes[lo]) == key) return std::min(lo, n - 2);
    return std::min(lo == 0 ? size_t{0} : lo - 1, n - 2);
}

double interpolation_weight(double left, double right, double value) {
    if (bits_of(value) == bits_of(right)) return 1.0;
    return (value - left) / (right - left);
}

struct Derivs {
    double w, wk, wkk, wt;
};

Derivs reporting_surface(const mcg_vega_kt_basis& b, double time, double k) {
    const size_t nm = b.maturity_count, nx = b.log_moneyness_count;
    const double* T = b.maturity_nodes;
    const double* X = b.log_moneyness_nodes;
    const size_t ti = lower_cell(T, nm, time);
    const double x = std::min(std::max(k, X[0]), X[nx - 1]);
    const size_t xi = lower_cell(X, nx, x);
    auto value = [&](size_t i, size_t j) {
        const double vol = b.implied_volatilities[i * nx + j];
        return T[i] * vol * vol;
    };
    const double tw = interpolation_weight(T[ti], T[ti + 1], time);
    const double xw = interpolation_weight(X[xi], X[xi + 1], x);
    const double w00 = value(ti, xi), w01 = value(ti, xi + 1);
    const double w10 = value(ti + 1, xi), w11 = value(ti + 1, xi + 1);
    const double lower = w00 * (1.0 - xw) + w01 * xw;
    const double upper = w10 * (1.0 - xw) + w11 * xw;
    Derivs d;
    d.w = lower * (1.0 - tw) + upper * tw;
    d.wt = (upper - lower) / (T[ti + 1] - T[ti]);
    d.wk = ((w01 - w00) * (1.0 - tw) + (w11 - w10) * tw) / (X[xi + 1] - X[xi]);
    d.wkk = 0.0;
    return d;
}

// analytic call density of the reporting surface at (t, k) for forward F.
bool call_density(const mcg_vega_kt_basis& b, double t, double k, double F, double& out) {
    const Derivs v = reporting_surface(b, t, k);
    const double strike = F * std::exp(k);
    const double root = std::sqrt(v.w);
    const double d2 = -k / root - root / 2.0;
    if (!(v.w > 0.0)) return false;
    const double u = 1.0 - k * v.wk / (2.0 * v.w);
    const double g = u * u - (v.wk * v.wk / 4.0) * (1.0 / v.w + 1.0 / 4.0) + v.wkk / 2.0;
    if (!std::isfinite(g) || g <= 0.0) return false;
    const double pdf = std::exp(-0.5 * d2 * d2) / std::sqrt(2.0 * kPi);
    out = pdf / (strike * root) * g;
    return std::isfinite(out);
}

}  // namespace

// allocate_local_vol_nodes over given node sensitivities (grid rows x nodes).
int vega_kt_project(const double* times, uint32_t nt, const double* xs, uint32_t nx, const double* nodes,
                    uint64_t paths, const mcg_vega_kt_basis* basis, mcg_vega_kt_projection* out) {
    const mcg_vega_kt_basis& b = *basis;
    const size_t nm = b.maturity_count, nr = b.log_moneyness_count;
    // density rows and their active domains
    std::vector<size_t> lo(nm), hi(nm);
    for (size_t m = 0; m < nm; ++m) {
        std::vector<double> dens(nr);
        for (size_t j = 0; j < nr; ++j)
            if (!call_density(b, b.maturity_nodes[m], b.log_moneyness_nodes[j], b.forwards[m], dens[j]))
                return MCG_ERR_MARKET;
        double mx = 0.0;  // maximum_positive_density: fold of f64::max from 0
        for (double d : dens) mx = std::max(mx, d);
        if (!(mx > 0.0)) return MCG_ERR_MARKET;
        size_t fwd = 0;
        double best = std::fabs(b.log_moneyness_nodes[0]);
        for (size_t j = 1; j < nr; ++j)
            if (std::fabs(b.log_moneyness_nodes[j]) < best) {
                best = std::fabs(b.log_moneyness_nodes[j]);
                fwd = j;
            }
        auto ok = [&](double d) { return d / mx >= b.relative_density_threshold; };
        if (!ok(dens[fwd])) return MCG_ERR_MARKET;
        size_t s = fwd, e = fwd;
        while (s > 0 && ok(dens[s - 1])) --s;
        while (e + 1 < nr && ok(dens[e + 1])) ++e;
        if (e >= nx) return MCG_ERR_INVALID_ARGUMENT;
        lo[m] = s;
        hi[m] = e;
    }
    std::vector<NeumaierSum> buckets(nm * nr);
    NeumaierSum initial, residual_sum, left_sum, right_sum, all;
    uint64_t left_count = 0, right_count = 0;
    for (uint32_t r = 0; r < nt; ++r) {
        const double* row = nodes + static_cast<size_t>(r) * nx;
        if (times[r] == 0.0) {
            NeumaierSum s;
            for (uint32_t j = 0; j < nx; ++j) s.add(row[j]);
            initial.add(s.total());
            continue;
        }
        size_t m = 0;
        while (m < nm && bits_of(b.maturity_nodes[m]) != bits_of(times[r])) ++m;
        if (m == nm) return MCG_ERR_INVALID_ARGUMENT;
        // project_local_vega_nodes_to_reporting_iv for this row
        std::vector<double> rb(nm * nr, 0.0);
        NeumaierSum residual, pre;
        double left_w = 0.0, right_w = 0.0;
        size_t ti;  // reporting_interval: Ok(i) -> min(i, n - 2)
        ti = std::min(m, nm - 2);
        const double tw = (times[r] - b.maturity_nodes[ti]) / (b.maturity_nodes[ti + 1] - b.maturity_nodes[ti]);
        for (uint32_t j = 0; j < nx; ++j) {
            const double a = row[j];
            pre.add(a);
            if (j < lo[m] || j > hi[m]) {
                residual.add(a);
                continue;
            }
            // reporting_log_moneyness_interval
            const double x = xs[j];
            const double* X = b.log_moneyness_nodes;
            size_t xi;
            double xw;
            if (x <= X[0]) {
                xi = 0;
                xw = 0.0;
                ++left_count;
                left_w += a;
            } else if (x >= X[nr - 1]) {
                xi = nr - 2;
                xw = 1.0;
                ++right_count;
                right_w += a;
            } else {
                const int64_t key = total_key(x);
                size_t l = 0, h = nr;
                while (l < h) {
                    const size_t mid = (l + h) / 2;
                    if (total_key(X[mid]) < key) l = mid + 1; else h = mid;
                }
                xi = (l < nr && total_key(X[l]) == key) ? std::min(l, nr - 2) : l - 1;
                xw = (x - X[xi]) / (X[xi + 1] - X[xi]);
            }
            const size_t row0 = ti * nr, row1 = row0 + nr;
            const size_t left = xi, right = std::min(xi + 1, nr - 1);
            const double tl = 1.0 - tw, tr = tw, xl = 1.0 - xw, xr = xw;
            rb[row0 + left] += a * tl * xl;
            rb[row0 + right] += a * tl * xr;
            rb[row1 + left] += a * tr * xl;
            rb[row1 + right] += a * tr * xr;
        }
        for (size_t q = 0; q < rb.size(); ++q) buckets[q].add(rb[q]);
        residual_sum.add(residual.total());
        left_sum.add(left_w);
        right_sum.add(right_w);
        all.add(pre.total());
    }
    NeumaierSum scalar;
    for (size_t q = 0; q < buckets.size(); ++q) {
        out->raw_buckets[q] = buckets[q].total();
        scalar.add(out->raw_buckets[q]);
    }
    out->scalar_vega = scalar.total();
    out->density_excluded = residual_sum.total();
    out->signed_residual = initial.total() + residual_sum.total();  // report.rs:206-216
    out->initial_time = initial.total();
    NeumaierSum whole;
    whole.add(initial.total());
    whole.add(all.total());
    out->pre_projection = whole.total();
    out->left_edge_sensitivity = left_sum.total();
    out->right_edge_sensitivity = right_sum.total();
    out->left_edge_count = left_count * paths;
    out->right_edge_count = right_count * paths;
    return MCG_OK;
}

}  // namespace oracle

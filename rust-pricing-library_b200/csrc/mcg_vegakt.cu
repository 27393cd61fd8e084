// mcg_vegakt.cu -- VegaKT node allocation (host code): the local-vega node
// sensitivities of the positive-time grid rows projected onto the
// reporting-IV buckets.
//
// Per positive-time grid row t (allocate_local_vol_nodes,
// crates/pricing/src/engine/risk/local_vol_allocation.rs:108-163):
//   * the active density domain of maturity t: analytic call densities of the
//     reporting-IV surface at the reporting log-moneyness nodes
//     (vegakt.rs:90-156; the surface is bilinear in total variance,
//     crates/pricing/src/engine/processes/local_vol_valuation.rs:67-123), the
//     domain grown from the node nearest the forward while density / max >=
//     threshold (active_density_domain, vegakt.rs:906-948);
//   * every grid node j of the row: inside the domain (by index, as the
//     reference applies it) its sensitivity is deposited bilinearly on the
//     buckets at (t, x_j) (ReportingIvBasis::project_weight / interpolate /
//     transpose_accumulate, vegakt.rs:364-377,512-570, flat beyond the
//     log-moneyness edges, which are counted); outside it goes to the residual
//     (project_local_vega_nodes_to_reporting_iv, vegakt.rs:856-904).
// The t = 0 row is the initial-time audit.  Sums are Neumaier sums in the
// reference's order.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mcg.h"

namespace mcg {
void set_last_error(const std::string& message);
}

namespace {

struct Neumaier {
    double sum = 0.0, corr = 0.0;
    void add(double v) {
        const double t = sum + v;
        if (std::fabs(sum) >= std::fabs(v)) corr += (sum - t) + v;
        else corr += (v - t) + sum;
        sum = t;
    }
    double total() const { return sum + corr; }
};

mcg_status vk_fail(mcg_status status, const std::string& message) {
    mcg::set_last_error(message);
    return status;
}

bool increasing(const double* v, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) {
        if (!std::isfinite(v[i])) return false;
        if (i && !(v[i] > v[i - 1])) return false;
    }
    return true;
}

// lower_cell under total_cmp (local_vol_valuation.rs:125-130): the node's own
// cell on an exact match, the last cell at the right end.
uint32_t lower_cell(const double* nodes, uint32_t n, double value) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (nodes[mid] < value) lo = mid + 1; else hi = mid;
    }
    if (lo < n && nodes[lo] == value) return std::min(lo, n - 2);
    return std::min(lo == 0 ? 0u : lo - 1, n - 2);
}

double weight_in(double left, double right, double value) {
    return value == right ? 1.0 : (value - left) / (right - left);
}

// Total variance derivatives of the reporting-IV surface: total variance
// T sigma^2 bilinear between the basis nodes (x clamped), the second
// x-derivative zero.
void reporting_variance(const mcg_vega_kt_basis& b, double t, double k, double& w, double& wk, double& wkk,
                        double& wt) {
    const uint32_t nm = b.maturity_count, nx = b.log_moneyness_count;
    const double* T = b.maturity_nodes;
    const double* X = b.log_moneyness_nodes;
    const uint32_t ti = lower_cell(T, nm, t);
    const double x = std::min(std::max(k, X[0]), X[nx - 1]);
    const uint32_t xi = lower_cell(X, nx, x);
    auto tv = [&](uint32_t i, uint32_t j) {
        const double s = b.implied_volatilities[i * nx + j];
        return T[i] * s * s;
    };
    const double tw = weight_in(T[ti], T[ti + 1], t);
    const double xw = weight_in(X[xi], X[xi + 1], x);
    const double w00 = tv(ti, xi), w01 = tv(ti, xi + 1), w10 = tv(ti + 1, xi), w11 = tv(ti + 1, xi + 1);
    const double lower = w00 * (1.0 - xw) + w01 * xw;
    const double upper = w10 * (1.0 - xw) + w11 * xw;
    w = lower * (1.0 - tw) + upper * tw;
    wt = (upper - lower) / (T[ti + 1] - T[ti]);
    wk = ((w01 - w00) * (1.0 - tw) + (w11 - w10) * tw) / (X[xi + 1] - X[xi]);
    wkk = 0.0;
}

}  // namespace

extern "C" mcg_status mcg_vega_kt_project(const double* grid_time_nodes, uint32_t time_count,
                                          const double* grid_log_moneyness_nodes, uint32_t log_moneyness_count,
                                          const double* node_sensitivities, uint64_t evaluated_paths,
                                          const mcg_vega_kt_basis* basis, mcg_vega_kt_projection* out) {
    if (!grid_time_nodes || !grid_log_moneyness_nodes || !node_sensitivities || !basis || !out || time_count < 2 ||
        log_moneyness_count < 2)
        return vk_fail(MCG_ERR_INVALID_ARGUMENT, "VegaKT projection inputs");
    const mcg_vega_kt_basis& b = *basis;
    const uint32_t nm = b.maturity_count, nr = b.log_moneyness_count, nx = log_moneyness_count;
    if (!b.maturity_nodes || !b.log_moneyness_nodes || !b.implied_volatilities || !b.forwards || nm < 2 || nr < 2)
        return vk_fail(MCG_ERR_INVALID_ARGUMENT, "reporting basis needs two maturities and two log-moneyness nodes");
    if (!increasing(b.maturity_nodes, nm) || !increasing(b.log_moneyness_nodes, nr) ||
        !increasing(grid_log_moneyness_nodes, nx))
        return vk_fail(MCG_ERR_INVALID_ARGUMENT, "reporting or grid nodes are not finite and increasing");
    for (uint32_t i = 0; i < nm * nr; ++i)
        if (!(b.implied_volatilities[i] > 0.0) || !std::isfinite(b.implied_volatilities[i]))
            return vk_fail(MCG_ERR_INVALID_ARGUMENT, "reporting implied volatilities must be positive");
    if (!(b.relative_density_threshold > 0.0) || b.relative_density_threshold > 1.0)
        return vk_fail(MCG_ERR_INVALID_ARGUMENT, "relative_density_threshold must lie in (0, 1]");
    if (out->bucket_capacity < nm * nr || !out->raw_buckets)
        return vk_fail(MCG_ERR_INVALID_ARGUMENT, "bucket_capacity");
    for (uint64_t i = 0; i < static_cast<uint64_t>(time_count) * nx; ++i)
        if (!std::isfinite(node_sensitivities[i]))
            return vk_fail(MCG_ERR_INVALID_ARGUMENT, "node sensitivities must be finite");

    // Active density domain of every maturity (analytic_call_density_row_from_surface).
    std::vector<uint32_t> dom_lo(nm), dom_hi(nm);
    for (uint32_t m = 0; m < nm; ++m) {
        const double t = b.maturity_nodes[m], F = b.forwards[m];
        if (!(t > 0.0) || !(F > 0.0) || !std::isfinite(F))
            return vk_fail(MCG_ERR_INVALID_ARGUMENT, "density maturity and forward must be positive");
        std::vector<double> dens(nr);
        for (uint32_t j = 0; j < nr; ++j) {
            const double k = b.log_moneyness_nodes[j];
            double w, wk, wkk, wt;
            reporting_variance(b, t, k, w, wk, wkk, wt);
            const double strike = F * std::exp(k);
            const double root = std::sqrt(w);
            const double d2 = -k / root - root / 2.0;
            // durrleman_density_factor (crates/pricing/src/market/ssvi.rs:226-273)
            const double u = 1.0 - k * wk / (2.0 * w);
            const double g = u * u - (wk * wk / 4.0) * (1.0 / w + 1.0 / 4.0) + wkk / 2.0;
            if (!(w > 0.0) || !std::isfinite(g) || g <= 0.0)
                return vk_fail(MCG_ERR_MARKET, "reporting surface has a non-positive variance or density");
            const double pdf = std::exp(-0.5 * d2 * d2) / std::sqrt(2.0 * 3.141592653589793);  // standard_normal_pdf
            dens[j] = pdf / (strike * root) * g;
        }
        double mx = 0.0;
        for (double d : dens) mx = std::max(mx, d);
        if (!(mx > 0.0)) return vk_fail(MCG_ERR_MARKET, "no positive call density");
        uint32_t fwd = 0;
        for (uint32_t j = 1; j < nr; ++j)
            if (std::fabs(b.log_moneyness_nodes[j]) < std::fabs(b.log_moneyness_nodes[fwd])) fwd = j;
        auto qualifies = [&](double d) { return d / mx >= b.relative_density_threshold; };
        if (!qualifies(dens[fwd])) return vk_fail(MCG_ERR_MARKET, "forward node below the density threshold");
        uint32_t lo = fwd, hi = fwd;
        while (lo > 0 && qualifies(dens[lo - 1])) --lo;
        while (hi + 1 < nr && qualifies(dens[hi + 1])) ++hi;
        if (hi >= nx) return vk_fail(MCG_ERR_INVALID_ARGUMENT, "active density domain beyond the grid nodes");
        dom_lo[m] = lo;
        dom_hi[m] = hi;
    }

    std::vector<Neumaier> buckets(static_cast<size_t>(nm) * nr);
    Neumaier residual, pre, initial, left_s, right_s;
    uint64_t left_n = 0, right_n = 0;
    const double* X = b.log_moneyness_nodes;
    for (uint32_t r = 0; r < time_count; ++r) {
        const double t = grid_time_nodes[r];
        const double* row = node_sensitivities + static_cast<size_t>(r) * nx;
        if (t == 0.0) {
            Neumaier s;
            for (uint32_t j = 0; j < nx; ++j) s.add(row[j]);
            initial.add(s.total());
            continue;
        }
        uint32_t m = 0;
        while (m < nm && std::memcmp(&b.maturity_nodes[m], &t, sizeof(double)) != 0) ++m;
        if (m == nm)
            return vk_fail(MCG_ERR_INVALID_ARGUMENT,
                           "grid time " + std::to_string(t) + " is not a reporting maturity (density row)");
        // reporting_interval: the maturity's own cell, the last one at the right end
        const uint32_t ti = std::min(m, nm - 2);
        const double tw = (t - b.maturity_nodes[ti]) / (b.maturity_nodes[ti + 1] - b.maturity_nodes[ti]);
        std::vector<double> rb(static_cast<size_t>(nm) * nr, 0.0);
        Neumaier row_res, row_pre;
        double row_left = 0.0, row_right = 0.0;  // ReportingIvProjectionStats: plain sums within a row
        uint64_t row_ln = 0, row_rn = 0;
        for (uint32_t j = 0; j < nx; ++j) {
            const double a = row[j];
            row_pre.add(a);
            if (j < dom_lo[m] || j > dom_hi[m]) {
                row_res.add(a);
                continue;
            }
            const double x = grid_log_moneyness_nodes[j];
            uint32_t xi;
            double xw;
            if (x <= X[0]) {
                xi = 0;
                xw = 0.0;
                ++row_ln;
                row_left += a;
            } else if (x >= X[nr - 1]) {
                xi = nr - 2;
                xw = 1.0;
                ++row_rn;
                row_right += a;
            } else {
                xi = lower_cell(X, nr, x);
                xw = (x - X[xi]) / (X[xi + 1] - X[xi]);
            }
            const uint32_t r0 = ti * nr, r1 = r0 + nr;
            const uint32_t left = xi, right = std::min(xi + 1, nr - 1);
            const double tl = 1.0 - tw, tr = tw, xl = 1.0 - xw, xr = xw;
            rb[r0 + left] += a * tl * xl;
            rb[r0 + right] += a * tl * xr;
            rb[r1 + left] += a * tr * xl;
            rb[r1 + right] += a * tr * xr;
        }
        for (size_t q = 0; q < rb.size(); ++q) buckets[q].add(rb[q]);
        residual.add(row_res.total());
        pre.add(row_pre.total());
        left_s.add(row_left);
        right_s.add(row_right);
        left_n += row_ln;
        right_n += row_rn;
    }
    Neumaier scalar;
    for (size_t q = 0; q < buckets.size(); ++q) {
        out->raw_buckets[q] = buckets[q].total();
        scalar.add(out->raw_buckets[q]);
    }
    out->scalar_vega = scalar.total();
    out->density_excluded = residual.total();
    out->signed_residual = initial.total() + residual.total();
    out->initial_time = initial.total();
    Neumaier all;
    all.add(initial.total());
    all.add(pre.total());
    out->pre_projection = all.total();
    out->left_edge_sensitivity = left_s.total();
    out->right_edge_sensitivity = right_s.total();
    out->left_edge_count = left_n * evaluated_paths;
    out->right_edge_count = right_n * evaluated_paths;
    return MCG_OK;
}

// oracle_multi.cpp -- correlated multi-asset Monte Carlo of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY: the oracle the CUDA engine is compared against.
// It restates MultiAssetPricingPlan (msfmfjt/rust-pricing-library, paths
// relative to that project) for Black--Scholes and local-volatility assets:
//   compile        crates/pricing/src/engine/multi_asset/compile.rs:200-470
//   shocks, paths  crates/pricing/src/engine/multi_asset/path.rs:24-200
//   run            crates/pricing/src/engine/multi_asset/evaluate.rs:92-300
//   Cholesky       crates/pricing-numerics/src/correlation.rs:61-180
//   products       crates/pricing/src/product/multi_asset.rs:77-246
// with the reference's fixed-block executor statistics.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../include/mcg.h"
#include "oracle_core.h"

namespace oracle {
namespace {

struct Failure {
    int code = MCG_OK;
    uint32_t step = 0;
    double value = 0.0;
};

uint64_t mbits(double v) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
}

// CorrelationFactor::compile: unpivoted lower Cholesky of a PSD matrix with
// zero pivots (tolerances 1e-12) left as zero columns.
bool cholesky(const double* raw, uint32_t n, std::vector<double>& lower) {
    const double tol = 1e-12;
    std::vector<double> c(raw, raw + static_cast<size_t>(n) * n);
    for (uint32_t i = 0; i < n; ++i) {
        if (std::fabs(raw[i * n + i] - 1.0) > tol) return false;
        c[i * n + i] = 1.0;
        for (uint32_t j = i + 1; j < n; ++j) {
            if (std::fabs(raw[i * n + j] - raw[j * n + i]) > tol) return false;
            const double avg = (raw[i * n + j] + raw[j * n + i]) * 0.5;
            if (!(avg >= -1.0 && avg <= 1.0)) return false;
            c[i * n + j] = avg;
            c[j * n + i] = avg;
        }
    }
    double scale = 1.0;
    for (uint32_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (uint32_t j = 0; j < n; ++j) s = s + std::fabs(c[i * n + j]);
        scale = std::max(scale, s);
    }
    const double psd = std::max(tol, tol * scale), zero = std::max(tol, tol * scale);
    lower.assign(static_cast<size_t>(n) * n, 0.0);
    for (uint32_t j = 0; j < n; ++j) {
        double sum = 0.0;
        for (uint32_t k = 0; k < j; ++k) sum += lower[j * n + k] * lower[j * n + k];
        const double pivot = c[j * n + j] - sum;
        if (!std::isfinite(pivot) || pivot < -psd) return false;
        if (pivot > zero) lower[j * n + j] = std::sqrt(pivot);
        for (uint32_t i = j + 1; i < n; ++i) {
            double s2 = 0.0;
            for (uint32_t k = 0; k < j; ++k) s2 += lower[i * n + k] * lower[j * n + k];
            const double residual = c[i * n + j] - s2;
            if (pivot > zero) {
                lower[i * n + j] = residual / lower[j * n + j];
            } else if (!std::isfinite(residual) || std::fabs(residual) > zero) {
                return false;
            }
        }
    }
    return true;
}

struct Asset {
    int model;
    double spot, vol;
    std::vector<double> fwd;  // forward normalisers on the common grid
    Grid grid;
};

struct Multi {
    uint32_t n = 0, steps = 0;
    std::vector<double> times;
    std::vector<Asset> assets;
    std::vector<std::vector<double>> lower;  // per correlation entry
    std::vector<uint32_t> step_entry;
    int engine;
    uint64_t seed, units;
    uint32_t scrambles;
    uint64_t block = 4096;
    bool antithetic, bridge_on;
    BridgePlan bridge;
    std::vector<Scramble> scr;  // scramble-major, dimension-minor
    std::vector<uint32_t> dirs;
    uint32_t dimension = 0;
    int product, side;
    double strike, notional, smoothing, df;
    std::vector<double> weights, scales;
};

double forward_of(const Curve& r, const Curve& q, double spot, double t) {
    return spot * std::exp(q.log_discount(t) - r.log_discount(t));
}

bool build(const mcg_multi_asset_desc* d, Multi& m) {
    if (!d || d->abi_version != MCG_ABI_VERSION || d->asset_count == 0 || d->asset_count > MCG_MAX_ASSETS)
        return false;
    m.n = d->asset_count;
    Curve rc;
    rc.set(d->discount_curve.times, d->discount_curve.discount_factors, d->discount_curve.pillar_count);
    const double horizon = d->expiry;
    // time grid: expiry, correlation changes, grid nodes up to the horizon, substeps
    std::vector<double> events{horizon};
    for (uint32_t k = 0; k < d->correlation_count; ++k) {
        const double t = d->correlation_times[k];
        if (t > 0.0 && t < horizon) events.push_back(t);
    }
    for (uint32_t i = 0; i < m.n; ++i) {
        const mcg_asset_desc& a = d->assets[i];
        if (a.model == MCG_MODEL_LOCAL_VOLATILITY)
            for (uint32_t k = 0; k < a.local_variance.time_count; ++k)
                if (a.local_variance.time_nodes[k] <= horizon) events.push_back(a.local_variance.time_nodes[k]);
    }
    std::sort(events.begin(), events.end(), [](double a, double b) { return total_key(a) < total_key(b); });
    events.erase(std::unique(events.begin(), events.end(), [](double a, double b) { return mbits(a) == mbits(b); }),
                 events.end());
    if (mbits(events[0]) != 0) events.insert(events.begin(), 0.0);
    m.times = {0.0};
    for (size_t i = 0; i + 1 < events.size(); ++i) {
        const double left = events[i], right = events[i + 1];
        if (right <= left) continue;
        const double interval = right - left;
        double sf = std::ceil(interval / d->maximum_step);
        const size_t steps = sf < 1.0 ? 1 : static_cast<size_t>(sf);
        const double sub = interval / static_cast<double>(steps);
        for (size_t k = 1; k < steps; ++k) m.times.push_back(left + sub * static_cast<double>(k));
        m.times.push_back(right);
    }
    m.steps = static_cast<uint32_t>(m.times.size() - 1);
    for (uint32_t i = 0; i < m.n; ++i) {
        const mcg_asset_desc& a = d->assets[i];
        Asset as;
        as.model = a.model;
        as.spot = a.spot;
        as.vol = a.volatility;
        Curve qc;
        qc.set(a.dividend_curve.times, a.dividend_curve.discount_factors, a.dividend_curve.pillar_count);
        for (double t : m.times) as.fwd.push_back(forward_of(rc, qc, a.spot, t));
        if (a.model == MCG_MODEL_LOCAL_VOLATILITY) {
            const auto& g = a.local_variance;
            as.grid.t.assign(g.time_nodes, g.time_nodes + g.time_count);
            as.grid.x.assign(g.log_moneyness_nodes, g.log_moneyness_nodes + g.log_moneyness_count);
            as.grid.v.assign(g.values, g.values + static_cast<size_t>(g.time_count) * g.log_moneyness_count);
            as.grid.floor = g.floor;
            as.grid.cap = g.cap;
        }
        m.assets.push_back(as);
    }
    // correlation: Cholesky per entry, the entry of each interval's start
    for (uint32_t k = 0; k < d->correlation_count; ++k) {
        std::vector<double> l;
        if (!cholesky(d->correlations + static_cast<size_t>(k) * m.n * m.n, m.n, l)) return false;
        m.lower.push_back(l);
    }
    for (uint32_t s = 0; s < m.steps; ++s) {
        uint32_t e = 0;
        while (e < d->correlation_count && d->correlation_times[e] <= m.times[s]) ++e;
        if (e == 0) return false;
        m.step_entry.push_back(e - 1);
    }
    m.engine = d->engine;
    m.seed = d->master_seed;
    m.units = d->sampling_units;
    m.scrambles = d->scramble_count;
    m.antithetic = d->antithetic != 0;
    m.bridge_on = d->brownian_bridge != 0;
    if (d->reduction_block_size) m.block = d->reduction_block_size;
    if (m.bridge_on && !m.bridge.compile(m.times)) return false;
    m.dimension = m.n * m.steps;
    if (m.engine == MCG_ENGINE_RQMC) {
        if (m.dimension > d->sobol_dimension_count) return false;
        m.dirs.assign(d->sobol_directions, d->sobol_directions + static_cast<size_t>(m.dimension) * 32u);
        for (uint32_t s = 0; s < m.scrambles; ++s)
            for (uint32_t dim = 0; dim < m.dimension; ++dim) m.scr.push_back(compile_scramble(m.seed, s, dim));
    }
    m.product = d->product;
    m.side = d->side;
    m.strike = d->strike;
    m.notional = d->notional;
    m.smoothing = d->smoothing_half_width;
    m.df = std::exp(rc.log_discount(d->payment_time));
    if (d->weights) m.weights.assign(d->weights, d->weights + m.n);
    m.scales.assign(d->scales, d->scales + m.n);
    return true;
}

// The compact-C2 maximum and minimum (smoothing.rs), value only.
double smooth_positive(double h, double input) {
    if (input <= -h) return 0.0;
    if (input >= h) return input;
    const double full = 2.0 * h;
    double u;
    if (std::isfinite(full)) u = (input + h) / full;
    else if (input < 0.0) u = 0.5 * ((input + h) / h);
    else u = 0.5 * (input / h + 1.0);
    const double u2 = u * u, u4 = u2 * u2;
    const double scaled = 2.0 * h * u4;
    const double poly = 2.5 + u * (-3.0 + u);
    return std::isnormal(scaled) ? scaled * poly : (2.0 * u4 * poly) * h;
}
double smooth_max(double h, double l, double r) {
    const double diff = l - r;
    if (diff >= h) return l;
    if (diff <= -h) return r;
    return r + smooth_positive(h, diff);
}
double smooth_min(double h, double l, double r) {
    const double diff = l - r;
    if (diff >= h) return r;
    if (diff <= -h) return l;
    return l - smooth_positive(h, diff);
}

// shocks (path.rs:24-98): independent normals per factor, bridged, then correlated.
void shocks(const Multi& m, uint32_t scramble, uint64_t point, std::vector<double>& out) {
    const uint32_t n = m.n, steps = m.steps;
    const bool rank_major = m.engine == MCG_ENGINE_RQMC && m.bridge_on;
    std::vector<double> ind(static_cast<size_t>(n) * steps), tmp(steps), scratch;
    for (uint32_t f = 0; f < n; ++f) {
        for (uint32_t s = 0; s < steps; ++s) {
            const uint32_t dim = rank_major ? s * n + f : f * steps + s;
            double z;
            if (m.engine == MCG_ENGINE_PSEUDO) {
                z = philox_normal(m.seed, point, dim, 0);
            } else {
                const uint32_t w = m.scr[static_cast<size_t>(scramble) * m.dimension + dim].apply(
                    sobol_word(m.dirs.data() + static_cast<size_t>(dim) * 32u, static_cast<uint32_t>(point)));
                z = inverse_standard_normal(open_unit_interval(w));
            }
            tmp[s] = z;
        }
        if (m.bridge_on) {
            std::vector<double> inc(steps);
            m.bridge.apply(tmp.data(), inc.data(), scratch);
            tmp = inc;
        }
        for (uint32_t s = 0; s < steps; ++s) ind[static_cast<size_t>(f) * steps + s] = tmp[s];
    }
    out.assign(static_cast<size_t>(n) * steps, 0.0);
    for (uint32_t s = 0; s < steps; ++s) {
        const std::vector<double>& l = m.lower[m.step_entry[s]];
        for (uint32_t i = 0; i < n; ++i) {
            double value = 0.0;
            for (uint32_t k = 0; k <= i; ++k) value += l[i * n + k] * ind[static_cast<size_t>(k) * steps + s];
            out[static_cast<size_t>(i) * steps + s] = value;
        }
    }
}

// paths (path.rs:99-200) and the product's PV on one set of shocks.
bool value(const Multi& m, const std::vector<double>& z, double& pv, Failure& fail) {
    const uint32_t n = m.n, steps = m.steps;
    std::vector<double> terminal(n);
    for (uint32_t i = 0; i < n; ++i) {
        const Asset& a = m.assets[i];
        double f = a.spot;
        for (uint32_t s = 0; s < steps; ++s) {
            const double dt = m.times[s + 1] - m.times[s];
            const double zz = z[static_cast<size_t>(i) * steps + s];
            double next;
            if (a.model == MCG_MODEL_BLACK_SCHOLES) {
                next = f * (a.fwd[s + 1] / a.fwd[s]) * std::exp(-0.5 * a.vol * a.vol * dt + a.vol * std::sqrt(dt) * zz);
            } else {
                Interpolation in;
                const double x = std::log(f / a.fwd[s]);
                if (!a.grid.interpolate(m.times[s], x, in)) {
                    fail = {MCG_ERR_INVALID_SURFACE_QUERY, s, x};
                    return false;
                }
                const double ratio = a.fwd[s + 1] / a.fwd[s];
                next = f * (ratio * std::exp(-0.5 * in.value * dt + std::sqrt(in.value) * std::sqrt(dt) * zz));
            }
            if (!std::isfinite(next) || next <= 0.0) {
                fail = {MCG_ERR_NON_FINITE_STATE, s + 1, next};
                return false;
            }
            f = next;
        }
        terminal[i] = f;
    }
    double w;
    if (m.product == MCG_MULTI_BASKET) {
        w = 0.0;
        for (uint32_t i = 0; i < n; ++i) w = w + (m.weights[i] * terminal[i]) / m.scales[i];
    } else {
        w = terminal[0] / m.scales[0];
        for (uint32_t i = 1; i < n; ++i) {
            const double x = terminal[i] / m.scales[i];
            w = m.smoothing > 0.0 ? smooth_min(m.smoothing, w, x) : (w <= x ? w : x);
        }
    }
    const double intrinsic = m.side == MCG_CALL ? w - m.strike : m.strike - w;
    const double positive = m.smoothing > 0.0 ? smooth_max(m.smoothing, intrinsic, 0.0)
                                              : (intrinsic >= 0.0 ? intrinsic : 0.0);
    const double payoff = m.notional * positive;
    pv = 0.0 + payoff * m.df;
    return true;
}

bool unit(const Multi& m, uint32_t scramble, uint64_t u, double& out, Failure& fail) {
    std::vector<double> z;
    shocks(m, scramble, u, z);
    double a;
    if (!value(m, z, a, fail)) return false;
    if (m.antithetic) {
        for (double& v : z) v = -v;
        double b;
        if (!value(m, z, b, fail)) return false;
        out = (a + b) * 0.5;
    } else {
        out = a;
    }
    return true;
}

bool reduce(const Multi& m, uint32_t scramble, int threads, Statistics& total, mcg_error_record& err) {
    const uint64_t block = m.block;
    const uint64_t nblocks = (m.units + block - 1) / block;
    std::vector<Statistics> res(nblocks);
    std::vector<Failure> fails(nblocks);
    std::vector<uint64_t> funit(nblocks, 0);
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const uint64_t b = next.fetch_add(1);
            if (b >= nblocks) break;
            const uint64_t begin = b * block, end = std::min(m.units, begin + block);
            for (uint64_t u = begin; u < end; ++u) {
                double v;
                if (!unit(m, scramble, u, v, fails[b])) {
                    funit[b] = u;
                    break;
                }
                res[b].add(v);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    for (uint64_t b = 0; b < nblocks; ++b)
        if (fails[b].code != MCG_OK) {
            err.code = fails[b].code;
            err.step = fails[b].step;
            err.sampling_unit = funit[b];
            err.value_bits = mbits(fails[b].value);
            return false;
        }
    std::vector<NeumaierSum> sums;
    std::vector<CenteredMoment> moms;
    for (const auto& r : res) {
        sums.push_back(r.sum);
        moms.push_back(r.moments);
    }
    total.sum = fixed_tree_reduce(sums, NeumaierSum::merged);
    total.moments = fixed_tree_reduce(moms, CenteredMoment::merged);
    return true;
}

}  // namespace
}  // namespace oracle

extern "C" int oracle_multi_asset_price(const mcg_multi_asset_desc* d, mcg_multi_asset_result* r, int threads) {
    using namespace oracle;
    Multi m;
    if (!r || !build(d, m)) return MCG_ERR_INVALID_ARGUMENT;
    std::memset(&r->error, 0, sizeof(r->error));
    Statistics st;
    uint64_t independent;
    if (m.engine == MCG_ENGINE_PSEUDO) {
        if (!reduce(m, 0, threads, st, r->error)) return r->error.code;
        independent = m.units;
    } else {
        std::vector<double> means;
        for (uint32_t s = 0; s < m.scrambles; ++s) {
            Statistics within;
            if (!reduce(m, s, threads, within, r->error)) return r->error.code;
            means.push_back(within.sum.total() / static_cast<double>(m.units));
        }
        st.moments = CenteredMoment::two_pass(means);
        for (double v : means) st.sum.add(v);
        independent = m.scrambles;
    }
    r->price_statistics = {st.sum.sum, st.sum.correction, st.moments.count, st.moments.mean,
                           st.moments.second_moment};
    const double inv = 1.0 / static_cast<double>(independent);
    const double value = st.sum.total() * inv;
    const double var = st.moments.count > 1 ? st.moments.second_moment / static_cast<double>(st.moments.count - 1) : 0.0;
    const double se = std::sqrt(var * inv);
    const double hw = 1.959963984540054 * se;
    r->price = {value, se, value - hw, value + hw, independent};
    r->sampling_variance = var;
    r->independent_sampling_units = independent;
    r->evaluated_paths = m.units * (m.engine == MCG_ENGINE_RQMC ? m.scrambles : 1) * (m.antithetic ? 2 : 1);
    r->time_steps = m.steps;
    r->dimension = m.dimension;
    return MCG_OK;
}

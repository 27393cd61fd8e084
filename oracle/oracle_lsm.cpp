// oracle_lsm.cpp -- Longstaff--Schwartz early exercise of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY: the oracle the CUDA engine is compared against,
// never linked into the engine.  Restates, from msfmfjt/rust-pricing-library
// (paths relative to that project):
//   FeatureScaling::fit                 crates/pricing/src/engine/mc/lsm.rs:537-574
//   PolynomialRegressionModel::predict  lsm.rs:776-790, should_exercise lsm.rs:805-818,2313-2320
//   value_exercise_policy               lsm.rs:1347-1482
//   train_exercise_policy               lsm.rs:1486-1695
//   fit_exercise_decision               lsm.rs:1928-2065
//   fit_polynomial_regression           lsm.rs:2067-2247 (+ evaluate_monomial :2249-2262)
//   fit_cpqr, column norms              lsm.rs:2374-2652
//   collapse_antithetic_values          crates/pricing/src/engine/mc/early_exercise.rs:616-650
//   rqmc_replicate_values               early_exercise.rs:652-712
//   execute_early_exercise(_rqmc)       crates/pricing/src/engine/risk/early_exercise.rs:24-120,251-313
// The path matrices come from oracle_plan.cpp (lsm_spots).  The regression is
// single-threaded, as in the reference.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <cstring>
#include <string>
#include <vector>

#include "../include/mcg.h"
#include "oracle_core.h"

namespace oracle {

int lsm_spots(const mcg_plan_desc* desc, uint32_t domain, int threads, std::vector<double>& spots,
              uint64_t& path_count, mcg_error_record& err, std::vector<double>* brownians = nullptr);
double plan_discount(const mcg_plan_desc* desc, double t);
double plan_forward(const mcg_plan_desc* desc, double t);
int lsm_fixed_policy_risk(const mcg_plan_desc* desc, const uint32_t* stops, const double* df, int threads,
                          mcg_lsm_result* result);
int lsm_lv_fixed_policy_risk(const mcg_plan_desc* desc, const uint32_t* stops, const double* df, int threads,
                             mcg_lsm_result* result);

namespace {

constexpr double kEpsilon = 2.220446049250313e-16;  // f64::EPSILON
constexpr double kNormal95 = 1.959963984540054;
constexpr uint32_t kDomainValuation = 0;
constexpr uint32_t kDomainLsmTrain = 1;

thread_local std::string g_lsm_error;

int lsm_fail(const char* msg) {
    g_lsm_error = msg;
    return MCG_ERR_LSM;
}

struct Scaling {
    double mean = 0.0, variance = 0.0, scale = 0.0, threshold = 0.0;
    bool inactive = false;
};

// FeatureScaling::fit, lsm.rs:537-574.
Scaling fit_scaling(const std::vector<double>& values) {
    NeumaierSum sum;
    double feature_scale = 1.0;
    for (double v : values) {
        sum.add(v);
        feature_scale = std::max(feature_scale, std::fabs(v));
    }
    Scaling s;
    s.mean = sum.total() / static_cast<double>(values.size());
    NeumaierSum sq;
    for (double v : values) {
        const double d = v - s.mean;
        sq.add(d * d);
    }
    s.variance = sq.total() / static_cast<double>(values.size());
    s.scale = std::sqrt(s.variance);
    s.threshold = (64.0 * kEpsilon) * feature_scale;
    s.inactive = s.scale <= s.threshold;
    return s;
}

double column_squared_norm(const std::vector<double>& m, size_t rows, size_t cols, size_t start,
                           size_t c) {
    NeumaierSum n;
    for (size_t r = start; r < rows; ++r) {
        const double v = m[r * cols + c];
        n.add(v * v);
    }
    return n.total();
}

// The scaled two-norm of column_norm, lsm.rs:2615-2650.
double column_norm(const std::vector<double>& m, size_t rows, size_t cols, size_t start, size_t c) {
    double scale = 0.0, ss = 1.0;
    for (size_t r = start; r < rows; ++r) {
        const double v = std::fabs(m[r * cols + c]);
        if (v == 0.0) continue;
        if (scale < v) {
            const double ratio = scale / v;
            ss = 1.0 + ss * (ratio * ratio);
            scale = v;
        } else {
            const double ratio = v / scale;
            ss += ratio * ratio;
        }
    }
    return scale == 0.0 ? 0.0 : scale * std::sqrt(ss);
}

struct Cpqr {
    std::vector<size_t> pivot;
    std::vector<double> diagonal, coefficients;
    double threshold = 0.0, rss = 0.0;
    size_t rank = 0;
};

// fit_cpqr, lsm.rs:2374-2568: Householder QR with column pivoting on the
// largest remaining squared norm (ties to the smaller original column).
bool fit_cpqr(const std::vector<double>& matrix, size_t rows, size_t cols,
              const std::vector<double>& target, double abs_tol, double rel_tol, Cpqr& fit) {
    std::vector<double> qr = matrix, y = target;
    fit.pivot.resize(cols);
    for (size_t c = 0; c < cols; ++c) fit.pivot[c] = c;
    fit.diagonal.clear();
    const size_t dcount = std::min(rows, cols);
    for (size_t p = 0; p < dcount; ++p) {
        size_t selected = p;
        double selected_norm = -1.0;
        for (size_t c = p; c < cols; ++c) {
            const double sn = column_squared_norm(qr, rows, cols, p, c);
            if (sn > selected_norm || (sn == selected_norm && fit.pivot[c] < fit.pivot[selected])) {
                selected = c;
                selected_norm = sn;
            }
        }
        if (selected != p) {
            for (size_t r = 0; r < rows; ++r) std::swap(qr[r * cols + p], qr[r * cols + selected]);
            std::swap(fit.pivot[p], fit.pivot[selected]);
        }
        const double norm = column_norm(qr, rows, cols, p, p);
        if (norm == 0.0) {
            qr[p * cols + p] = 0.0;
            fit.diagonal.push_back(0.0);
            continue;
        }
        const size_t di = p * cols + p;
        const double leading = qr[di];
        const double alpha = leading >= 0.0 ? -norm : norm;
        const double denominator = leading - alpha;
        const double tau = (alpha - leading) / alpha;
        if (!std::isfinite(denominator) || !std::isfinite(tau)) {
            g_lsm_error = "Householder reflector";
            return false;
        }
        qr[di] = alpha;
        for (size_t r = p + 1; r < rows; ++r) qr[r * cols + p] /= denominator;
        for (size_t c = p + 1; c < cols; ++c) {
            NeumaierSum dot;
            dot.add(qr[p * cols + c]);
            for (size_t r = p + 1; r < rows; ++r) dot.add(qr[r * cols + p] * qr[r * cols + c]);
            const double projection = tau * dot.total();
            qr[p * cols + c] -= projection;
            for (size_t r = p + 1; r < rows; ++r) qr[r * cols + c] -= qr[r * cols + p] * projection;
        }
        NeumaierSum td;
        td.add(y[p]);
        for (size_t r = p + 1; r < rows; ++r) td.add(qr[r * cols + p] * y[r]);
        const double tp = tau * td.total();
        y[p] -= tp;
        for (size_t r = p + 1; r < rows; ++r) y[r] -= qr[r * cols + p] * tp;
        fit.diagonal.push_back(std::fabs(alpha));
    }
    const double first = fit.diagonal.empty() ? 0.0 : fit.diagonal[0];
    fit.threshold = std::max(abs_tol, rel_tol * first);
    fit.rank = 0;
    while (fit.rank < fit.diagonal.size() && fit.diagonal[fit.rank] > fit.threshold) ++fit.rank;
    std::vector<double> pc(cols, 0.0);
    for (size_t r = fit.rank; r-- > 0;) {
        NeumaierSum up;
        for (size_t c = r + 1; c < fit.rank; ++c) up.add(qr[r * cols + c] * pc[c]);
        pc[r] = (y[r] - up.total()) / qr[r * cols + r];
        if (!std::isfinite(pc[r])) {
            g_lsm_error = "back substitution";
            return false;
        }
    }
    fit.coefficients.assign(cols, 0.0);
    for (size_t p = 0; p < cols; ++p) fit.coefficients[fit.pivot[p]] = pc[p];
    NeumaierSum rs;
    for (size_t r = 0; r < rows; ++r) {
        NeumaierSum pred;
        for (size_t c = 0; c < cols; ++c) pred.add(matrix[r * cols + c] * fit.coefficients[c]);
        const double res = target[r] - pred.total();
        rs.add(res * res);
    }
    fit.rss = rs.total();
    return true;
}

// evaluate_monomial, lsm.rs:2249-2262, for one feature.
double monomial(double z, uint32_t exponent) {
    double v = 1.0;
    for (uint32_t e = 0; e < exponent; ++e) v *= z;
    return v;
}

struct DateModel {
    mcg_lsm_date_model rec{};
    // PolynomialRegressionModel::predict, lsm.rs:776-790.
    double predict(double x, uint32_t degree) const {
        const double z = rec.feature_inactive ? 0.0 : (x - rec.feature_mean) / rec.feature_scale;
        NeumaierSum p;
        for (uint32_t e = 0; e <= degree; ++e) p.add(monomial(z, e) * rec.coefficients[e]);
        return p.total();
    }
    // ExerciseDecisionModel::should_exercise, lsm.rs:805-818.
    bool exercise(double immediate, double x, uint32_t degree) const {
        return rec.regression && immediate > predict(x, degree);
    }
};

struct Config {
    uint32_t degree;
    double itm_tol, abs_tol, rel_tol;
    uint64_t max_elements;
};

// fit_exercise_decision + fit_polynomial_regression for one date.
int fit_date(const Config& cfg, const double* immediate, const double* spots,
             const std::vector<double>& targets, size_t paths, DateModel& m) {
    std::memset(&m.rec, 0, sizeof(m.rec));
    m.rec.candidate_rows = static_cast<uint32_t>(paths);
    std::vector<double> x, y;
    for (size_t p = 0; p < paths; ++p) {
        if (immediate[p] <= cfg.itm_tol) continue;
        x.push_back(spots[p]);
        y.push_back(targets[p]);
    }
    m.rec.itm_rows = static_cast<uint32_t>(x.size());
    if (x.empty()) return MCG_OK;  // ContinueAll { ZeroItmTrainingPaths }
    if (x.size() > cfg.max_elements) return lsm_fail("ITM feature matrix exceeds max_matrix_elements");
    const Scaling sc = fit_scaling(x);
    m.rec.regression = 1;
    m.rec.feature_mean = sc.mean;
    m.rec.feature_variance = sc.variance;
    m.rec.feature_scale = sc.scale;
    m.rec.zero_scale_threshold = sc.threshold;
    m.rec.feature_inactive = sc.inactive ? 1 : 0;
    std::vector<uint32_t> active;
    for (uint32_t e = 0; e <= cfg.degree; ++e)
        if (e == 0 || !sc.inactive) active.push_back(e);
    const size_t rows = x.size(), cols = active.size();
    if (rows * cols > cfg.max_elements) return lsm_fail("design matrix exceeds max_matrix_elements");
    std::vector<double> design(rows * cols);
    for (size_t r = 0; r < rows; ++r) {
        const double z = sc.inactive ? 0.0 : (x[r] - sc.mean) / sc.scale;
        for (size_t c = 0; c < cols; ++c) design[r * cols + c] = monomial(z, active[c]);
    }
    Cpqr fit;
    if (!fit_cpqr(design, rows, cols, y, cfg.abs_tol, cfg.rel_tol, fit)) return MCG_ERR_LSM;
    m.rec.active_columns = static_cast<uint32_t>(cols);
    m.rec.diagonal_count = static_cast<uint32_t>(fit.diagonal.size());
    m.rec.rank = static_cast<uint32_t>(fit.rank);
    m.rec.rank_threshold = fit.threshold;
    m.rec.residual_sum_squares = fit.rss;
    for (size_t k = 0; k < cols; ++k) m.rec.pivot_order[k] = active[fit.pivot[k]];
    for (size_t k = 0; k < fit.diagonal.size(); ++k) m.rec.diagonal_abs[k] = fit.diagonal[k];
    for (size_t c = 0; c < cols; ++c) m.rec.coefficients[active[c]] = fit.coefficients[c];
    return MCG_OK;
}

// The American payoff graph's output at one date, compile.rs:67-101.
double intrinsic(const mcg_product_desc& pr, double s) {
    const double in = pr.side == MCG_CALL ? s - pr.strike : pr.strike - s;
    return (in >= 0.0 ? in : 0.0) * pr.notional;
}

// Collapses per-path discounted cash flows to sampling-unit values
// (collapse_antithetic_values) or RQMC replicates (rqmc_replicate_values).
std::vector<double> unit_values(const std::vector<double>& cf, bool antithetic, bool rqmc,
                                uint64_t points, uint32_t scrambles) {
    std::vector<double> out;
    if (!rqmc) {
        if (!antithetic) return cf;
        out.resize(cf.size() / 2);
        for (size_t i = 0; i < out.size(); ++i) out[i] = (cf[2 * i] + cf[2 * i + 1]) * 0.5;
        return out;
    }
    const size_t per = static_cast<size_t>(points) * (antithetic ? 2 : 1);
    for (uint32_t s = 0; s < scrambles; ++s) {
        NeumaierSum sum;
        const double* v = cf.data() + static_cast<size_t>(s) * per;
        if (antithetic) {
            for (size_t i = 0; i < points; ++i) sum.add((v[2 * i] + v[2 * i + 1]) * 0.5);
        } else {
            for (size_t i = 0; i < points; ++i) sum.add(v[i]);
        }
        out.push_back(sum.total() / static_cast<double>(points));
    }
    return out;
}

// Backward induction over the training paths (train_exercise_policy,
// lsm.rs:1486-1695): one fitted decision model per date before the last and
// the in-sample value of the training paths under it.
int train_policy(const mcg_plan_desc* desc, const mcg_lsm_desc* lsm, int threads, const std::vector<double>& df,
                 std::vector<DateModel>& models, uint64_t& tp, double& in_sample_value, mcg_error_record& err) {
    const size_t dates = desc->observation_count;
    const mcg_product_desc& pr = desc->products[0];
    const Config cfg{lsm->max_degree, lsm->itm_abs_tolerance, lsm->cpqr_abs_tolerance,
                     lsm->cpqr_rel_tolerance, lsm->max_matrix_elements};
    const bool rqmc = desc->engine == MCG_ENGINE_RQMC;
    mcg_plan_desc train = *desc;
    train.master_seed = lsm->training_seed;
    train.sampling_units = lsm->training_units;
    train.scramble_count = lsm->training_scramble_count;
    train.scramble_begin = 0;
    train.antithetic = lsm->training_antithetic;
    train.brownian_bridge = lsm->training_brownian_bridge;
    std::vector<double> spots;
    tp = 0;
    int rc = lsm_spots(&train, kDomainLsmTrain, threads, spots, tp, err);
    if (rc != MCG_OK) return rc;
    std::vector<double> imm(spots.size());
    for (size_t i = 0; i < spots.size(); ++i) imm[i] = intrinsic(pr, spots[i]);
    std::vector<double> realized(imm.begin() + (dates - 1) * tp, imm.begin() + dates * tp);
    std::vector<uint32_t> stop(tp, static_cast<uint32_t>(dates - 1));
    std::vector<double> targets(tp);
    models.assign(dates - 1, DateModel{});
    for (size_t d = dates - 1; d-- > 0;) {
        for (size_t p = 0; p < tp; ++p) targets[p] = realized[p] * df[stop[p]] / df[d];
        rc = fit_date(cfg, &imm[d * tp], &spots[d * tp], targets, tp, models[d]);
        if (rc != MCG_OK) return rc;
        for (size_t p = 0; p < tp; ++p)
            if (models[d].exercise(imm[d * tp + p], spots[d * tp + p], cfg.degree)) {
                realized[p] = imm[d * tp + p];
                stop[p] = static_cast<uint32_t>(d);
            }
    }
    std::vector<double> in_sample(tp);
    for (size_t p = 0; p < tp; ++p) in_sample[p] = realized[p] * df[stop[p]];
    const std::vector<double> in_units =
        unit_values(in_sample, lsm->training_antithetic != 0, rqmc, lsm->training_units,
                    lsm->training_scramble_count);
    NeumaierSum in_sum;
    for (double v : in_units) in_sum.add(v);
    in_sample_value = in_sum.total() / static_cast<double>(in_units.size());
    return MCG_OK;
}

}  // namespace

// The early-exercise evaluation of mcg_lsm_price on the CPU.
int lsm_price(const mcg_plan_desc* desc, const mcg_lsm_desc* lsm, mcg_lsm_result* out, int threads) {
    g_lsm_error.clear();
    if (!desc || !lsm || !out) return lsm_fail("null argument");
    std::memset(&out->error, 0, sizeof(out->error));
    if (desc->product_count != 1 || desc->products[0].kind != MCG_PRODUCT_AMERICAN)
        return lsm_fail("one American product expected");
    if (lsm->max_degree < 1 || lsm->max_degree > MCG_LSM_MAX_DEGREE) return lsm_fail("max_degree");
    if (lsm->continuation != MCG_CONTINUATION_POLYNOMIAL) return MCG_ERR_UNSUPPORTED;
    const size_t dates = desc->observation_count;
    if (dates < 1 || out->date_capacity < dates || !out->exercise_counts)
        return lsm_fail("date_capacity");
    const mcg_product_desc& pr = desc->products[0];
    const Config cfg{lsm->max_degree, lsm->itm_abs_tolerance, lsm->cpqr_abs_tolerance,
                     lsm->cpqr_rel_tolerance, lsm->max_matrix_elements};
    std::vector<double> df(dates);
    for (size_t d = 0; d < dates; ++d) df[d] = plan_discount(desc, desc->observation_times[d]);
    const bool rqmc = desc->engine == MCG_ENGINE_RQMC;

    // Training phase.
    std::vector<DateModel> models;
    uint64_t tp = 0;
    int rc = train_policy(desc, lsm, threads, df, models, tp, out->in_sample_value, out->error);
    if (rc != MCG_OK) return rc;
    std::vector<double> spots, imm, realized;
    std::vector<uint32_t> stop;

    // Valuation phase.
    uint64_t vp = 0;
    rc = lsm_spots(desc, kDomainValuation, threads, spots, vp, out->error);
    if (rc != MCG_OK) return rc;
    imm.resize(spots.size());
    for (size_t i = 0; i < spots.size(); ++i) imm[i] = intrinsic(pr, spots[i]);
    realized.assign(imm.begin() + (dates - 1) * vp, imm.begin() + dates * vp);
    stop.assign(vp, static_cast<uint32_t>(dates - 1));
    for (size_t d = 0; d + 1 < dates; ++d)
        for (size_t p = 0; p < vp; ++p) {
            if (stop[p] != dates - 1) continue;
            if (models[d].exercise(imm[d * vp + p], spots[d * vp + p], cfg.degree)) {
                realized[p] = imm[d * vp + p];
                stop[p] = static_cast<uint32_t>(d);
            }
        }
    std::vector<double> discounted(vp);
    for (size_t d = 0; d < dates; ++d) out->exercise_counts[d] = 0;
    for (size_t p = 0; p < vp; ++p) {
        out->exercise_counts[stop[p]] += 1;
        discounted[p] = realized[p] * df[stop[p]];
    }
    if (out->stopping_indices && out->stopping_capacity >= vp)
        for (size_t p = 0; p < vp; ++p) out->stopping_indices[p] = stop[p];
    const std::vector<double> values = unit_values(discounted, desc->antithetic != 0, rqmc,
                                                   desc->sampling_units, desc->scramble_count);
    Statistics st;
    for (double v : values) st.sum.add(v);
    st.moments = CenteredMoment::two_pass(values);
    const uint64_t independent = rqmc ? desc->scramble_count : desc->sampling_units;
    const double inv = 1.0 / static_cast<double>(independent);
    const double value = st.sum.total() * inv;
    const double var = st.moments.count > 1
                           ? st.moments.second_moment / static_cast<double>(st.moments.count - 1)
                           : 0.0;
    const double se = std::sqrt(var * inv);
    out->price_statistics = {st.sum.sum, st.sum.correction, st.moments.count, st.moments.mean,
                             st.moments.second_moment};
    out->price = {value, se, value - kNormal95 * se, value + kNormal95 * se, independent};
    out->sampling_variance = var;
    out->estimator_variance = var / static_cast<double>(independent);
    out->training_paths = tp;
    out->valuation_paths = vp;
    out->independent_sampling_units = independent;
    out->date_count = static_cast<uint32_t>(dates);
    if (out->models)
        for (size_t d = 0; d + 1 < dates; ++d) out->models[d] = models[d].rec;
    // Fixed-policy risk: the valuation stopping dates held fixed, Greeks of
    // the discounted exercise values (early_exercise.rs:454-600).
    std::memset(out->risk_components, 0, sizeof(out->risk_components));
    out->delta = out->gamma = out->vega = mcg_estimate{};
    out->bump_delta = out->bump_gamma = out->bump_vega = mcg_estimate{};
    if (desc->request_delta || desc->request_gamma || desc->request_vega || desc->request_local_vega_nodes) {
        if (desc->model == MCG_MODEL_BLACK_SCHOLES) {
            if (desc->request_local_vega_nodes) return MCG_ERR_UNSUPPORTED;
            rc = lsm_fixed_policy_risk(desc, stop.data(), df.data(), threads, out);
        } else {
            rc = lsm_lv_fixed_policy_risk(desc, stop.data(), df.data(), threads, out);
        }
        if (rc != MCG_OK) return rc;
    }
    return MCG_OK;
}

namespace {

constexpr uint32_t kDomainDualInner = 0x4455414cu;  // dual.rs:22, INNER_DOMAIN

bool finite_or_fail(double v, const char* stage) {
    if (std::isfinite(v)) return true;
    g_lsm_error = std::string("non-finite ") + stage;
    return false;
}

// DualPath, dual.rs:462-500: equation (9) telescoped; the policy is applied
// after the first exercise as well.
struct DualPath {
    NeumaierSum correction;
    double gap = -INFINITY;
    bool observe(double payoff, double continuation, bool exercise, bool terminal) {
        const double value = exercise ? payoff : continuation;
        const double candidate = (payoff - value) - correction.total();
        if (!finite_or_fail(candidate, "dual gap candidate")) return false;
        gap = std::max(gap, candidate);
        if (exercise && !terminal) {
            const double c = payoff - continuation;
            if (!finite_or_fail(c, "dual exercise correction")) return false;
            correction.add(c);
            if (!finite_or_fail(correction.total(), "dual accumulated correction")) return false;
        }
        return true;
    }
};

}  // namespace

// AndersenBroadiePlan::evaluate on the CPU (dual.rs:216-404): the fitted
// policy of train_policy, outer valuation paths stopped by it, inner
// rollouts from every non-terminal exercise date, per-unit (lower, upper,
// gap) reduced in fixed blocks as DeterministicExecutor does.
int lsm_dual(const mcg_plan_desc* desc, const mcg_lsm_desc* lsm, const mcg_dual_desc* dual,
             mcg_dual_result* out, int threads) {
    g_lsm_error.clear();
    if (!desc || !lsm || !dual || !out) return lsm_fail("null argument");
    std::memset(&out->error, 0, sizeof(out->error));
    if (desc->product_count != 1 || desc->products[0].kind != MCG_PRODUCT_AMERICAN)
        return lsm_fail("one American product expected");
    if (desc->model != MCG_MODEL_BLACK_SCHOLES || desc->engine != MCG_ENGINE_PSEUDO ||
        lsm->continuation != MCG_CONTINUATION_POLYNOMIAL || desc->request_delta || desc->request_gamma ||
        desc->request_vega || desc->request_local_vega_nodes)
        return MCG_ERR_UNSUPPORTED;
    if (dual->continuation_inner_paths < 1 || dual->exercise_inner_paths < 1)
        return lsm_fail("inner path counts must be positive");
    if (lsm->max_degree < 1 || lsm->max_degree > MCG_LSM_MAX_DEGREE) return lsm_fail("max_degree");
    const size_t dates = desc->observation_count;
    const mcg_product_desc& pr = desc->products[0];
    std::vector<double> df(dates);
    for (size_t d = 0; d < dates; ++d) df[d] = plan_discount(desc, desc->observation_times[d]);
    std::vector<DateModel> models;
    uint64_t tp = 0;
    double in_sample = 0.0;
    int rc = train_policy(desc, lsm, threads, df, models, tp, in_sample, out->error);
    if (rc != MCG_OK) return rc;
    std::vector<double> spots, brown;
    uint64_t vp = 0;
    rc = lsm_spots(desc, kDomainValuation, threads, spots, vp, out->error, &brown);
    if (rc != MCG_OK) return rc;
    const uint32_t degree = lsm->max_degree;
    const double vol = desc->volatility;
    const double* t = desc->observation_times;
    // forwards of the exercise dates (as the path store uses them) and the
    // step roots sqrt(t_j - t_{j-1}) of the inner paths
    std::vector<double> fwd(dates), sqdt(dates, 0.0);
    for (size_t d = 0; d < dates; ++d) fwd[d] = plan_forward(desc, t[d]);
    for (size_t d = 1; d < dates; ++d) sqdt[d] = std::sqrt(t[d] - t[d - 1]);
    const uint64_t units = desc->sampling_units;
    const uint64_t lanes = desc->antithetic ? 2 : 1;
    const uint64_t stride = std::max(dual->continuation_inner_paths, dual->exercise_inner_paths);
    std::vector<double> values(3 * units);
    std::vector<std::string> errors(static_cast<size_t>(std::max(1, threads)));
    std::atomic<uint64_t> next{0};
    std::atomic<bool> failed{false};
    std::atomic<uint64_t> inner_total{0};
    auto outer = [&](uint64_t trajectory, double res[3], uint64_t& inner_count) -> bool {
        double lower = 0.0;
        bool have_lower = false;
        DualPath dp;
        for (size_t d = 0; d < dates; ++d) {
            const double s = spots[d * vp + trajectory];
            const double payoff = intrinsic(pr, s);
            const bool terminal = d + 1 == dates;
            const bool exercise = terminal || models[d].exercise(payoff, s, degree);
            const double discounted = payoff * df[d];
            if (!finite_or_fail(discounted, "dual discounted payoff")) return false;
            if (exercise && !have_lower) {
                lower = discounted;
                have_lower = true;
            }
            double continuation = 0.0;
            if (!terminal) {
                // rollout_mean, dual.rs:340-400
                const uint32_t configured = exercise ? dual->exercise_inner_paths : dual->continuation_inner_paths;
                const uint32_t paths = vol == 0.0 ? 1u : configured;
                NeumaierSum sum;
                for (uint32_t inner = 0; inner < paths; ++inner) {
                    const uint64_t path = trajectory * stride + inner;
                    double w = brown[d * vp + trajectory];
                    for (size_t j = d + 1; j < dates; ++j) {
                        const uint32_t dim = static_cast<uint32_t>(d * dates + j);
                        const double z = vol == 0.0 ? 0.0 : philox_normal(dual->inner_seed, path, dim, kDomainDualInner);
                        w += sqdt[j] * z;
                        const double variance = vol * vol * t[j];
                        const double canonical = fwd[j] * std::exp(-0.5 * variance + vol * w);
                        const double spot_j = 0.0 * desc->spot + 1.0 * canonical;
                        if (!finite_or_fail(spot_j, "dual inner spot")) return false;
                        const double imm = intrinsic(pr, spot_j);
                        if (j + 1 == dates || models[j].exercise(imm, spot_j, degree)) {
                            const double v = imm * df[j];
                            if (!finite_or_fail(v, "dual inner payoff")) return false;
                            sum.add(v);
                            break;
                        }
                    }
                }
                inner_count += paths;
                continuation = sum.total() / static_cast<double>(paths);
                if (!finite_or_fail(continuation, "dual inner mean")) return false;
            }
            if (!dp.observe(discounted, continuation, exercise, terminal)) return false;
        }
        res[0] = lower;
        res[1] = lower + dp.gap;
        res[2] = dp.gap;
        return finite_or_fail(res[1], "dual upper sample");
    };
    auto worker = [&](size_t tid) {
        uint64_t inner_count = 0;
        for (;;) {
            const uint64_t u = next.fetch_add(1);
            if (u >= units || failed.load()) break;
            double a[3], b[3];
            if (!outer(u * lanes, a, inner_count)) {
                errors[tid] = g_lsm_error;
                failed = true;
                break;
            }
            if (lanes == 2) {
                if (!outer(u * lanes + 1, b, inner_count)) {
                    errors[tid] = g_lsm_error;
                    failed = true;
                    break;
                }
                for (int c = 0; c < 3; ++c) a[c] = 0.5 * a[c] + 0.5 * b[c];
            }
            for (int c = 0; c < 3; ++c) values[3 * u + c] = a[c];
        }
        inner_total += inner_count;
    };
    std::vector<std::thread> pool;
    for (size_t i = 0; i < errors.size(); ++i) pool.emplace_back(worker, i);
    for (auto& th : pool) th.join();
    if (failed) {
        for (auto& e : errors)
            if (!e.empty()) g_lsm_error = e;
        out->error.code = MCG_ERR_LSM;
        return MCG_ERR_LSM;
    }
    // DeterministicExecutor blocks of reduction_block_size, merged in the fixed tree.
    const uint64_t block = desc->reduction_block_size ? desc->reduction_block_size : 4096;
    const uint64_t nblocks = (units + block - 1) / block;
    const double inv = 1.0 / static_cast<double>(units);
    mcg_estimate* est[3] = {&out->lower_bound, &out->upper_bound, &out->duality_gap};
    for (int c = 0; c < 3; ++c) {
        std::vector<NeumaierSum> sums(nblocks);
        std::vector<CenteredMoment> moms(nblocks);
        for (uint64_t b = 0; b < nblocks; ++b) {
            Statistics st;
            for (uint64_t u = b * block; u < std::min(units, (b + 1) * block); ++u) st.add(values[3 * u + c]);
            sums[b] = st.sum;
            moms[b] = st.moments;
        }
        Statistics total;
        total.sum = fixed_tree_reduce(sums, NeumaierSum::merged);
        total.moments = fixed_tree_reduce(moms, CenteredMoment::merged);
        out->components[c] = {total.sum.sum, total.sum.correction, total.moments.count, total.moments.mean,
                              total.moments.second_moment};
        const double value = total.sum.total() * inv * 1.0;
        const double var = total.moments.count > 1
                               ? total.moments.second_moment / static_cast<double>(total.moments.count - 1)
                               : 0.0;
        const double se = std::sqrt(var * inv) * 1.0;
        *est[c] = {value, se, value - kNormal95 * se, value + kNormal95 * se, units};
    }
    out->price_confidence_interval_95[0] = out->lower_bound.confidence_lower;
    out->price_confidence_interval_95[1] = out->upper_bound.confidence_upper;
    out->outer_trajectories = units * lanes;
    out->inner_paths = inner_total.load();
    out->exercise_date_count = static_cast<uint32_t>(dates);
    return MCG_OK;
}

const char* lsm_last_error() { return g_lsm_error.c_str(); }

// FeatureScaling::fit of given values: out = mean, population variance,
// scale, zero-scale threshold; the return value is the inactive flag.
int lsm_scaling_api(const double* values, size_t n, double out[4]) {
    const Scaling s = fit_scaling(std::vector<double>(values, values + n));
    out[0] = s.mean;
    out[1] = s.variance;
    out[2] = s.scale;
    out[3] = s.threshold;
    return s.inactive ? 1 : 0;
}

// fit_cpqr of a row-major design matrix: pivot order, rank, coefficients in
// the original column order and the residual sum of squares.
int lsm_cpqr_api(const double* matrix, size_t rows, size_t cols, const double* target, double abs_tol,
                 double rel_tol, uint32_t* pivot, uint32_t* rank, double* coefficients, double* rss) {
    Cpqr fit;
    if (!fit_cpqr(std::vector<double>(matrix, matrix + rows * cols), rows, cols,
                  std::vector<double>(target, target + rows), abs_tol, rel_tol, fit))
        return MCG_ERR_LSM;
    for (size_t c = 0; c < cols; ++c) {
        pivot[c] = static_cast<uint32_t>(fit.pivot[c]);
        coefficients[c] = fit.coefficients[c];
    }
    *rank = static_cast<uint32_t>(fit.rank);
    *rss = fit.rss;
    return MCG_OK;
}

int lsm_fit_api(const double* spots, const double* immediate, const double* targets, size_t rows,
                const mcg_lsm_desc* lsm, mcg_lsm_date_model* out) {
    g_lsm_error.clear();
    if (lsm->max_degree < 1 || lsm->max_degree > MCG_LSM_MAX_DEGREE) return lsm_fail("max_degree");
    const Config cfg{lsm->max_degree, lsm->itm_abs_tolerance, lsm->cpqr_abs_tolerance,
                     lsm->cpqr_rel_tolerance, lsm->max_matrix_elements};
    DateModel m;
    const int rc = fit_date(cfg, immediate, spots, std::vector<double>(targets, targets + rows), rows, m);
    *out = m.rec;
    return rc;
}

}  // namespace oracle

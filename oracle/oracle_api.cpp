// oracle_api.cpp -- extern "C" surface of the CPU oracle (liboracle.so).
//
// TEST INFRASTRUCTURE ONLY.  Loaded by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py to check and time the CUDA engine; never linked
// into the engine itself.
#include <cstring>
#include <vector>

#include "../include/mcg.h"
#include "oracle_core.h"

namespace oracle {
int evaluate(const mcg_plan_desc* desc, mcg_result* result, int threads);
const char* last_error();
int unit_shocks_api(const mcg_plan_desc* desc, uint32_t scramble, uint64_t unit, double* out);
int unit_values_api(const mcg_plan_desc* desc, uint32_t scramble, uint64_t unit, double* out);
int bump_evaluate_api(const mcg_plan_desc* desc, const mcg_bump_request* req, uint32_t count,
                      mcg_bump_estimate* est, mcg_bump_report* rep, int threads);
int time_grid_api(const mcg_plan_desc* desc, double* nodes_out, uint32_t capacity, uint32_t* count);
std::vector<double> pchip_derivatives(const std::vector<double>& t, const std::vector<double>& v);
int vega_kt_project(const double* times, uint32_t nt, const double* xs, uint32_t nx, const double* nodes,
                    uint64_t paths, const mcg_vega_kt_basis* basis, mcg_vega_kt_projection* out);
int surface_grid(const mcg_surface_desc& d, const std::vector<double>& tn, const std::vector<double>& xn,
                 double floor, double cap, std::vector<double>& out);
bool surface_derivatives(const mcg_surface_desc& d, const std::vector<double>& pd, double time, double k,
                         double out[4]);
int ssvi_grid(const std::vector<double>& theta_t, const std::vector<double>& theta_v, double slope,
              double rho, double eta, double gamma, const std::vector<double>& tn,
              const std::vector<double>& xn, double floor, double cap, std::vector<double>& out);
std::vector<double> piecewise_sinh_nodes(double left, double right, size_t nl, size_t nr,
                                         double ls, double rs);
int lsm_price(const mcg_plan_desc* desc, const mcg_lsm_desc* lsm, mcg_lsm_result* out, int threads);
const char* lsm_last_error();
int lsm_spots(const mcg_plan_desc* desc, uint32_t domain, int threads, std::vector<double>& spots,
              uint64_t& path_count, mcg_error_record& err, std::vector<double>* brownians);
int lsm_dual(const mcg_plan_desc* desc, const mcg_lsm_desc* lsm, const mcg_dual_desc* dual,
             mcg_dual_result* out, int threads);
int lsm_scaling_api(const double* values, size_t n, double out[4]);
int lv_barrier_adjoints_api(const double* times, uint32_t n_times, const double* forwards, const double* grid_t,
                            uint32_t nt, const double* grid_x, uint32_t nx, const double* values, double initial,
                            const double* shocks, double barrier, int up, int knock_out, uint32_t monitor_end,
                            double quadratic, double rebate, double discount, double* price_out,
                            double* grid_adj_out);
int lv_step_adjoints_api(const double* times, uint32_t n_times, const double* forwards, const double* grid_t,
                         uint32_t nt, const double* grid_x, uint32_t nx, const double* values, double initial,
                         const double* shocks, const double* state_seeds, double* states_out,
                         double* grid_adj_out);
int lsm_cpqr_api(const double* matrix, size_t rows, size_t cols, const double* target, double abs_tol,
                 double rel_tol, uint32_t* pivot, uint32_t* rank, double* coefficients, double* rss);
int lsm_fit_api(const double* spots, const double* immediate, const double* targets, size_t rows,
                const mcg_lsm_desc* lsm, mcg_lsm_date_model* out);
}  // namespace oracle

extern "C" {

void oracle_philox_block(uint64_t seed, const uint32_t counter[4], uint32_t out[4]) {
    oracle::Block4 c{{counter[0], counter[1], counter[2], counter[3]}};
    const oracle::Block4 r = oracle::philox_generate(seed, c);
    std::memcpy(out, r.v, sizeof(r.v));
}

uint32_t oracle_philox_word(uint64_t seed, uint64_t path, uint32_t dimension, uint32_t domain) {
    return oracle::philox_word(seed, path, dimension, domain);
}

double oracle_open_unit_interval(uint32_t word) { return oracle::open_unit_interval(word); }

double oracle_inverse_normal(double p) { return oracle::inverse_standard_normal(p); }

double oracle_philox_normal(uint64_t seed, uint64_t path, uint32_t dimension, uint32_t domain) {
    return oracle::philox_normal(seed, path, dimension, domain);
}

uint32_t oracle_sobol_word(const uint32_t* directions32, uint32_t point) {
    return oracle::sobol_word(directions32, point);
}

void oracle_scramble(uint64_t seed, uint32_t scramble, uint32_t dimension, uint32_t* shift,
                     uint32_t rows[32]) {
    const oracle::Scramble s = oracle::compile_scramble(seed, scramble, dimension);
    *shift = s.shift;
    std::memcpy(rows, s.rows, sizeof(s.rows));
}

uint32_t oracle_rqmc_word(const uint32_t* directions32, uint64_t seed, uint32_t scramble,
                          uint32_t dimension, uint32_t point) {
    const oracle::Scramble s = oracle::compile_scramble(seed, scramble, dimension);
    return s.apply(oracle::sobol_word(directions32, point));
}

// Brownian bridge: returns the instruction count (or -1 on an invalid grid) and
// fills node/rank order plus coefficients when the outputs are non-null.
int oracle_bridge_compile(const double* times, uint32_t count, uint32_t* nodes, uint32_t* ranks,
                          double* left_weights, double* right_weights, double* sds) {
    oracle::BridgePlan plan;
    if (!plan.compile(std::vector<double>(times, times + count))) return -1;
    for (size_t i = 0; i < plan.instructions.size(); ++i) {
        const auto& ins = plan.instructions[i];
        if (nodes) nodes[i] = ins.node;
        if (ranks) ranks[i] = ins.rank;
        if (left_weights) left_weights[i] = ins.left_weight;
        if (right_weights) right_weights[i] = ins.right_weight;
        if (sds) sds[i] = ins.standard_deviation;
    }
    return static_cast<int>(plan.instructions.size());
}

int oracle_bridge_apply(const double* times, uint32_t count, const double* normals,
                        double* increments) {
    oracle::BridgePlan plan;
    if (!plan.compile(std::vector<double>(times, times + count))) return -1;
    std::vector<double> scratch;
    plan.apply(normals, increments, scratch);
    return 0;
}

int oracle_bridge_reverse(const double* times, uint32_t count, const double* increment_adjoints,
                          double* normal_adjoints) {
    oracle::BridgePlan plan;
    if (!plan.compile(std::vector<double>(times, times + count))) return -1;
    std::vector<double> scratch;
    plan.reverse(increment_adjoints, normal_adjoints, scratch);
    return 0;
}

int oracle_evaluate(const mcg_plan_desc* desc, mcg_result* result, int threads) {
    return oracle::evaluate(desc, result, threads);
}

int oracle_unit_shocks(const mcg_plan_desc* desc, uint32_t scramble, uint64_t unit, double* out) {
    return oracle::unit_shocks_api(desc, scramble, unit, out);
}

int oracle_unit_values(const mcg_plan_desc* desc, uint32_t scramble, uint64_t unit, double* out) {
    return oracle::unit_values_api(desc, scramble, unit, out);
}

int oracle_bump_evaluate(const mcg_plan_desc* desc, const mcg_bump_request* requests, uint32_t count,
                         mcg_bump_estimate* estimates, mcg_bump_report* report, int threads) {
    return oracle::bump_evaluate_api(desc, requests, count, estimates, report, threads);
}

int oracle_time_grid(const mcg_plan_desc* desc, double* nodes, uint32_t capacity,
                     uint32_t* count) {
    return oracle::time_grid_api(desc, nodes, capacity, count);
}

const char* oracle_last_error(void) { return oracle::last_error(); }

int oracle_lsm_price(const mcg_plan_desc* desc, const mcg_lsm_desc* lsm, mcg_lsm_result* out,
                     int threads) {
    return oracle::lsm_price(desc, lsm, out, threads);
}

const char* oracle_lsm_last_error(void) { return oracle::lsm_last_error(); }

// Spot matrix [date][path] of an early-exercise plan under `domain`; returns the
// path count, or -status on a failure.
int64_t oracle_lsm_spots(const mcg_plan_desc* desc, uint32_t domain, int threads, double* out,
                         uint64_t capacity) {
    std::vector<double> spots;
    uint64_t paths = 0;
    mcg_error_record err{};
    const int rc = oracle::lsm_spots(desc, domain, threads, spots, paths, err, nullptr);
    if (rc != MCG_OK) return -static_cast<int64_t>(rc);
    if (out && capacity >= spots.size()) std::memcpy(out, spots.data(), spots.size() * sizeof(double));
    return static_cast<int64_t>(paths);
}

// One date's regression (fit_exercise_decision) on given rows.
int oracle_lsm_dual(const mcg_plan_desc* desc, const mcg_lsm_desc* lsm, const mcg_dual_desc* dual,
                    mcg_dual_result* out, int threads) {
    return oracle::lsm_dual(desc, lsm, dual, out, threads);
}

int oracle_lv_step_adjoints(const double* times, uint32_t n_times, const double* forwards, const double* grid_t,
                            uint32_t nt, const double* grid_x, uint32_t nx, const double* values, double initial,
                            const double* shocks, const double* state_seeds, double* states_out,
                            double* grid_adj_out) {
    return oracle::lv_step_adjoints_api(times, n_times, forwards, grid_t, nt, grid_x, nx, values, initial, shocks,
                                        state_seeds, states_out, grid_adj_out);
}

int oracle_lv_barrier_adjoints(const double* times, uint32_t n_times, const double* forwards,
                               const double* grid_t, uint32_t nt, const double* grid_x, uint32_t nx,
                               const double* values, double initial, const double* shocks, double barrier, int up,
                               int knock_out, uint32_t monitor_end, double quadratic, double rebate,
                               double discount, double* price_out, double* grid_adj_out) {
    return oracle::lv_barrier_adjoints_api(times, n_times, forwards, grid_t, nt, grid_x, nx, values, initial, shocks,
                                           barrier, up, knock_out, monitor_end, quadratic, rebate, discount,
                                           price_out, grid_adj_out);
}

int oracle_lsm_scaling(const double* values, uint64_t n, double* out) {
    return oracle::lsm_scaling_api(values, n, out);
}

int oracle_lsm_cpqr(const double* matrix, uint64_t rows, uint32_t cols, const double* target, double abs_tol,
                    double rel_tol, uint32_t* pivot, uint32_t* rank, double* coefficients, double* rss) {
    return oracle::lsm_cpqr_api(matrix, rows, cols, target, abs_tol, rel_tol, pivot, rank, coefficients, rss);
}

int oracle_lsm_fit(const double* spots, const double* immediate, const double* targets,
                   uint64_t rows, const mcg_lsm_desc* lsm, mcg_lsm_date_model* out) {
    return oracle::lsm_fit_api(spots, immediate, targets, rows, lsm, out);
}

int oracle_ssvi_grid(const double* theta_t, const double* theta_v, uint32_t theta_count,
                     double slope, double rho, double eta, double gamma, const double* tn,
                     uint32_t nt, const double* xn, uint32_t nx, double floor, double cap,
                     double* out) {
    std::vector<double> values;
    const int repairs = oracle::ssvi_grid(std::vector<double>(theta_t, theta_t + theta_count),
                                          std::vector<double>(theta_v, theta_v + theta_count), slope,
                                          rho, eta, gamma, std::vector<double>(tn, tn + nt),
                                          std::vector<double>(xn, xn + nx), floor, cap, values);
    if (repairs >= 0) std::memcpy(out, values.data(), values.size() * sizeof(double));
    return repairs;
}

// Dupire grid of any surface kind (mcg_surface_desc); repairs or -1.
int oracle_surface_grid(const mcg_surface_desc* d, const double* tn, uint32_t nt, const double* xn, uint32_t nx,
                        double floor, double cap, double* out) {
    std::vector<double> values;
    const int repairs = oracle::surface_grid(*d, std::vector<double>(tn, tn + nt), std::vector<double>(xn, xn + nx),
                                             floor, cap, values);
    if (repairs >= 0) std::memcpy(out, values.data(), values.size() * sizeof(double));
    return repairs;
}

// w, w_k, w_kk, w_t of a surface at (t, k); 0, or -1 where the surface fails.
int oracle_surface_total_variance(const mcg_surface_desc* d, double t, double k, double* out) {
    std::vector<double> pd;
    if (d->kind != MCG_SURFACE_ESSVI)
        pd = oracle::pchip_derivatives(std::vector<double>(d->theta_times, d->theta_times + d->theta_count),
                                       std::vector<double>(d->theta_values, d->theta_values + d->theta_count));
    return oracle::surface_derivatives(*d, pd, t, k, out) ? 0 : -1;
}

// VegaKT node allocation of node sensitivities (grid rows x nodes).
int oracle_vega_kt_project(const double* times, uint32_t nt, const double* xs, uint32_t nx, const double* nodes,
                           uint64_t paths, const mcg_vega_kt_basis* basis, mcg_vega_kt_projection* out) {
    return oracle::vega_kt_project(times, nt, xs, nx, nodes, paths, basis, out);
}

int oracle_piecewise_sinh_nodes(double left, double right, uint32_t nl, uint32_t nr,
                                double left_shape, double right_shape, double* out) {
    const std::vector<double> n =
        oracle::piecewise_sinh_nodes(left, right, nl, nr, left_shape, right_shape);
    std::memcpy(out, n.data(), n.size() * sizeof(double));
    return static_cast<int>(n.size());
}

}  // extern "C"

namespace oracle {
int barrier_path_api(int up, double barrier, double h, const double* states,
                     const double* variances, const double* times, size_t count, double* survival,
                     double* diag);
}

extern "C" int oracle_barrier_path(int up, double barrier, double h, const double* states,
                                   const double* variances, const double* times, uint32_t count,
                                   double* survival, double* diag) {
    return oracle::barrier_path_api(up, barrier, h, states, variances, times, count, survival, diag);
}

namespace oracle {
void smoothing_api(double h, double input, double* out);
void extrema_api(double h, double left, double right, double* out);
int exact_bridge_api(int up, double barrier, double s0, double s1, double integrated, double* survival);
int smoothed_bridge_api(int up, double barrier, double s0, double s1, double h, double integrated, double* out);
}

extern "C" {
void oracle_smoothing(double h, double input, double* out) { oracle::smoothing_api(h, input, out); }
void oracle_smooth_extrema(double h, double l, double r, double* out) { oracle::extrema_api(h, l, r, out); }
int oracle_exact_bridge(int up, double barrier, double s0, double s1, double iv, double* survival) {
    return oracle::exact_bridge_api(up, barrier, s0, s1, iv, survival);
}
int oracle_smoothed_bridge(int up, double barrier, double s0, double s1, double h, double iv, double* out) {
    return oracle::smoothed_bridge_api(up, barrier, s0, s1, h, iv, out);
}
}

namespace oracle {
int interval_adjoint_api(int up, double barrier, double h, double lsa, double ls, double rs, double lv,
                         double rv, double dt, double* out);
}
extern "C" int oracle_interval_adjoint(int up, double barrier, double h, double lsa, double ls, double rs,
                                       double lv, double rv, double dt, double* out) {
    return oracle::interval_adjoint_api(up, barrier, h, lsa, ls, rs, lv, rv, dt, out);
}

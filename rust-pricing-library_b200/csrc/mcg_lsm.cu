// mcg_lsm.cu -- Longstaff--Schwartz early exercise on the GPU.
//
// Replaces, from msfmfjt/rust-pricing-library (paths relative to that project):
//   pseudo/rqmc_lsm_path_matrices, write_lsm_trajectory
//       crates/pricing/src/engine/mc/early_exercise.rs:28-175,330-385
//   train_exercise_policy        crates/pricing/src/engine/mc/lsm.rs:1486-1695
//   fit_exercise_decision        lsm.rs:1928-2065
//   fit_polynomial_regression    lsm.rs:2067-2247
//   fit_cpqr                     lsm.rs:2374-2652
//   value_exercise_policy        lsm.rs:1347-1482
//   collapse_antithetic_values / rqmc_replicate_values  early_exercise.rs:616-712
//
// Layout.  The training phase stores one FP64 spot per (date, path), date-major
// (`spots[d * paths + p]`, antithetic mates adjacent so a thread stores one
// 16-byte pair).  The immediate value is the American payoff graph's output,
// max(+-(S - K), 0) * notional (crates/pricing/src/engine/payoff/compile.rs:67-101),
// recomputed from the spot wherever it is needed instead of being stored.
// Each training path keeps two words of state: its realised cash flow
// discounted to time zero, cf = realised * df[stop] (the reference's target
// realised * df[stop] / df[d] is then cf / df[d], bit for bit), and its
// stopping date.
//
// Backward induction, per non-terminal date d (three launches):
//   sweep(d):    applies the decision of date d+1 to every path (exercise if
//                immediate > continuation) while summing the residuals of that
//                date's fit, and gathers count, sum and max |S| of the ITM rows
//                of date d;
//   variance(d): the population variance of the ITM spots about their mean;
//   gram(d):     the Gram matrix of the standardised monomial basis and its
//                right-hand side over the ITM rows; the last CTA solves.
// Every sum is an error-free double-double accumulation (TwoSum, FMA TwoProd)
// reduced in a fixed order, so it is the exactly rounded sum the reference's
// sequential Neumaier sums approximate.  The last CTA to finish a pass (a
// ticket counter, no waiting) merges the per-CTA partials and finalises.
//
// The solve.  The reference runs Householder QR with column pivoting on the
// ITM design matrix.  In exact arithmetic the pivot sequence, |R_kk| and the
// coefficients of CPQR equal those of a diagonally pivoted Cholesky
// factorisation of the Gram matrix (the squared norm of a remaining column
// after k reflections is the Schur-complement diagonal), so one thread runs
// that factorisation in double-double arithmetic on the exactly accumulated
// Gram matrix.  The result is the least-squares solution to ~1e-30, i.e. the
// coefficients the reference approximates to its own O(kappa * eps).
//
// Valuation needs no path store: one thread generates a valuation path and
// applies the fitted policy date by date, stopping at the first exercise.
#include <cstdint>

#include "mcg_kernels.cuh"
#include "mcg_lsm.cuh"

namespace mcg {

constexpr int kLsmThreads = 256;
constexpr int kLsmWarps = kLsmThreads / 32;
constexpr int kLsmMaxBasis = MCG_LSM_MAX_BASIS;
constexpr double kEpsilon64 = 2.220446049250313e-16;

// ------------------------------------------------------------ double-double

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Accumulating forms: `hi` carries the running sum, `lo` the collected errors.
__device__ __forceinline__ DD acc_add(DD a, double v) {
    double s, e;
    two_sum(a.hi, v, s, e);
    return {s, a.lo + e};
}

__device__ __forceinline__ DD acc_prod(DD a, double x, double y) {
    const double p = x * y;
    const double pe = __fma_rn(x, y, -p);
    double s, e;
    two_sum(a.hi, p, s, e);
    return {s, a.lo + (e + pe)};
}

__device__ __forceinline__ DD acc_merge(DD a, DD b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    return {s, (a.lo + b.lo) + e};
}

__device__ __forceinline__ double dd_round(DD a) { return a.hi + a.lo; }

// Normalised double-double arithmetic for the small solve (the algorithms of
// Hida, Li and Bailey's QD library: Dekker/Knuth error-free transformations).
__device__ __forceinline__ DD quick_two_sum(double a, double b) {
    const double s = a + b;
    return {s, b - (s - a)};
}

__device__ __forceinline__ DD dd_from(double a) { return {a, 0.0}; }

__device__ __forceinline__ DD dd_norm(DD a) { return quick_two_sum(a.hi, a.lo); }

__device__ __forceinline__ DD dd_add(DD a, DD b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    double t, f;
    two_sum(a.lo, b.lo, t, f);
    e += t;
    DD r = quick_two_sum(s, e);
    r.lo += f;
    return quick_two_sum(r.hi, r.lo);
}

__device__ __forceinline__ DD dd_neg(DD a) { return {-a.hi, -a.lo}; }

__device__ __forceinline__ DD dd_sub(DD a, DD b) { return dd_add(a, dd_neg(b)); }

__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = a.hi * b.hi;
    double e = __fma_rn(a.hi, b.hi, -p);
    e += a.hi * b.lo + a.lo * b.hi;
    return quick_two_sum(p, e);
}

__device__ __forceinline__ DD dd_mul_d(DD a, double b) {
    const double p = a.hi * b;
    double e = __fma_rn(a.hi, b, -p);
    e += a.lo * b;
    return quick_two_sum(p, e);
}

__device__ __forceinline__ DD dd_div(DD a, DD b) {
    const double q1 = a.hi / b.hi;
    DD r = dd_sub(a, dd_mul_d(b, q1));
    const double q2 = r.hi / b.hi;
    r = dd_sub(r, dd_mul_d(b, q2));
    const double q3 = r.hi / b.hi;
    DD q = quick_two_sum(q1, q2);
    return dd_add(q, dd_from(q3));
}

__device__ __forceinline__ DD dd_sqrt(DD a) {
    if (a.hi <= 0.0) return dd_from(0.0);
    const double s = sqrt(a.hi);
    const DD sq = {s * s, __fma_rn(s, s, -(s * s))};
    const DD r = dd_sub(a, sq);
    return quick_two_sum(s, r.hi / (2.0 * s));
}

__device__ __forceinline__ bool dd_greater(DD a, DD b) {
    return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo);
}

__device__ __forceinline__ bool dd_equal(DD a, DD b) { return a.hi == b.hi && a.lo == b.lo; }

// ------------------------------------------------------------- arguments


constexpr int kLsmPartials = kLsmMaxBasis * (kLsmMaxBasis + 1) / 2 + 2 * kLsmMaxBasis + 4;

// The fields of a date model the decisions read.
struct Policy {
    int32_t regression, inactive;
    double mean, scale;
    double coef[kLsmMaxBasis];
};

__device__ __forceinline__ Policy policy_of(const mcg_lsm_date_model& m, uint32_t nb) {
    Policy q;
    q.regression = m.regression;
    q.inactive = m.feature_inactive;
    q.mean = m.feature_mean;
    q.scale = m.feature_scale;
    for (uint32_t e = 0; e < nb; ++e) q.coef[e] = m.coefficients[e];
    return q;
}

__device__ __forceinline__ double intrinsic(int32_t side, double strike, double notional, double s) {
    const double in = side == MCG_CALL ? s - strike : strike - s;
    return (in >= 0.0 ? in : 0.0) * notional;
}

// PolynomialRegressionModel::predict (lsm.rs:776-790): basis values are the
// monomials of evaluate_monomial (repeated products from 1.0), summed with a
// sequential Neumaier sum in basis order.
__device__ __forceinline__ double predict(const Policy& m, uint32_t nb, double x) {
    const double z = m.inactive ? 0.0 : (x - m.mean) / m.scale;
    double sum = 0.0, corr = 0.0, b = 1.0;
    for (uint32_t e = 0; e < nb; ++e) {
        if (e) b *= z;
        neumaier_add(sum, corr, b * m.coef[e]);
    }
    return sum + corr;
}

__device__ __forceinline__ DD warp_reduce_dd(DD v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        DD o;
        o.hi = __shfl_down_sync(0xffffffffu, v.hi, off);
        o.lo = __shfl_down_sync(0xffffffffu, v.lo, off);
        v = acc_merge(v, o);
    }
    return v;
}

// Reduces K accumulators of every thread to one per CTA (fixed order) and
// stores them at partials[blockIdx.x * kLsmPartials + k] (thread 0's `extra`,
// if given, at k = K).  Returns true in the CTA that finished last, after
// which every CTA's partials are visible to it.
template <int K>
__device__ bool cta_reduce_publish(DD (&v)[K], DD* partials, unsigned int* ticket, DD* smem,
                                   const DD* extra = nullptr) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const DD r = warp_reduce_dd(v[k]);
        if (lane == 0) smem[warp * K + k] = r;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        DD m = smem[threadIdx.x];
        for (int w = 1; w < kLsmWarps; ++w) m = acc_merge(m, smem[w * K + threadIdx.x]);
        partials[static_cast<size_t>(blockIdx.x) * kLsmPartials + threadIdx.x] = m;
    }
    if (extra && threadIdx.x == 0) partials[static_cast<size_t>(blockIdx.x) * kLsmPartials + K] = *extra;
    __threadfence();
    __syncthreads();
    __shared__ unsigned int s_last;
    if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1 ? 1u : 0u;
    __syncthreads();
    if (s_last) __threadfence();
    return s_last != 0;
}

// In the last CTA: merges the partials of every CTA for k < K in block order
// (a lane-strided pass per warp, then a butterfly), into smem[k].
template <int K>
__device__ void merge_partials(const DD* partials, DD* out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = warp; k < K; k += kLsmWarps) {
        DD acc = {0.0, 0.0};
        for (uint32_t b = lane; b < gridDim.x; b += 32) {
            const DD* p = partials + static_cast<size_t>(b) * kLsmPartials + k;
            acc = acc_merge(acc, DD{__ldcg(&p->hi), __ldcg(&p->lo)});
        }
        acc = warp_reduce_dd(acc);
        if (lane == 0) out[k] = acc;
    }
    __syncthreads();
}

__device__ __forceinline__ void lsm_fail(unsigned long long* word, uint32_t date) {
    atomicMin(word, (static_cast<unsigned long long>(date) << 8) | static_cast<unsigned>(MCG_ERR_LSM));
}

// ---------------------------------------------------------------- path store

// Black--Scholes path spots at the exercise dates, path_observations_from_normals
// (crates/pricing/src/engine/processes/black_scholes.rs:297-331).  One thread
// per sampling unit (RQMC: per point, scramble = blockIdx.y) and its mate.
__global__ void __launch_bounds__(kLsmThreads) lsm_bs_spots_kernel(const DevicePlan P, uint32_t domain,
                                                                   double* spots, uint64_t paths,
                                                                   unsigned long long* bad) {
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (point >= P.units) return;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = point;
    ns.gray = static_cast<uint32_t>(point ^ (point >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    ns.domain = domain;
    const uint64_t unit = static_cast<uint64_t>(scramble) * P.units + point;
    const bool pair = P.antithetic != 0;
    const uint64_t col = unit * (pair ? 2u : 1u);
    const uint32_t n = P.observation_count;
    double w0 = 0.0, w1 = 0.0;
    bool finite = true;
    for (uint32_t i = 0; i < n; ++i) {
        const double z = P.zero_variance ? 0.0 : ns.normal(i);
        const double t = P.obs_time[i];
        const double tv = P.vol * P.vol * t;
        double f0, f1;
        if (n == 1) {
            const double sd = sqrt(tv);
            f0 = P.obs_fwd[0] * 1.0 * exp(-0.5 * tv + sd * z);
            f1 = P.obs_fwd[0] * 1.0 * exp(-0.5 * tv + sd * -z);
        } else {
            w0 += P.obs_sqrt_step[i] * z;
            w1 += P.obs_sqrt_step[i] * -z;
            f0 = P.obs_fwd[i] * 1.0 * exp(-0.5 * tv + P.vol * w0);
            f1 = P.obs_fwd[i] * 1.0 * exp(-0.5 * tv + P.vol * w1);
        }
        finite &= isfinite(f0) && (!pair || isfinite(f1));
        double* row = spots + static_cast<size_t>(i) * paths + col;
        if (pair) {
            *reinterpret_cast<double2*>(row) = make_double2(f0, f1);
        } else {
            *row = f0;
        }
    }
    if (!finite) atomicMin(bad, unit);
}

// ------------------------------------------------------------- training sweep

// One pass over every training path: initialise (first pass), apply the
// decision of date `update` and sum that fit's residuals over its ITM rows,
// and gather the ITM count, spot sum and max |spot| of date `gather`.
__global__ void __launch_bounds__(kLsmThreads) lsm_sweep_kernel(const LsmArgs A, int init, int update,
                                                                int gather) {
    __shared__ DD s_red[kLsmWarps * 2];
    __shared__ DD s_fin[2];
    __shared__ unsigned long long s_cnt[kLsmWarps];
    __shared__ double s_max[kLsmWarps];
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint32_t last = A.dates - 1;
    Policy mu{};
    if (update >= 0) mu = policy_of(A.models[update], A.nb);
    const bool decide = update >= 0 && mu.regression;
    const double df_u = update >= 0 ? A.df[update] : 1.0;
    DD acc[2] = {{0.0, 0.0}, {0.0, 0.0}};  // residual squares of `update`, ITM spot sum of `gather`
    unsigned long long cnt = 0;
    double maxabs = 1.0;
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.paths; p += stride) {
        double cf;
        if (init) {
            const double x = A.spots[static_cast<size_t>(last) * A.paths + p];
            cf = intrinsic(A.side, A.strike, A.notional, x) * A.df[last];
            A.stop[p] = last;
        } else {
            cf = A.cf[p];
        }
        if (decide) {
            const double x = A.spots[static_cast<size_t>(update) * A.paths + p];
            const double imm = intrinsic(A.side, A.strike, A.notional, x);
            const double cont = predict(mu, A.nb, x);
            if (imm > A.itm_tol) {
                const double res = cf / df_u - cont;
                acc[0] = acc_add(acc[0], res * res);
            }
            if (imm > cont) {
                cf = imm * df_u;
                A.stop[p] = static_cast<uint32_t>(update);
            }
        }
        if (init || decide) A.cf[p] = cf;
        if (gather >= 0) {
            const double x = A.spots[static_cast<size_t>(gather) * A.paths + p];
            if (intrinsic(A.side, A.strike, A.notional, x) > A.itm_tol) {
                ++cnt;
                acc[1] = acc_add(acc[1], x);
                maxabs = fmax(maxabs, fabs(x));
            }
        }
    }
    // integer count and maximum: exact in any order
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, off);
        maxabs = fmax(maxabs, __shfl_down_sync(0xffffffffu, maxabs, off));
    }
    if (lane == 0) {
        s_cnt[warp] = cnt;
        s_max[warp] = maxabs;
    }
    __syncthreads();
    DD extra = {0.0, 1.0};  // the CTA's ITM count and max |spot|, both exact as doubles
    if (threadIdx.x == 0) {
        unsigned long long c = 0;
        double m = 1.0;
        for (int w = 0; w < kLsmWarps; ++w) {
            c += s_cnt[w];
            m = fmax(m, s_max[w]);
        }
        extra = {static_cast<double>(c), m};
    }
    if (!cta_reduce_publish<2>(acc, A.partials, &A.tickets[0], s_red, &extra)) return;
    merge_partials<2>(A.partials, s_fin);
    if (threadIdx.x == 0) {
        unsigned long long total = 0;
        double m = 1.0;
        for (uint32_t b = 0; b < gridDim.x; ++b) {
            const DD* q = A.partials + static_cast<size_t>(b) * kLsmPartials + 2;
            total += static_cast<unsigned long long>(__ldcg(&q->hi));
            m = fmax(m, __ldcg(&q->lo));
        }
        if (decide) A.models[update].residual_sum_squares = dd_round(s_fin[0]);
        if (gather >= 0) {
            mcg_lsm_date_model& g = A.models[gather];
            g.candidate_rows = static_cast<uint32_t>(A.paths);
            g.itm_rows = static_cast<uint32_t>(total);
            g.regression = 0;
            if (total > 0) {
                g.feature_mean = dd_round(s_fin[1]) / static_cast<double>(total);
                g.zero_scale_threshold = (64.0 * kEpsilon64) * m;
                if (total > A.max_elements) lsm_fail(A.lsm_error, static_cast<uint32_t>(gather));
            }
        }
        A.tickets[0] = 0;
    }
}

// Population variance of the ITM spots of date `d` about their mean
// (FeatureScaling::fit, lsm.rs:537-574).
__global__ void __launch_bounds__(kLsmThreads) lsm_variance_kernel(const LsmArgs A, int d) {
    __shared__ DD s_red[kLsmWarps * 1];
    __shared__ DD s_fin[1];
    const mcg_lsm_date_model m = A.models[d];
    if (m.itm_rows == 0) return;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    DD acc[1] = {{0.0, 0.0}};
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.paths; p += stride) {
        const double x = A.spots[static_cast<size_t>(d) * A.paths + p];
        if (intrinsic(A.side, A.strike, A.notional, x) > A.itm_tol) {
            const double dv = x - m.feature_mean;
            acc[0] = acc_add(acc[0], dv * dv);
        }
    }
    if (!cta_reduce_publish<1>(acc, A.partials, &A.tickets[1], s_red)) return;
    merge_partials<1>(A.partials, s_fin);
    if (threadIdx.x == 0) {
        mcg_lsm_date_model& g = A.models[d];
        g.feature_variance = dd_round(s_fin[0]) / static_cast<double>(m.itm_rows);
        g.feature_scale = sqrt(g.feature_variance);
        g.feature_inactive = g.feature_scale <= g.zero_scale_threshold ? 1 : 0;
        A.tickets[1] = 0;
    }
}

// The CPQR-equivalent solve of one date (one thread).  `gram` holds the upper
// triangle of the NB x NB Gram matrix row by row, the NB right-hand sides, and
// the NB sums of rounded squares fl(b_j * b_j): the reference's first pivot
// compares exactly those column norms (column_squared_norm, lsm.rs:2594-2613),
// and for standardised data sum z^2 ties with sum 1 = n in exact arithmetic, so
// the first choice is made on the same rounded quantities.  Later pivots use
// the Schur-complement diagonals.
template <int NB>
__device__ void lsm_solve(const LsmArgs& A, int d, const DD* gram) {
    mcg_lsm_date_model& m = A.models[d];
    const uint32_t rows = m.itm_rows;
    const int na = m.feature_inactive ? 1 : NB;  // active basis columns: all, or z^0 alone
    if (static_cast<unsigned long long>(rows) * static_cast<unsigned long long>(na) > A.max_elements) {
        lsm_fail(A.lsm_error, static_cast<uint32_t>(d));
        return;
    }
    DD S[NB][NB], b[NB], R[NB][NB], qty[NB];
    int perm[NB];
    int idx = 0;
    for (int i = 0; i < NB; ++i)
        for (int j = i; j < NB; ++j) {
            S[i][j] = gram[idx];
            S[j][i] = gram[idx];
            ++idx;
        }
    for (int i = 0; i < NB; ++i) {
        b[i] = gram[idx + i];
        perm[i] = i;
        qty[i] = dd_from(0.0);
        for (int j = 0; j < NB; ++j) R[i][j] = dd_from(0.0);
    }
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < na; ++j) S[i][j] = dd_norm(S[i][j]);
    for (int i = 0; i < na; ++i) b[i] = dd_norm(b[i]);
    const int dcount = static_cast<int>(rows) < na ? static_cast<int>(rows) : na;
    const DD* rounded_squares = gram + idx + NB;
    double diag[NB];
    for (int p = 0; p < dcount; ++p) {
        // pivot: the largest remaining squared norm, ties to the smaller basis column
        int sel = p;
        if (p == 0) {
            double best = -1.0;
            for (int c = 0; c < na; ++c) {
                const double sn = dd_round(rounded_squares[c]);
                if (sn > best || (sn == best && perm[c] < perm[sel])) {
                    sel = c;
                    best = sn;
                }
            }
        } else {
            DD best = S[p][p];
            for (int c = p + 1; c < na; ++c)
                if (dd_greater(S[c][c], best) || (dd_equal(S[c][c], best) && perm[c] < perm[sel])) {
                    sel = c;
                    best = S[c][c];
                }
        }
        if (sel != p) {
            for (int k = 0; k < na; ++k) {
                const DD t = S[k][p];
                S[k][p] = S[k][sel];
                S[k][sel] = t;
            }
            for (int k = 0; k < na; ++k) {
                const DD t = S[p][k];
                S[p][k] = S[sel][k];
                S[sel][k] = t;
            }
            for (int k = 0; k < p; ++k) {
                const DD t = R[k][p];
                R[k][p] = R[k][sel];
                R[k][sel] = t;
            }
            const DD tb = b[p];
            b[p] = b[sel];
            b[sel] = tb;
            const int tp = perm[p];
            perm[p] = perm[sel];
            perm[sel] = tp;
        }
        if (!(S[p][p].hi > 0.0)) {  // an exactly zero remaining column (lsm.rs:2461-2465)
            diag[p] = 0.0;
            continue;
        }
        const DD r = dd_sqrt(S[p][p]);
        R[p][p] = r;
        for (int c = p + 1; c < na; ++c) R[p][c] = dd_div(S[p][c], r);
        for (int i = p + 1; i < na; ++i)
            for (int j = p + 1; j < na; ++j) S[i][j] = dd_sub(S[i][j], dd_mul(R[p][i], R[p][j]));
        // forward substitution R^T qty = b
        DD acc = b[p];
        for (int k = 0; k < p; ++k) acc = dd_sub(acc, dd_mul(R[k][p], qty[k]));
        qty[p] = dd_div(acc, r);
        diag[p] = fabs(dd_round(r));
    }
    const double first = dcount > 0 ? diag[0] : 0.0;
    const double threshold = fmax(A.abs_tol, A.rel_tol * first);
    int rank = 0;
    while (rank < dcount && diag[rank] > threshold) ++rank;
    DD coef[NB];
    for (int i = 0; i < NB; ++i) coef[i] = dd_from(0.0);
    for (int r = rank - 1; r >= 0; --r) {
        DD acc = qty[r];
        for (int k = r + 1; k < rank; ++k) acc = dd_sub(acc, dd_mul(R[r][k], coef[k]));
        coef[r] = dd_div(acc, R[r][r]);
    }
    m.regression = 1;
    m.active_columns = static_cast<uint32_t>(na);
    m.diagonal_count = static_cast<uint32_t>(dcount);
    m.rank = static_cast<uint32_t>(rank);
    m.rank_threshold = threshold;
    for (int k = 0; k < kLsmMaxBasis; ++k) {
        m.pivot_order[k] = 0;
        m.diagonal_abs[k] = 0.0;
        m.coefficients[k] = 0.0;
    }
    for (int k = 0; k < na; ++k) m.pivot_order[k] = static_cast<uint32_t>(perm[k]);
    for (int k = 0; k < dcount; ++k) m.diagonal_abs[k] = diag[k];
    for (int k = 0; k < na; ++k) m.coefficients[perm[k]] = dd_round(coef[k]);
    for (int k = 0; k < NB; ++k)
        if (!isfinite(m.coefficients[k])) lsm_fail(A.lsm_error, static_cast<uint32_t>(d));
}

// Gram matrix and right-hand side of date `d` over its ITM rows; the last CTA
// solves and publishes the date's decision model.
template <int NB>
__global__ void __launch_bounds__(kLsmThreads) lsm_gram_kernel(const LsmArgs A, int d) {
    constexpr int K = NB * (NB + 1) / 2 + 2 * NB;
    static_assert(K <= kLsmPartials && K <= kLsmThreads, "partials stride too small");
    __shared__ DD s_red[kLsmWarps * K];
    __shared__ DD s_fin[K];
    const mcg_lsm_date_model m = A.models[d];
    if (m.itm_rows == 0) return;  // ContinueAll { ZeroItmTrainingPaths }
    const bool inactive = m.feature_inactive != 0;
    const double df_d = A.df[d];
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    DD acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = {0.0, 0.0};
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.paths; p += stride) {
        const double x = A.spots[static_cast<size_t>(d) * A.paths + p];
        if (!(intrinsic(A.side, A.strike, A.notional, x) > A.itm_tol)) continue;
        const double z = inactive ? 0.0 : (x - m.feature_mean) / m.feature_scale;
        double bv[NB];
        bv[0] = 1.0;
#pragma unroll
        for (int e = 1; e < NB; ++e) bv[e] = bv[e - 1] * z;
        const double y = A.cf[p] / df_d;
        int idx = 0;
#pragma unroll
        for (int i = 0; i < NB; ++i)
#pragma unroll
            for (int j = i; j < NB; ++j) {
                acc[idx] = acc_prod(acc[idx], bv[i], bv[j]);
                ++idx;
            }
#pragma unroll
        for (int i = 0; i < NB; ++i) acc[idx + i] = acc_prod(acc[idx + i], bv[i], y);
#pragma unroll
        for (int i = 0; i < NB; ++i) acc[idx + NB + i] = acc_add(acc[idx + NB + i], bv[i] * bv[i]);
    }
    if (!cta_reduce_publish<K>(acc, A.partials, &A.tickets[2], s_red)) return;
    merge_partials<K>(A.partials, s_fin);
    if (threadIdx.x == 0) {
        lsm_solve<NB>(A, d, s_fin);
        A.tickets[2] = 0;
    }
}

// ------------------------------------------------------------------ valuation


// A valuation path generated and stopped by the fitted policy in one pass
// (value_exercise_policy, lsm.rs:1347-1482): exercise at the first date whose
// immediate value beats the predicted continuation value.
__global__ void __launch_bounds__(kLsmThreads) lsm_bs_value_kernel(const DevicePlan P, LsmValueArgs V) {
    extern __shared__ unsigned int s_counts[];
    for (uint32_t i = threadIdx.x; i < V.dates; i += blockDim.x) s_counts[i] = 0;
    __syncthreads();
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (point < P.units) {
        NormalSource ns;
        ns.rqmc = P.engine == MCG_ENGINE_RQMC;
        ns.seed = P.seed;
        ns.unit = point;
        ns.gray = static_cast<uint32_t>(point ^ (point >> 1));
        ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
        ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
        ns.cached_block = 0xffffffffu;
        ns.domain = 0;
        const uint64_t unit = static_cast<uint64_t>(scramble) * P.units + point;
        const int pairs = P.antithetic ? 2 : 1;
        const uint32_t n = P.observation_count;
        double w[2] = {0.0, 0.0};
        double realized[2] = {0.0, 0.0};
        uint32_t stop[2] = {n - 1, n - 1};
        bool open[2] = {true, pairs == 2};
        for (uint32_t i = 0; i < n && (open[0] || open[1]); ++i) {
            const double z = P.zero_variance ? 0.0 : ns.normal(i);
            const double t = P.obs_time[i];
            const double tv = P.vol * P.vol * t;
            for (int e = 0; e < pairs; ++e) {
                const double ze = e == 0 ? z : -z;
                double f;
                if (n == 1) {
                    f = P.obs_fwd[0] * 1.0 * exp(-0.5 * tv + sqrt(tv) * ze);
                } else {
                    w[e] += P.obs_sqrt_step[i] * ze;
                    f = P.obs_fwd[i] * 1.0 * exp(-0.5 * tv + P.vol * w[e]);
                }
                if (!open[e]) continue;
                const double imm = intrinsic(V.side, V.strike, V.notional, f);
                if (i + 1 == n) {
                    realized[e] = imm;
                    open[e] = false;
                } else if (V.models[i].regression && imm > predict(policy_of(V.models[i], V.nb), V.nb, f)) {
                    realized[e] = imm;
                    stop[e] = i;
                    open[e] = false;
                }
            }
        }
        const double d0 = realized[0] * V.df[stop[0]];
        double value = d0;
        if (pairs == 2) value = (d0 + realized[1] * V.df[stop[1]]) * 0.5;
        V.unit_values[unit] = value;
        for (int e = 0; e < pairs; ++e) {
            atomicAdd(&s_counts[stop[e]], 1u);
            if (V.stops) V.stops[unit * pairs + e] = stop[e];
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < V.dates; i += blockDim.x)
        if (s_counts[i]) atomicAdd(&V.counts[i], static_cast<unsigned long long>(s_counts[i]));
}

// ----------------------------------------------------------------- reductions

// Sum of per-unit values of each group (blockIdx.y): the value itself, the
// antithetic pair mean (v[2i] + v[2i+1]) * 0.5, or -- with `centers` -- the
// squared deviation from the group's centre.  Partials per CTA.
__global__ void __launch_bounds__(kLsmThreads) lsm_group_sum_kernel(const double* values, uint64_t per_group,
                                                                    int pairs, const double* centers,
                                                                    DD* partials) {
    __shared__ DD s_red[kLsmWarps];
    const uint32_t g = blockIdx.y;
    const double* v = values + static_cast<size_t>(g) * per_group * (pairs ? 2u : 1u);
    const double c = centers ? centers[g] : 0.0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    DD acc = {0.0, 0.0};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < per_group; i += stride) {
        double x = pairs ? (v[2 * i] + v[2 * i + 1]) * 0.5 : v[i];
        if (centers) {
            const double dv = x - c;
            x = dv * dv;
        }
        acc = acc_add(acc, x);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    acc = warp_reduce_dd(acc);
    if (lane == 0) s_red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        DD m = s_red[0];
        for (int w = 1; w < kLsmWarps; ++w) m = acc_merge(m, s_red[w]);
        partials[static_cast<size_t>(g) * gridDim.x + blockIdx.x] = m;
    }
}

// Merges the partials of each group in CTA order; out[g] = {hi, lo} and
// means[g] = rounded sum / per_group.
__global__ void lsm_group_finish_kernel(const DD* partials, uint32_t ctas, uint64_t per_group, DD* out,
                                        double* means) {
    const uint32_t g = blockIdx.x;
    const int lane = threadIdx.x;
    DD acc = {0.0, 0.0};
    for (uint32_t b = lane; b < ctas; b += 32) acc = acc_merge(acc, partials[static_cast<size_t>(g) * ctas + b]);
    acc = warp_reduce_dd(acc);
    if (lane == 0) {
        out[g] = acc;
        if (means) means[g] = dd_round(acc) / static_cast<double>(per_group);
    }
}

// ------------------------------------------------------------------ launchers

cudaError_t launch_lsm_bs_spots(const DevicePlan& P, uint32_t domain, double* spots, uint64_t paths,
                                unsigned long long* bad, cudaStream_t stream) {
    const dim3 grid(static_cast<unsigned>((P.units + kLsmThreads - 1) / kLsmThreads), P.scramble_count);
    lsm_bs_spots_kernel<<<grid, kLsmThreads, 0, stream>>>(P, domain, spots, paths, bad);
    return cudaGetLastError();
}

cudaError_t launch_lsm_sweep(const LsmArgs& A, unsigned ctas, int init, int update, int gather,
                             cudaStream_t stream) {
    lsm_sweep_kernel<<<ctas, kLsmThreads, 0, stream>>>(A, init, update, gather);
    return cudaGetLastError();
}

cudaError_t launch_lsm_variance(const LsmArgs& A, unsigned ctas, int d, cudaStream_t stream) {
    lsm_variance_kernel<<<ctas, kLsmThreads, 0, stream>>>(A, d);
    return cudaGetLastError();
}

cudaError_t launch_lsm_gram(const LsmArgs& A, unsigned ctas, int d, cudaStream_t stream) {
    switch (A.nb) {
    case 2: lsm_gram_kernel<2><<<ctas, kLsmThreads, 0, stream>>>(A, d); break;
    case 3: lsm_gram_kernel<3><<<ctas, kLsmThreads, 0, stream>>>(A, d); break;
    case 4: lsm_gram_kernel<4><<<ctas, kLsmThreads, 0, stream>>>(A, d); break;
    case 5: lsm_gram_kernel<5><<<ctas, kLsmThreads, 0, stream>>>(A, d); break;
    case 6: lsm_gram_kernel<6><<<ctas, kLsmThreads, 0, stream>>>(A, d); break;
    case 7: lsm_gram_kernel<7><<<ctas, kLsmThreads, 0, stream>>>(A, d); break;
    case 8: lsm_gram_kernel<8><<<ctas, kLsmThreads, 0, stream>>>(A, d); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_lsm_bs_value(const DevicePlan& P, const LsmValueArgs& V, cudaStream_t stream) {
    const dim3 grid(static_cast<unsigned>((P.units + kLsmThreads - 1) / kLsmThreads), P.scramble_count);
    lsm_bs_value_kernel<<<grid, kLsmThreads, V.dates * sizeof(unsigned int), stream>>>(P, V);
    return cudaGetLastError();
}

cudaError_t launch_lsm_group_sum(const double* values, uint64_t per_group, uint32_t groups, int pairs,
                                 const double* centers, DD* partials, unsigned ctas, DD* out, double* means,
                                 cudaStream_t stream) {
    lsm_group_sum_kernel<<<dim3(ctas, groups), kLsmThreads, 0, stream>>>(values, per_group, pairs, centers,
                                                                         partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    lsm_group_finish_kernel<<<groups, 32, 0, stream>>>(partials, ctas, per_group, out, means);
    return cudaGetLastError();
}

size_t lsm_partial_stride() { return kLsmPartials; }

}  // namespace mcg

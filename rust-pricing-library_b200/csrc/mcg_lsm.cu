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
// Backward induction: one launch per non-terminal date d.  Each thread takes
// its paths through the decision of date d+1 (exercise if immediate >
// continuation, summing that fit's residuals) and, with the updated cash
// flow, adds its ITM rows of date d to power sums of the spot about a centre
// c near their mean, P_k = sum (S - c)^k (k <= 2 degree) and T_k = sum (S - c)^k y.
// Mean, population variance and the Gram matrix of the standardised monomial
// basis all follow from these sums by a binomial shift, so one pass replaces
// the reference's three (scaling, design matrix, QR).  Every sum is a
// compensated (TwoSum) double-double accumulation reduced in a fixed order.  The last CTA to finish (a
// ticket counter, no waiting) merges the per-CTA partials and fits the date.
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


constexpr int kLsmPartials = (2 * kLsmMaxBasis - 1) + kLsmMaxBasis + 2;  // step-kernel sums + count/max

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

// In the last CTA: merges the partials of every CTA.  Components k < K are
// double-double sums; with EXTRA, component K is a (count, max) pair.  Thread
// (k, g) of C = K + EXTRA components and G = threads / C groups merges the
// CTAs g, g + G, ... of component k; thread k then merges the G groups in
// order into out[k].  Deterministic for a given grid.
template <int K, bool EXTRA>
__device__ void merge_partials(const DD* partials, DD* out) {
    constexpr int C = K + (EXTRA ? 1 : 0);
    constexpr int G = kLsmThreads / C;
    __shared__ DD s_part[kLsmThreads];
    const int t = threadIdx.x;
    const int k = t % C, g = t / C;
    const bool pair = EXTRA && k == K;
    DD acc = {0.0, pair ? 1.0 : 0.0};
    if (g < G) {
#pragma unroll 4
        for (uint32_t b = g; b < gridDim.x; b += G) {
            const DD* p = partials + static_cast<size_t>(b) * kLsmPartials + k;
            const DD q = {__ldcg(&p->hi), __ldcg(&p->lo)};
            if (pair) {
                acc.hi += q.hi;  // counts: exact integers below 2^53
                acc.lo = fmax(acc.lo, q.lo);
            } else {
                acc = acc_merge(acc, q);
            }
        }
    }
    s_part[t] = acc;
    __syncthreads();
    if (t < C) {
        DD m = s_part[t];
        for (int gg = 1; gg < G; ++gg) {
            const DD q = s_part[gg * C + t];
            if (pair) {
                m.hi += q.hi;
                m.lo = fmax(m.lo, q.lo);
            } else {
                m = acc_merge(m, q);
            }
        }
        out[t] = m;
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

// ------------------------------------------------------------- training step

// Adds a double-double value to an accumulator.
__device__ __forceinline__ DD acc_add_dd(DD a, DD b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    return {s, a.lo + (e + b.lo)};
}

// Binomial coefficients for the shift of the power sums.
__device__ __forceinline__ double binomial(int n, int k) {
    // C(n, k) = n! / (k! (n - k)!) by the multiplicative formula over exact
    // integers (every intermediate product is an integer below 2^53).
    double c = 1.0;
    for (int i = 1; i <= k; ++i) c = (c * static_cast<double>(n - k + i)) / static_cast<double>(i);
    return c;
}

// The CPQR-equivalent solve of one date, run by one thread.  G (NB x NB) and
// r (NB) are the Gram matrix and right-hand side of the standardised monomial
// basis, double-double.  Pivoted Cholesky: the pivot is the largest remaining
// squared column norm (the Schur-complement diagonal), ties to the smaller
// basis column, as fit_cpqr chooses (lsm.rs:2441-2459); |R_kk|, the rank
// threshold max(abs, rel * |R_00|) and the back substitution over the leading
// `rank` pivots follow lsm.rs:2500-2533.
template <int NB>
__device__ void lsm_solve(const LsmArgs& A, mcg_lsm_date_model& m, int na, DD (&S)[NB][NB], DD (&b)[NB]) {
    // Every array index below is a compile-time constant after unrolling, so
    // the factorisation lives in registers; pivot swaps are predicated.
    DD R[NB][NB], qty[NB], inv_diag[NB];
    int perm[NB];
    double diag[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        perm[i] = i;
        qty[i] = dd_from(0.0);
        diag[i] = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j) R[i][j] = dd_from(0.0);
    }
    const int dcount = static_cast<int>(m.itm_rows) < na ? static_cast<int>(m.itm_rows) : na;
#pragma unroll
    for (int p = 0; p < NB; ++p) {
        if (p >= dcount) break;
        int sel = p;
        DD best = S[p][p];
        int best_perm = perm[p];
#pragma unroll
        for (int c = p + 1; c < NB; ++c) {
            if (c >= na) break;
            if (dd_greater(S[c][c], best) || (dd_equal(S[c][c], best) && perm[c] < best_perm)) {
                sel = c;
                best = S[c][c];
                best_perm = perm[c];
            }
        }
#pragma unroll
        for (int c = p + 1; c < NB; ++c) {
            if (c != sel) continue;
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                const DD t = S[k][p];
                S[k][p] = S[k][c];
                S[k][c] = t;
            }
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                const DD t = S[p][k];
                S[p][k] = S[c][k];
                S[c][k] = t;
            }
#pragma unroll
            for (int k = 0; k < p; ++k) {
                const DD t = R[k][p];
                R[k][p] = R[k][c];
                R[k][c] = t;
            }
            const DD tb = b[p];
            b[p] = b[c];
            b[c] = tb;
            const int tp = perm[p];
            perm[p] = perm[c];
            perm[c] = tp;
        }
        if (!(S[p][p].hi > 0.0)) continue;  // an exactly zero remaining column (lsm.rs:2461-2465)
        const DD r = dd_sqrt(S[p][p]);
        const DD inv_r = dd_div(dd_from(1.0), r);
        R[p][p] = r;
        inv_diag[p] = inv_r;
#pragma unroll
        for (int c = p + 1; c < NB; ++c)
            if (c < na) R[p][c] = dd_mul(S[p][c], inv_r);
#pragma unroll
        for (int i = p + 1; i < NB; ++i)
#pragma unroll
            for (int j = i; j < NB; ++j)
                if (j < na) {
                    S[i][j] = dd_sub(S[i][j], dd_mul(R[p][i], R[p][j]));
                    S[j][i] = S[i][j];
                }
        DD acc = b[p];
#pragma unroll
        for (int k = 0; k < p; ++k) acc = dd_sub(acc, dd_mul(R[k][p], qty[k]));
        qty[p] = dd_mul(acc, inv_r);
        diag[p] = fabs(dd_round(r));
    }
    const double first = dcount > 0 ? diag[0] : 0.0;
    const double threshold = fmax(A.abs_tol, A.rel_tol * first);
    int rank = 0;
#pragma unroll
    for (int p = 0; p < NB; ++p)
        if (rank == p && p < dcount && diag[p] > threshold) ++rank;
    DD coef[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) coef[i] = dd_from(0.0);
#pragma unroll
    for (int r = NB - 1; r >= 0; --r) {
        if (r >= rank) continue;
        DD acc = qty[r];
#pragma unroll
        for (int k = r + 1; k < NB; ++k)
            if (k < rank) acc = dd_sub(acc, dd_mul(R[r][k], coef[k]));
        coef[r] = dd_mul(acc, inv_diag[r]);
    }
    m.regression = 1;
    m.active_columns = static_cast<uint32_t>(na);
    m.diagonal_count = static_cast<uint32_t>(dcount);
    m.rank = static_cast<uint32_t>(rank);
    m.rank_threshold = threshold;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        if (k < na) m.pivot_order[k] = static_cast<uint32_t>(perm[k]);
        if (k < dcount) m.diagonal_abs[k] = diag[k];
    }
    // coefficients back in basis order: coefficient of column perm[k] is coef[k]
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < NB; ++k)
            if (k < na && perm[k] == c) v = dd_round(coef[k]);
        m.coefficients[c] = v;
    }
}

// Fits date `d` from its merged sums, in the last CTA (every thread calls
// it): n ITM rows, max |S|, the power sums P_k = sum (S - c)^k, k < 2 NB - 1,
// about the date's centre c, and T_k = sum (S - c)^k y, k < NB, of the
// targets y.  The feature scaling of FeatureScaling::fit (lsm.rs:537-574) comes
// from the mean m = (n c + P_1) / n and the central sums M_k = sum (S - m)^k,
// obtained from the P_k by the binomial shift in double-double (one thread per
// k); the standardised Gram matrix is M_{i+j} / s^{i+j} (one thread per
// entry); one thread factorises.  The mean becomes the centre of date d - 1.
template <int NB>
__device__ void lsm_fit_date(const LsmArgs& A, int d, unsigned long long n, double maxabs, const DD* P,
                             const DD* T) {
    constexpr int NP = 2 * NB - 1;
    __shared__ DD s_M[NP], s_U[NB], s_G[NB][NB], s_rhs[NB], s_inv[NP];
    __shared__ int s_go;
    mcg_lsm_date_model& m = A.models[d];
    const double c = A.centers[d];
    const double nd = static_cast<double>(n);
    // sum.total() / len and squared_deviations.total() / len: the rounded sum,
    // then one division, as the reference rounds them.
    const double mean = n ? dd_round(dd_add(dd_mul_d(dd_from(c), nd), dd_norm(P[1]))) / nd : 0.0;
    double dh, dl;
    two_sum(mean, -c, dh, dl);  // delta = mean - c exactly
    const DD neg_delta = dd_neg(quick_two_sum(dh, dl));
    const int t = threadIdx.x;
    if (n && t < NP + NB) {
        // t < NP: M_t = sum_j C(t, j) (-delta)^(t - j) P_j; else U_i likewise from T.
        const int k = t < NP ? t : t - NP;
        const DD* src = t < NP ? P : T;
        DD acc = dd_from(0.0), pw = dd_from(1.0);
        for (int j = k; j >= 0; --j) {
            acc = dd_add(acc, dd_mul(dd_mul_d(pw, binomial(k, j)), dd_norm(src[j])));
            pw = dd_mul(pw, neg_delta);
        }
        if (t < NP) s_M[k] = acc;
        else s_U[k] = acc;
    }
    __syncthreads();
    if (t == 0) {
        m.candidate_rows = static_cast<uint32_t>(A.paths);
        m.itm_rows = static_cast<uint32_t>(n);
        m.regression = 0;
        s_go = 0;
        if (n && d > 0) A.centers[d - 1] = mean;
        if (n == 0) {
            // ContinueAll { ZeroItmTrainingPaths }
        } else if (n > A.max_elements) {
            lsm_fail(A.lsm_error, static_cast<uint32_t>(d));
        } else {
            const double variance = dd_round(s_M[2]) / nd;
            const double scale = sqrt(variance);
            const double threshold = (64.0 * kEpsilon64) * maxabs;
            const bool inactive = scale <= threshold;
            m.feature_mean = mean;
            m.feature_variance = variance;
            m.feature_scale = scale;
            m.zero_scale_threshold = threshold;
            m.feature_inactive = inactive ? 1 : 0;
            if (n * static_cast<unsigned long long>(inactive ? 1 : NB) > A.max_elements) {
                lsm_fail(A.lsm_error, static_cast<uint32_t>(d));
            } else {
                const DD inv_s = inactive ? dd_from(0.0) : dd_div(dd_from(1.0), dd_from(scale));
                s_inv[0] = dd_from(1.0);
                for (int k = 1; k < NP; ++k) s_inv[k] = dd_mul(s_inv[k - 1], inv_s);
                s_go = 1;
            }
        }
    }
    __syncthreads();
    if (!s_go) return;
    if (t < NB * NB) {
        const int i = t / NB, j = t % NB;
        s_G[i][j] = dd_mul(s_M[i + j], s_inv[i + j]);
    } else if (t < NB * NB + NB) {
        const int i = t - NB * NB;
        s_rhs[i] = dd_mul(s_U[i], s_inv[i]);
    }
    __syncthreads();
    if (t == 0) {
        DD G[NB][NB], rhs[NB];
        for (int i = 0; i < NB; ++i) {
            rhs[i] = s_rhs[i];
            for (int j = 0; j < NB; ++j) G[i][j] = s_G[i][j];
        }
        lsm_solve<NB>(A, m, m.feature_inactive ? 1 : NB, G, rhs);
        for (int k = 0; k < NB; ++k)
            if (!isfinite(m.coefficients[k])) lsm_fail(A.lsm_error, static_cast<uint32_t>(d));
    }
}

// The expiry cash flows cf = immediate(T) * df(T), stop = T of every training
// path, and the mean of the ITM spots of the last non-terminal date, the
// centre of that date's power sums.
__global__ void __launch_bounds__(kLsmThreads) lsm_init_kernel(const LsmArgs A) {
    __shared__ DD s_red[kLsmWarps];
    __shared__ DD s_fin[2];
    __shared__ unsigned long long s_cnt[kLsmWarps];
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint32_t last = A.dates - 1;
    double sum = 0.0;
    unsigned long long cnt = 0;
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.paths; p += stride) {
        const double x = A.spots[static_cast<size_t>(last) * A.paths + p];
        A.cf[p] = intrinsic(A.side, A.strike, A.notional, x) * A.df[last];
        A.stop[p] = last;
        if (last > 0) {
            const double g = A.spots[static_cast<size_t>(last - 1) * A.paths + p];
            if (intrinsic(A.side, A.strike, A.notional, g) > A.itm_tol) {
                ++cnt;
                sum += g;
            }
        }
    }
    DD acc[1] = {{sum, 0.0}};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    if (lane == 0) s_cnt[warp] = cnt;
    __syncthreads();
    DD extra = {0.0, 0.0};
    if (threadIdx.x == 0) {
        unsigned long long total = 0;
        for (int w = 0; w < kLsmWarps; ++w) total += s_cnt[w];
        extra = {static_cast<double>(total), 0.0};
    }
    if (!cta_reduce_publish<1>(acc, A.partials, &A.tickets[1], s_red, &extra)) return;
    merge_partials<1, true>(A.partials, s_fin);
    if (threadIdx.x == 0) {
        const unsigned long long n = static_cast<unsigned long long>(s_fin[1].hi);
        if (n && last > 0) A.centers[last - 1] = dd_round(s_fin[0]) / static_cast<double>(n);
        A.tickets[1] = 0;
    }
}

// One backward-induction step over every training path, one launch per date:
//   * `update` >= 0: the decision of that date (exercise when immediate >
//     continuation, for every path, lsm.rs:1604-1614) and the residual squares
//     of its ITM rows against the pre-update targets (the fit's residual sum,
//     lsm.rs:2535-2550);
//   * `gather` >= 0: the ITM rows of that date with their targets cf / df
//     (lsm.rs:1586-1597) after the update, as compensated power sums of
//     u = S - c about the date's centre c (the ITM mean of the next date, close
//     to this date's mean, so the binomial shift to the exact mean amplifies
//     the per-term rounding of u^k by a factor near one).
// The last CTA merges every CTA's sums in CTA order and fits `gather`.
template <int NB>
__global__ void __launch_bounds__(kLsmThreads, 2) lsm_step_kernel(const LsmArgs A, int update, int gather) {
    constexpr int NP = 2 * NB - 1;
    constexpr int K = NP + NB + 1;  // power sums, target sums, residual squares
    static_assert(K + 1 <= kLsmPartials && K <= kLsmThreads && NB * NB + NB <= kLsmThreads,
                  "partials stride or CTA too small");
    __shared__ DD s_red[kLsmWarps * K];
    __shared__ DD s_fin[K + 1];
    __shared__ unsigned long long s_cnt[kLsmWarps];
    __shared__ double s_max[kLsmWarps];
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    Policy mu{};
    if (update >= 0) mu = policy_of(A.models[update], A.nb);
    const bool decide = update >= 0 && mu.regression;
    const double df_u = update >= 0 ? A.df[update] : 1.0;
    const double df_g = gather >= 0 ? A.df[gather] : 1.0;
    const double c = gather >= 0 ? A.centers[gather] : 0.0;
    // Per-thread partial sums are plain (a thread sees a few dozen paths); the
    // cross-thread and cross-CTA merges are double-double.
    double part[K];
#pragma unroll
    for (int k = 0; k < K; ++k) part[k] = 0.0;
    unsigned long long cnt = 0;
    double maxabs = 1.0;
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.paths; p += stride) {
        double cf = A.cf[p];
        if (decide) {
            const double x = A.spots[static_cast<size_t>(update) * A.paths + p];
            const double imm = intrinsic(A.side, A.strike, A.notional, x);
            const double cont = predict(mu, NB, x);
            if (imm > A.itm_tol) {
                const double res = cf / df_u - cont;
                part[K - 1] += res * res;
            }
            if (imm > cont) {
                cf = imm * df_u;
                A.stop[p] = static_cast<uint32_t>(update);
            }
        }
        if (decide) A.cf[p] = cf;
        if (gather >= 0) {
            const double x = A.spots[static_cast<size_t>(gather) * A.paths + p];
            if (intrinsic(A.side, A.strike, A.notional, x) > A.itm_tol) {
                ++cnt;
                maxabs = fmax(maxabs, fabs(x));
                const double u = x - c;
                const double y = cf / df_g;
                double pw = 1.0;
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    if (k) pw *= u;
                    part[k] += pw;
                    if (k < NB) part[NP + k] += pw * y;
                }
            }
        }
    }
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
        unsigned long long total = 0;
        double mx = 1.0;
        for (int w = 0; w < kLsmWarps; ++w) {
            total += s_cnt[w];
            mx = fmax(mx, s_max[w]);
        }
        extra = {static_cast<double>(total), mx};
    }
    DD acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = {part[k], 0.0};
    if (!cta_reduce_publish<K>(acc, A.partials, &A.tickets[0], s_red, &extra)) return;
    merge_partials<K, true>(A.partials, s_fin);
    const unsigned long long n = static_cast<unsigned long long>(s_fin[K].hi);
    const double mx = s_fin[K].lo;
    if (threadIdx.x == 0) {
        if (decide) A.models[update].residual_sum_squares = dd_round(s_fin[K - 1]);
        A.tickets[0] = 0;
    }
    if (gather >= 0) lsm_fit_date<NB>(A, gather, n, mx, s_fin, s_fin + NP);
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
        const double* row = V.spots ? V.spots + unit * pairs : nullptr;
        for (uint32_t i = 0; i < n && (open[0] || open[1]); ++i) {
            const double z = (P.zero_variance || row) ? 0.0 : ns.normal(i);
            const double t = P.obs_time[i];
            const double tv = P.vol * P.vol * t;
            for (int e = 0; e < pairs; ++e) {
                const double ze = e == 0 ? z : -z;
                double f;
                if (row) {
                    f = row[static_cast<size_t>(i) * V.paths + e];
                } else if (n == 1) {
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

// ------------------------------------------------------------ fixed-policy risk

// Price, AAD delta and AAD vega of one path's exercise cash flow at stopping
// date k under (spot, vol): pathwise_aad_for_output
// (crates/pricing/src/engine/processes/black_scholes.rs:567-643) for the
// American payoff graph's output k, observation k of
// path_observations_from_normals (:297-331).  `w` is the path's Brownian
// value at t_k, `z` its first normal (single-date plans take the exact
// terminal step sqrt(sigma^2 t) z).
struct ExerciseAad {
    double price, delta, vega;
};

__device__ __forceinline__ ExerciseAad exercise_aad(const DevicePlan& P, const LsmRiskArgs& R, uint32_t k,
                                                    double w, double z, double spot, double vol) {
    const double t = P.obs_time[k];
    const double tv = vol * vol * t;
    const double lr = P.observation_count == 1 ? -0.5 * tv + sqrt(tv) * z : -0.5 * tv + vol * w;
    const double f = P.obs_fwd[k] * (spot / P.spot) * exp(lr);
    const double s = 0.0 * spot + 1.0 * f;
    const bool call = R.side == MCG_CALL;
    const double in = call ? s - R.strike : R.strike - s;
    const double value = (in >= 0.0 ? in : 0.0) * R.notional;
    const double adj = (in >= 0.0 ? R.notional : 0.0) * (call ? 1.0 : -1.0);
    double delta = 0.0, vega = 0.0;
    if (adj != 0.0) {
        delta += adj * 1.0 * f / spot;
        vega += adj * 1.0 * f * (-vol * t + w);
    }
    const double df = R.df[k];
    return {df * value, df * delta, df * vega};
}

// The ten pathwise components of fixed_policy_pathwise_values
// (black_scholes.rs:358-415): base price/delta/vega, gamma from the AAD deltas
// at spot +- gamma_bump, bumped delta/gamma from prices at spot +- spot_bump,
// bumped vega from prices at vol +- vol_bump, and the differences.
__device__ __forceinline__ void fixed_policy_values(const DevicePlan& P, const LsmRiskArgs& R, uint32_t k,
                                                    double w, double z, double (&v)[kComponents]) {
    const double S = P.spot, vol = P.vol;
    const ExerciseAad base = exercise_aad(P, R, k, w, z, S, vol);
    double gamma = 0.0;
    if (R.gamma) {
        const double b = R.gamma_bump;
        const double dd = exercise_aad(P, R, k, w, z, S - b, vol).delta;
        const double du = exercise_aad(P, R, k, w, z, S + b, vol).delta;
        gamma = (du - dd) / (2.0 * b);
    }
    const double sb = R.spot_bump;
    const double pd = exercise_aad(P, R, k, w, z, S - sb, vol).price;
    const double pu = exercise_aad(P, R, k, w, z, S + sb, vol).price;
    const double bump_delta = (pu - pd) / (2.0 * sb);
    const double bump_gamma = (pu - 2.0 * base.price + pd) / (sb * sb);
    double bump_vega = 0.0;
    if (R.vol_bump != 0.0) {
        const double vb = R.vol_bump;
        const double lo = exercise_aad(P, R, k, w, z, S, vol - vb).price;
        const double hi = exercise_aad(P, R, k, w, z, S, vol + vb).price;
        bump_vega = (hi - lo) / (2.0 * vb);
    }
#pragma unroll
    for (int c = 0; c < kComponents; ++c) v[c] = 0.0;
    v[MCG_PRICE] = base.price;
    v[MCG_DELTA] = base.delta;
    v[MCG_VEGA] = base.vega;
    v[MCG_GAMMA] = gamma;
    v[MCG_BUMP_DELTA] = bump_delta;
    v[MCG_DELTA_DIFFERENCE] = bump_delta - base.delta;
    v[MCG_BUMP_VEGA] = bump_vega;
    v[MCG_VEGA_DIFFERENCE] = bump_vega - base.vega;
    v[MCG_BUMP_GAMMA] = bump_gamma;
    v[MCG_GAMMA_DIFFERENCE] = bump_gamma - gamma;
}

// One thread per sampling unit: regenerate the unit's normals up to the later
// stopping date of its (antithetic) paths, evaluate the components of each
// path at its own stopping date, average the pair, reduce per 128-unit tile
// (constant_vol_fixed_policy_pseudo/rqmc_statistics,
// crates/pricing/src/engine/mc/early_exercise.rs:454-600).
__global__ void __launch_bounds__(kThreads) lsm_bs_risk_kernel(const DevicePlan P, const LsmRiskArgs R,
                                                               StatRecord* partials) {
    __shared__ Stat s_red[4 * kComponents];
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < P.units;
    const uint64_t unit = valid ? point : 0;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = unit;
    ns.gray = static_cast<uint32_t>(unit ^ (unit >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    ns.domain = 0;
    const int pairs = P.antithetic ? 2 : 1;
    const uint32_t n = P.observation_count;
    const uint64_t base = (static_cast<uint64_t>(scramble) * P.units + unit) * pairs;
    uint32_t k[2] = {min(R.stops[base], n - 1), pairs == 2 ? min(R.stops[base + 1], n - 1) : 0u};
    const uint32_t last = max(k[0], k[1]);
    double w[2] = {0.0, 0.0}, wk[2] = {0.0, 0.0}, z0 = 0.0;
    for (uint32_t i = 0; i <= last; ++i) {
        const double z = P.zero_variance ? 0.0 : ns.normal(i);
        if (i == 0) z0 = z;
        for (int e = 0; e < pairs; ++e) {
            const double ze = e == 0 ? z : -z;
            w[e] += P.obs_sqrt_step[i] * ze;
            if (i == k[e]) wk[e] = w[e];
        }
    }
    double vals[kComponents];
    fixed_policy_values(P, R, k[0], wk[0], z0, vals);
    if (pairs == 2) {
        double mate[kComponents];
        fixed_policy_values(P, R, k[1], wk[1], -z0, mate);
#pragma unroll
        for (int c = 0; c < kComponents; ++c) vals[c] = (vals[c] + mate[c]) * 0.5;
    }
    StatRecord* out = partials + (static_cast<size_t>(scramble) * gridDim.x + blockIdx.x) * kComponents;
    cta_reduce_write<kComponents>(vals, valid, 0x3ffu, out, s_red);
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

cudaError_t launch_lsm_init(const LsmArgs& A, unsigned ctas, cudaStream_t stream) {
    lsm_init_kernel<<<ctas, kLsmThreads, 0, stream>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_lsm_step(const LsmArgs& A, unsigned ctas, int update, int gather, cudaStream_t stream) {
    switch (A.nb) {
    case 2: lsm_step_kernel<2><<<ctas, kLsmThreads, 0, stream>>>(A, update, gather); break;
    case 3: lsm_step_kernel<3><<<ctas, kLsmThreads, 0, stream>>>(A, update, gather); break;
    case 4: lsm_step_kernel<4><<<ctas, kLsmThreads, 0, stream>>>(A, update, gather); break;
    case 5: lsm_step_kernel<5><<<ctas, kLsmThreads, 0, stream>>>(A, update, gather); break;
    case 6: lsm_step_kernel<6><<<ctas, kLsmThreads, 0, stream>>>(A, update, gather); break;
    case 7: lsm_step_kernel<7><<<ctas, kLsmThreads, 0, stream>>>(A, update, gather); break;
    case 8: lsm_step_kernel<8><<<ctas, kLsmThreads, 0, stream>>>(A, update, gather); break;
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

uint32_t lsm_risk_tiles(uint64_t units) { return static_cast<uint32_t>((units + kThreads - 1) / kThreads); }

cudaError_t launch_lsm_bs_risk(const DevicePlan& P, const LsmRiskArgs& R, StatRecord* partials,
                               cudaStream_t stream) {
    const dim3 grid(lsm_risk_tiles(P.units), P.scramble_count);
    lsm_bs_risk_kernel<<<grid, kThreads, 0, stream>>>(P, R, partials);
    return cudaGetLastError();
}

size_t lsm_partial_stride() { return kLsmPartials; }

}  // namespace mcg

// mcg_kernels.cuh -- path kernels of the B200 Monte Carlo engine.
//
// One thread evaluates one sampling unit (a pseudo-random path or one Sobol
// point of one scramble) from its normals to its 18 pathwise components, in
// registers; a CTA reduces its units into one statistics record per component
// with a fixed-shape tree.  This replaces the per-unit closures that
// DeterministicExecutor runs on a Rayon pool
// (crates/pricing/src/engine/mc/execution.rs:550-726) and the closures of
// crates/pricing/src/engine/risk/valuation.rs:126-437 and
// crates/pricing/src/engine/risk/local_vol.rs:24-420.
#pragma once

#include "mcg_device.cuh"
#include "mcg_payoff.cuh"

namespace mcg {

constexpr int kThreads = 128;

struct ErrorWord {
    unsigned long long key;  // (unit << 8) | code, atomicMin over failing units
    int32_t code;
    uint32_t step;
    unsigned long long unit;
    unsigned long long value_bits;
};

__device__ __forceinline__ void report_error(ErrorWord* err, uint64_t unit, int code, uint32_t step,
                                             double value, bool detail) {
    atomicMin(&err->key, (static_cast<unsigned long long>(unit) << 8) | static_cast<unsigned>(code));
    if (detail) {
        err->code = code;
        err->step = step;
        err->unit = unit;
        err->value_bits = static_cast<unsigned long long>(__double_as_longlong(value));
    }
}

// ----------------------------------------------------------------- normals

// Normal for dimension `dim` of one unit.  RQMC: scrambled Sobol word as
// shift XOR the pre-applied scrambled directions of the set Gray-code bits
// (qmc.rs:71-84,125-132: apply is GF(2)-linear, so apply(XOR v_k) =
// XOR M v_k ^ shift); pseudo: Philox coordinate (unit, dim, domain).
//
// The Gray code of point p splits as gray(p & ~31) ^ gray(p & 31) (the two
// halves of p ^ (p >> 1) touch disjoint bits), so for a warp of 32
// consecutive points the high part is the same in every lane -- a uniform
// loop of broadcast loads -- and the lane part is five predicated XORs.  The
// word is the same XOR of the same directions, bit for bit.
struct NormalSource {
    int32_t rqmc;
    uint64_t seed;
    uint64_t unit;        // pseudo: sampling unit
    uint32_t gray;        // rqmc: Gray code of the point
    const uint32_t* dirs; // rqmc: this scramble's [dim][32] table
    const uint32_t* shift;
    uint32_t cached_block;
    uint4 block;
    uint32_t domain = 0;  // pseudo: RandomDomain (Valuation 0, LsmTrain 1)

    __device__ __forceinline__ uint32_t word(uint32_t dim) {
        if (rqmc) {
            const uint32_t* d = dirs + static_cast<size_t>(dim) * 32u;
            uint32_t x = __ldg(shift + dim);
            const uint32_t low = unit & 31u;
            const uint32_t gl = low ^ (low >> 1);
            uint32_t g = gray ^ gl;  // gray(unit & ~31)
            while (g) {
                const int b = __ffs(g) - 1;
                x ^= __ldg(d + b);
                g &= g - 1u;
            }
#pragma unroll
            for (int b = 0; b < 5; ++b) {
                const uint32_t v = __ldg(d + b);
                x ^= (gl >> b) & 1u ? v : 0u;
            }
            return x;
        }
        const uint32_t blk = dim >> 2;
        if (blk != cached_block) {
            block = philox_block(seed, unit, blk, domain);
            cached_block = blk;
        }
        return lane_of(block, dim & 3u);
    }

    __device__ __forceinline__ double normal(uint32_t dim) { return as241(open_unit(word(dim))); }

    // RQMC word with the whole warp: the 32 lanes hold 32 consecutive points
    // of one 32-aligned block, so gray(p) = gray(p & ~31) ^ gray(p & 31) with
    // the first part common to the warp.  Lane b contributes table word b
    // where bit b of the common part is set (one coalesced load and one XOR
    // reduction); the lane part is the precomputed low word of its lane.
    // Bit-identical to word(); every lane of the warp must call it.
    const uint32_t* low;   // this scramble's [dim][32] low words
    uint32_t high_gray;    // gray(p & ~31), common to the warp
    uint32_t lane_low;     // p & 31
    __device__ __forceinline__ uint32_t word_warp(uint32_t dim) {
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t v = __ldg(dirs + static_cast<size_t>(dim) * 32u + lane);
        const uint32_t h = __reduce_xor_sync(0xffffffffu, (high_gray >> lane) & 1u ? v : 0u);
        return __ldg(shift + dim) ^ h ^ __ldg(low + static_cast<size_t>(dim) * 32u + lane_low);
    }
    __device__ __forceinline__ double normal_warp(uint32_t dim) { return as241(open_unit(word_warp(dim))); }
};

// ------------------------------------------------------- step exponential

// exp of a step's increment.  For |x| < 1/8 (every daily step short of an
// eight-sigma move) the Taylor series of e^x to degree 10 in Horner form with
// fused multiply-adds: the truncation is below x^11/11! < 2.3e-18 relative,
// so the value is within an ulp or two of the library exp; larger arguments
// take the library exp.  The step's result is held to 1e-12 of the reference.
__device__ __forceinline__ double exp_step(double x) {
    if (!(fabs(x) < 0.125)) return exp(x);
    double p = 1.0 / 3628800.0;
    p = fma(p, x, 1.0 / 362880.0);
    p = fma(p, x, 1.0 / 40320.0);
    p = fma(p, x, 1.0 / 5040.0);
    p = fma(p, x, 1.0 / 720.0);
    p = fma(p, x, 1.0 / 120.0);
    p = fma(p, x, 1.0 / 24.0);
    p = fma(p, x, 1.0 / 6.0);
    p = fma(p, x, 0.5);
    p = fma(p, x, 1.0);
    return fma(p, x, 1.0);
}

// ------------------------------------------------------- grid interpolation

// LocalVarianceGrid::interpolate_with_hints, local_variance.rs:303-414: the
// x cell is found by walking from the previous cell (the same answer as the
// binary search under total_cmp), the time cell and weight of each step are
// plan constants.
struct GridView {
    const double* v;        // nt x nx values (shared memory or global through L1)
    const double* x;        // nx nodes
    const long long* xkey;  // total-order keys of the nodes
    int nx;
    // interp_variance_walk (the path tiles): cell bounds {x[c], x[c+1]}
    // (nx - 1, shared memory), the cells {v[t][c], slope} of every row
    // (DevicePlan::grid_cells, through L1) and the clamp interval.
    const double2* bounds;
    const double2* cells;
    double x_first, x_last;
};
// A view carries either xkey (for interp_variance: the LSM path store and the
// adjoint sweep) or bounds and cells (for interp_variance_walk: the path tiles).


__device__ __forceinline__ double interp_variance(const GridView& g, int tc, double tw, double xq,
                                                  int& hint) {
    double xv = xq;
    if (xq < g.x[0]) xv = g.x[0];
    else if (xq > g.x[g.nx - 1]) xv = g.x[g.nx - 1];
    const long long k = total_key(xv);
    int count = min(hint + 1, g.nx);
    while (count < g.nx && g.xkey[count] <= k) ++count;
    while (count > 0 && g.xkey[count - 1] > k) --count;
    const int c = min(max(count - 1, 0), g.nx - 2);
    hint = c;
    const double xw = (xv - g.x[c]) / (g.x[c + 1] - g.x[c]);
    const double* row = g.v + static_cast<size_t>(tc) * g.nx;
    const double* next = row + g.nx;
    const double lower = row[c] * (1.0 - xw) + row[c + 1] * xw;
    const double upper = next[c] * (1.0 - xw) + next[c + 1] * xw;
    return lower * (1.0 - tw) + upper * tw;
}

// The path kernels' form of interp_variance: the same clamp and cell as the
// reference's total-order search (a walk from the previous cell: up while
// x[c+1] <= x, down while x[c] > x, within [0, nx - 2] -- for finite,
// strictly increasing nodes the last node <= x, the ends clamped), one
// 16-byte shared load per cell visited; each row's linear interpolation
// v[t][c] + slope (x - x[c]) as one fused multiply-add from the row's cell
// record, and the time interpolation lower + (upper - lower) tw as another.
// The reference's a (1 - w) + b w to rounding: the variance enters the path
// only through the step, whose results are held to 1e-12 of the reference.
__device__ __forceinline__ double interp_variance_walk(const GridView& g, int tc, double tw, double xq,
                                                       int& hint) {
    double xv = xq;
    if (xq < g.x_first) xv = g.x_first;
    else if (xq > g.x_last) xv = g.x_last;
    int c = hint;
    double2 b = g.bounds[c];
    while (c < g.nx - 2 && b.y <= xv) b = g.bounds[++c];
    while (c > 0 && b.x > xv) b = g.bounds[--c];
    hint = c;
    const double dx = xv - b.x;
    const double2* row = g.cells + static_cast<size_t>(tc) * (g.nx - 1) + c;
    const double2 lo = row[0];
    const double2 hi = row[g.nx - 1];
    const double lower = fma(lo.y, dx, lo.x);
    const double upper = fma(hi.y, dx, hi.x);
    return fma(upper - lower, tw, lower);
}

// ------------------------------------------------------- CTA reduction

// Reduce NC component values of every thread into one record per component.
// Fixed tree: warp butterfly with the lower lane on the left, then the warps
// in index order -- deterministic for a given launch shape.
template <int NC>
__device__ __forceinline__ void cta_reduce_write(const double (&vals)[NC], bool valid,
                                                 uint32_t mask, StatRecord* out, Stat* scratch) {
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    constexpr int kWarps = kThreads / 32;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        if (!(mask & (1u << (c % 32)))) continue;
        const Stat s = warp_reduce_stat(stat_of(vals[c], valid));
        if (lane == 0) scratch[warp * NC + c] = s;
    }
    __syncthreads();
    if (threadIdx.x < NC && (mask & (1u << (threadIdx.x % 32)))) {
        const int c = threadIdx.x;
        Stat a = stat_merge(scratch[0 * NC + c], scratch[1 * NC + c]);
        Stat b = stat_merge(scratch[2 * NC + c], scratch[3 * NC + c]);
        static_assert(kWarps == 4, "tree below assumes four warps");
        const Stat m = stat_merge(a, b);
        out[c] = {m.sum, m.corr, m.count, m.mean, m.m2};
    }
    __syncthreads();
}

// Batched normals: z_batch<Q>() normals per path at a time -- the ranks
// ranks[first..first+count) of a local-volatility program, or (ranks null)
// the dimensions first..first+count of a Black--Scholes path --
// (eight per thread either way), in s_z[(k * Q + q)][thread] for the thread's
// Q paths.  The warp forms the uniforms, takes AS241's central branch for
// every lane (its fused multiply-add form), and evaluates the tail branch only
// for the lanes that need it, 32 at a time from a compacted list (s_zlist,
// 32 * z_batch<Q>() * Q entries per warp), without a warp executing the tail
// branch for each normal that one of its lanes sends there.  The branch
// decision is that of as241 on the same word, the tail values are as241's bit
// for bit, the central ones within a few ulps.
template <int Q>
__host__ __device__ constexpr int z_batch() { return Q == 2 ? 4 : 8; }

template <int Q>
__device__ __forceinline__ void fill_normals(NormalSource (&ns)[Q], bool wsob, uint32_t first, uint32_t count,
                                             double* s_z, uint16_t* s_zlist, const uint32_t* ranks) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    uint16_t* list = s_zlist + warp * (32u * z_batch<Q>() * Q);
    uint32_t tails = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t rank = ranks ? __ldg(ranks + first + k) : first + k;
        uint32_t words[Q];
        if constexpr (Q == 1) {
            words[0] = wsob ? ns[0].word_warp(rank) : ns[0].word(rank);
        } else {
            // Q paths of one warp lane share the lane part of the Gray code and
            // the direction row: one load of each, one XOR reduction per path.
            if (wsob) {
                const uint32_t v = __ldg(ns[0].dirs + static_cast<size_t>(rank) * 32u + lane);
                const uint32_t common = __ldg(ns[0].shift + rank) ^
                                        __ldg(ns[0].low + static_cast<size_t>(rank) * 32u + ns[0].lane_low);
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    words[q] = common ^ __reduce_xor_sync(0xffffffffu, (ns[q].high_gray >> lane) & 1u ? v : 0u);
            } else {
#pragma unroll
                for (int q = 0; q < Q; ++q) words[q] = ns[q].word(rank);
            }
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            // (w + 0.5) 2^-32 as one exact fused multiply-add (w 2^-32 + 2^-33 needs 33 bits)
            const double p = fma(static_cast<double>(words[q]), 0x1p-32, 0x1p-33);
            const double c = p - 0.5;
            const bool tail = !(fabs(c) <= 0.425);
            const double central = as241_central_fma(c);
            const uint32_t slot = k * Q + q;
            s_z[slot * kThreads + threadIdx.x] = tail ? p : central;
            const unsigned m = __ballot_sync(0xffffffffu, tail);
            if (tail) list[tails + __popc(m & ((1u << lane) - 1u))] = static_cast<uint16_t>(slot * 32u + lane);
            tails += static_cast<uint32_t>(__popc(m));
        }
    }
    __syncwarp();
    for (uint32_t b = 0; b < tails; b += 32u) {
        const uint32_t i = b + lane;
        if (i < tails) {
            const uint32_t idx = list[i];
            double* at = s_z + (idx >> 5) * kThreads + warp * 32u + (idx & 31u);
            const double p = *at;
            *at = as241_tail(p, p - 0.5);
        }
    }
    __syncwarp();
}

}  // namespace mcg

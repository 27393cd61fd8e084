// mcg_setup.cu -- plan-setup and reduction kernels (FP64, -fmad=false).
//
//  * scramble_table_kernel: compiles the LMS scrambles of an RQMC plan and
//    pre-applies them to the Joe--Kuo directions
//    (crates/pricing/src/engine/sampling/qmc.rs:204-259,348-369).
//  * reduce_tiles_kernel: merges per-CTA statistics records of one scramble in
//    a fixed tree (the role of fixed_tree_reduce,
//    crates/pricing-numerics/src/reduction.rs:244-272).
//  * philox_normals_kernel / rqmc_words_kernel: sampling known-answer entry points.
//  * surface_grid_kernel: the Dupire local-variance grid of an SSVI or eSSVI
//    surface (crates/pricing/src/market/local_variance.rs:149-206).
#include "mcg_kernels.cuh"
#include "mcg_surface.cuh"

namespace mcg {

// One thread per (scramble, dimension): 33 Philox words (domain RqmcScramble),
// then D[s][d][k] = M_{s,d} v_{d,k} for the 32 direction words.
__global__ void scramble_table_kernel(const uint32_t* directions, uint32_t dims, uint32_t scrambles,
                                      uint32_t scramble_begin, uint64_t seed, uint32_t* table,
                                      uint32_t* shifts) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= dims * scrambles) return;
    const uint32_t s = idx / dims;  // local scramble; the Philox coordinate uses the global index
    const uint32_t d = idx % dims;
    uint32_t rows[32];
    const uint32_t block = d * 32u;
    // Coordinates (scramble, 32 d + r) with r = 0 the shift: blocks of four lanes.
#pragma unroll
    for (uint32_t q = 0; q < 8; ++q) {
        const uint4 b = philox_block(seed, scramble_begin + s, (block >> 2) + q, 2u);
        rows[4 * q + 0] = b.x;
        rows[4 * q + 1] = b.y;
        rows[4 * q + 2] = b.z;
        rows[4 * q + 3] = b.w;
    }
    const uint32_t shift = rows[0];
    rows[0] = 0x80000000u;
#pragma unroll
    for (uint32_t r = 1; r < 32; ++r) {
        const uint32_t before = 0xffffffffu << (32u - r);
        rows[r] = (rows[r] & before) | (1u << (31u - r));
    }
    shifts[static_cast<size_t>(s) * dims + d] = shift;
    const uint32_t* v = directions + static_cast<size_t>(d) * 32u;
    uint32_t* out = table + (static_cast<size_t>(s) * dims + d) * 32u;
    for (int k = 0; k < 32; ++k) {
        const uint32_t x = v[k];
        uint32_t y = 0;
#pragma unroll
        for (int r = 0; r < 32; ++r) y |= (static_cast<uint32_t>(__popc(x & rows[r])) & 1u) << (31 - r);
        out[k] = y;
    }
}

// Per-lane low Gray-code words: low[row][l] = XOR of table[row][b] over the
// set bits b of gray(l), l < 32 (row = scramble * dims + dim).
__global__ void scramble_low_kernel(const uint32_t* table, uint32_t rows, uint32_t* low) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= rows * 32u) return;
    const uint32_t row = idx >> 5, l = idx & 31u;
    const uint32_t g = l ^ (l >> 1);
    uint32_t x = 0;
    for (uint32_t b = 0; b < 5; ++b)
        if ((g >> b) & 1u) x ^= table[static_cast<size_t>(row) * 32u + b];
    low[idx] = x;
}

// Merge `tiles` records of one (scramble, slot): thread t folds tiles
// t, t+256, ... in order, then a pairwise tree over the 256 threads.
__global__ void reduce_tiles_kernel(const StatRecord* partials, uint32_t tiles, uint32_t slots,
                                    StatRecord* out) {
    __shared__ Stat s[256];
    const uint32_t slot = blockIdx.x;
    const uint32_t scramble = blockIdx.y;
    Stat acc{0.0, 0.0, 0.0, 0.0, 0.0};
    for (uint32_t t = threadIdx.x; t < tiles; t += 256) {
        const StatRecord r = partials[(static_cast<size_t>(scramble) * tiles + t) * slots + slot];
        const Stat x{r.sum, r.corr, r.count, r.mean, r.m2};
        acc = t == threadIdx.x ? x : stat_merge(acc, x);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int width = 128; width > 0; width >>= 1) {
        if (threadIdx.x < width) s[threadIdx.x] = stat_merge(s[threadIdx.x], s[threadIdx.x + width]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const Stat m = s[0];
        out[static_cast<size_t>(scramble) * slots + slot] = {m.sum, m.corr, m.count, m.mean, m.m2};
    }
}

__global__ void philox_normals_kernel(uint64_t seed, uint64_t first, uint64_t count, uint32_t dims,
                                      uint32_t domain, double* out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= count) return;
    const uint64_t unit = first + i;
    for (uint32_t d = 0; d < dims; ++d) {
        const uint4 b = philox_block(seed, unit, d >> 2, domain);
        out[static_cast<size_t>(d) * count + i] = as241(open_unit(lane_of(b, d & 3u)));
    }
}

__global__ void rqmc_words_kernel(const uint32_t* table, const uint32_t* shifts, uint32_t dims,
                                  uint32_t scramble, uint64_t first, uint64_t count, uint32_t* out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= count) return;
    const uint32_t point = static_cast<uint32_t>(first + i);
    NormalSource ns;
    ns.rqmc = 1;
    ns.gray = point ^ (point >> 1);
    ns.dirs = table + static_cast<size_t>(scramble) * dims * 32u;
    ns.shift = shifts + static_cast<size_t>(scramble) * dims;
    for (uint32_t d = 0; d < dims; ++d) out[static_cast<size_t>(d) * count + i] = ns.word(d);
}

// The same words formed the way the path kernels form them: each warp holds
// 32 consecutive, 32-aligned points (first % 32 == 0, count % 32 == 0) and
// calls NormalSource::word_warp, the common Gray-code part by one coalesced
// load and an XOR reduction, the lane part from the low table.
__global__ void rqmc_words_warp_kernel(const uint32_t* table, const uint32_t* shifts, const uint32_t* low,
                                       uint32_t dims, uint32_t scramble, uint64_t first, uint64_t count,
                                       uint32_t* out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t warp_first = i & ~static_cast<uint64_t>(31);
    if (warp_first >= count) return;  // whole warps leave together (count % 32 == 0)
    const uint32_t point = static_cast<uint32_t>(first + i);
    NormalSource ns;
    ns.rqmc = 1;
    ns.gray = point ^ (point >> 1);
    ns.dirs = table + static_cast<size_t>(scramble) * dims * 32u;
    ns.shift = shifts + static_cast<size_t>(scramble) * dims;
    const uint32_t q = point & ~31u;
    ns.high_gray = q ^ (q >> 1);
    ns.lane_low = point & 31u;
    ns.low = low + static_cast<size_t>(scramble) * dims * 32u;
    for (uint32_t d = 0; d < dims; ++d) out[static_cast<size_t>(d) * count + i] = ns.word_warp(d);
}

// ----------------------------------------------------------- SSVI grid

// One thread per grid node: the surface's total variance derivatives at
// (t, k), the Durrleman density factor (ssvi.rs:226-273) and the floor/cap
// classification (local_variance.rs:607-627).  The t = 0 row is evaluated at
// the first positive time node (local_variance.rs:164).  counters[0] counts
// repairs, counters[1] nodes where the surface or the density is invalid.
__global__ void surface_grid_kernel(const Surface S, const double* tn, uint32_t nt, const double* xn, uint32_t nx,
                                    double floor, double cap, double* out, uint32_t* counters) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nt * nx) return;
    const uint32_t i = idx / nx, j = idx % nx;
    const double st = tn[i] == 0.0 ? tn[1] : tn[i];
    const double x = xn[j];
    TotalVariance tv;
    if (!surface_total_variance(S, st, x, tv)) {
        atomicAdd(&counters[1], 1u);
        out[idx] = floor;
        return;
    }
    const double u = 1.0 - x * tv.wk / (2.0 * tv.w);
    const double density = u * u - (tv.wk * tv.wk / 4.0) * (1.0 / tv.w + 1.0 / 4.0) + tv.wkk / 2.0;
    if (!isfinite(density) || density <= 0.0) {
        atomicAdd(&counters[1], 1u);
        out[idx] = floor;
        return;
    }
    const double raw = tv.wt / density;
    double value = raw;
    bool repaired = true;
    if (isnan(raw)) value = floor;
    else if (raw == -INFINITY) value = floor;
    else if (raw == INFINITY) value = cap;
    else if (raw <= 0.0) value = floor;
    else if (raw < floor) value = floor;
    else if (raw > cap) value = cap;
    else repaired = false;
    if (repaired) atomicAdd(&counters[0], 1u);
    out[idx] = value;
}

// Total variance derivatives at explicit points (the surface known-answer entry point).
__global__ void surface_eval_kernel(const Surface S, const double* times, const double* ks, uint32_t count,
                                    double* out, uint32_t* failures) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    TotalVariance tv;
    if (!surface_total_variance(S, times[i], ks[i], tv)) atomicAdd(failures, 1u);
    out[4 * i + 0] = tv.w;
    out[4 * i + 1] = tv.wk;
    out[4 * i + 2] = tv.wkk;
    out[4 * i + 3] = tv.wt;
}

cudaError_t launch_surface_grid(const Surface& s, const double* tn, uint32_t nt, const double* xn, uint32_t nx,
                                double floor, double cap, double* out, uint32_t* counters, cudaStream_t stream) {
    const size_t nv = static_cast<size_t>(nt) * nx;
    surface_grid_kernel<<<static_cast<unsigned>((nv + 127) / 128), 128, 0, stream>>>(s, tn, nt, xn, nx, floor, cap,
                                                                                    out, counters);
    return cudaGetLastError();
}

cudaError_t launch_surface_eval(const Surface& s, const double* times, const double* ks, uint32_t count,
                                double* out, uint32_t* failures, cudaStream_t stream) {
    surface_eval_kernel<<<(count + 127) / 128, 128, 0, stream>>>(s, times, ks, count, out, failures);
    return cudaGetLastError();
}

}  // namespace mcg

namespace mcg {

// FP64 FMA throughput probe for the benchmark's roofline: independent chains
// of DFMA per thread (explicit fma(), unaffected by -fmad=false).
__global__ void fp64_peak_kernel(double* sink, int iterations) {
    double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
    double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
    const double m = 0.999999999, c = 1e-12;
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 12345.678) sink[threadIdx.x] = s;
}

}  // namespace mcg

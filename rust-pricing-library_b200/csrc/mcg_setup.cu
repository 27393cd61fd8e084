// mcg_setup.cu -- plan-setup and reduction kernels (FP64, -fmad=false).
//
//  * scramble_table_kernel: compiles the LMS scrambles of an RQMC plan and
//    pre-applies them to the Joe--Kuo directions
//    (crates/pricing/src/engine/sampling/qmc.rs:204-259,348-369).
//  * reduce_tiles_kernel: merges per-CTA statistics records of one scramble in
//    a fixed tree (the role of fixed_tree_reduce,
//    crates/pricing-numerics/src/reduction.rs:244-272).
//  * philox_normals_kernel / rqmc_words_kernel: sampling known-answer entry points.
//  * ssvi_grid_kernel: the Dupire local-variance grid of an SSVI surface
//    (crates/pricing/src/market/local_variance.rs:149-206).
#include "mcg_kernels.cuh"

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

// ----------------------------------------------------------- SSVI grid

struct Pchip {
    const double* t;
    const double* v;
    const double* d;
    uint32_t n;
    double slope;
};

// ThetaPchip::evaluate, crates/pricing/src/market/pchip.rs:111-176.
__device__ void pchip_eval(const Pchip& c, double time, double& theta, double& deriv) {
    if (time == 0.0) time = 0.0;
    if (time < c.t[0]) {
        deriv = c.v[0] / c.t[0];
        theta = time * deriv;
        return;
    }
    const long long key = total_key(time);
    uint32_t lo = 0, hi = c.n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (total_key(c.t[mid]) < key) lo = mid + 1; else hi = mid;
    }
    if (lo < c.n && total_key(c.t[lo]) == key) {
        theta = c.v[lo];
        deriv = c.d[lo];
        return;
    }
    if (lo < c.n) {
        const uint32_t r = lo, l = lo - 1;
        const double width = c.t[r] - c.t[l];
        const double sc = (time - c.t[l]) / width;
        const double sc2 = sc * sc;
        const double sc3 = sc2 * sc;
        const double h00 = 2.0 * sc3 - 3.0 * sc2 + 1.0;
        const double h10 = sc3 - 2.0 * sc2 + sc;
        const double h01 = -2.0 * sc3 + 3.0 * sc2;
        const double h11 = sc3 - sc2;
        theta = h00 * c.v[l] + h10 * width * c.d[l] + h01 * c.v[r] + h11 * width * c.d[r];
        const double d00 = (6.0 * sc2 - 6.0 * sc) / width;
        const double d10 = 3.0 * sc2 - 4.0 * sc + 1.0;
        const double d01 = (-6.0 * sc2 + 6.0 * sc) / width;
        const double d11 = 3.0 * sc2 - 2.0 * sc;
        deriv = d00 * c.v[l] + d10 * c.d[l] + d01 * c.v[r] + d11 * c.d[r];
        return;
    }
    const uint32_t last = c.n - 1;
    theta = c.v[last] + c.slope * (time - c.t[last]);
    deriv = c.slope;
}

// One thread per grid node: StandardSsvi::total_variance_derivatives
// (ssvi.rs:410-479) with the power-law phi (ssvi.rs:121-176), the Durrleman
// density factor (ssvi.rs:226-273) and the floor/cap classification
// (local_variance.rs:607-627).  The t = 0 row is evaluated at the first
// positive time node (local_variance.rs:164).
__global__ void ssvi_grid_kernel(Pchip theta, double rho, double eta, double gamma,
                                 const double* tn, uint32_t nt, const double* xn, uint32_t nx,
                                 double floor, double cap, double* out, uint32_t* repairs,
                                 uint32_t* failures) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nt * nx) return;
    const uint32_t i = idx / nx, j = idx % nx;
    const double st = tn[i] == 0.0 ? tn[1] : tn[i];
    double th, dth;
    pchip_eval(theta, st, th, dth);
    const double phi = eta / (pow(th, gamma) * pow(1.0 + th, 1.0 - gamma));
    const double phi_td = -phi * (gamma / th + (1.0 - gamma) / (1.0 + th));
    const double x = xn[j];
    const double y = phi * x;
    const double a = y + rho;
    const double q = sqrt(a * a + 1.0 - rho * rho);
    const double shape = 1.0 + rho * y + q;
    const double w = th * shape / 2.0;
    const double common = rho + a / q;
    const double wk = th * phi * common / 2.0;
    const double wkk = th * phi * phi * (1.0 - rho * rho) / (2.0 * q * q * q);
    const double partial = shape / 2.0 + th * x * phi_td * common / 2.0;
    const double wt = partial * dth;
    if (!(w > 0.0) || !isfinite(w) || !isfinite(wt)) {
        atomicAdd(failures, 1u);
        out[idx] = floor;
        return;
    }
    const double u = 1.0 - x * wk / (2.0 * w);
    const double density = u * u - (wk * wk / 4.0) * (1.0 / w + 1.0 / 4.0) + wkk / 2.0;
    if (!isfinite(density) || density <= 0.0) {
        atomicAdd(failures, 1u);
        out[idx] = floor;
        return;
    }
    const double raw = wt / density;
    double value = raw;
    bool repaired = true;
    if (isnan(raw)) value = floor;
    else if (raw == -INFINITY) value = floor;
    else if (raw == INFINITY) value = cap;
    else if (raw <= 0.0) value = floor;
    else if (raw < floor) value = floor;
    else if (raw > cap) value = cap;
    else repaired = false;
    if (repaired) atomicAdd(repairs, 1u);
    out[idx] = value;
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

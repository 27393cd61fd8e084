// mcg_device.cuh -- device primitives of the B200 Monte Carlo engine.
//
// Counter-based Philox normals, scrambled Sobol words from a pre-applied
// direction table, the AS241 quantile, compact-C2 smoothing, barrier-bridge
// intervals and deterministic statistics merges.  The FP64 translation units
// that include this header are compiled with -fmad=false so that every a*b+c
// rounds twice, as the reference's Rust arithmetic does; the functions cite the
// reference file:line whose arithmetic they follow.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "mcg_plan.h"

// Functions marked MCG_HD are plain arithmetic that also compiles for the
// host, so the test suite can check them against the oracle without a GPU.
#define MCG_HD __host__ __device__ __forceinline__

namespace mcg {

// ---------------------------------------------------------------- Philox

// Philox4x32-10 with the Random123 multipliers and Weyl key increments,
// crates/pricing/src/engine/sampling/random.rs:4-8,100-137.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xd2511f53u * c.x;
        const uint32_t hi0 = __umulhi(0xd2511f53u, c.x);
        const uint32_t lo1 = 0xcd9e8d57u * c.z;
        const uint32_t hi1 = __umulhi(0xcd9e8d57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9e3779b9u;
        k1 += 0xbb67ae85u;
    }
    return c;
}

// RandomCoordinate layout, random.rs:63-75: counter = [path lo, path hi,
// dimension / 4, domain], lane = dimension % 4.
__device__ __forceinline__ uint4 philox_block(uint64_t seed, uint64_t path, uint32_t block,
                                              uint32_t domain) {
    return philox4x32_10(make_uint4(static_cast<uint32_t>(path), static_cast<uint32_t>(path >> 32),
                                    block, domain),
                         static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
}

__device__ __forceinline__ uint32_t lane_of(const uint4& b, uint32_t lane) {
    return lane == 0 ? b.x : lane == 1 ? b.y : lane == 2 ? b.z : b.w;
}

// Bin midpoint of a 32-bit word, random.rs:139-143: (w + 0.5) * 2^-32, exact.
__device__ __forceinline__ double open_unit(uint32_t w) {
    return (static_cast<double>(w) + 0.5) * 2.3283064365386963e-10;
}

// ----------------------------------------------------------------- AS241

// Wichura AS241 coefficients (Applied Statistics 37(3), 1988) as the binary64
// values the reference uses, random.rs:181-240.
__device__ __forceinline__ double poly8(double x, double c0, double c1, double c2, double c3,
                                        double c4, double c5, double c6, double c7) {
    double v = c7;
    v = v * x + c6;
    v = v * x + c5;
    v = v * x + c4;
    v = v * x + c3;
    v = v * x + c2;
    v = v * x + c1;
    v = v * x + c0;
    return v;
}

// inverse_standard_normal, random.rs:176-266, same branch structure and
// operation order; the tail uses CUDA's log and sqrt.  The two branches are
// also callable on their own (the batched normals of the path kernels take
// the central branch for every lane and the tail only for the lanes that
// need it).
__device__ __forceinline__ double as241_central(double centered) {
    const double a = 0.180625 - centered * centered;
    const double num = poly8(a, 0x1.b18d91e9eef75p+1, 0x1.0a4888b1a436ep+7, 0x1.ece5d2213c0ccp+10,
                             0x1.ad1d8cd4ee71dp+13, 0x1.66c3e869b752ap+15, 0x1.06c1c55b78f20p+16,
                             0x1.052d26b2e4604p+15, 0x1.39a296f7d925ep+11);
    const double den = poly8(a, 1.0, 0x1.5281b386e1ab5p+5, 0x1.5797efdc8b3f7p+9,
                             0x1.512322e75c89fp+12, 0x1.4b772d5d65266p+14, 0x1.3317caa64f4bep+15,
                             0x1.c0e457cb1ae76p+14, 0x1.46a7eca984b6ap+12);
    return centered * num / den;
}

// The central branch with each Horner step a fused multiply-add (and a = 0.180625
// - c^2 as one), for the path kernels' batched normals: within a few ulps of
// as241_central, whose two-rounding form the exported normals keep bit for bit.
// The path results are held to 1e-12 of the reference, not to the bit.
__device__ __forceinline__ double poly8_fma(double x, double c0, double c1, double c2, double c3, double c4,
                                           double c5, double c6, double c7) {
    double v = c7;
    v = fma(v, x, c6);
    v = fma(v, x, c5);
    v = fma(v, x, c4);
    v = fma(v, x, c3);
    v = fma(v, x, c2);
    v = fma(v, x, c1);
    v = fma(v, x, c0);
    return v;
}

__device__ __forceinline__ double as241_central_fma(double centered) {
    const double a = fma(-centered, centered, 0.180625);
    const double num = poly8_fma(a, 0x1.b18d91e9eef75p+1, 0x1.0a4888b1a436ep+7, 0x1.ece5d2213c0ccp+10,
                                 0x1.ad1d8cd4ee71dp+13, 0x1.66c3e869b752ap+15, 0x1.06c1c55b78f20p+16,
                                 0x1.052d26b2e4604p+15, 0x1.39a296f7d925ep+11);
    const double den = poly8_fma(a, 1.0, 0x1.5281b386e1ab5p+5, 0x1.5797efdc8b3f7p+9,
                                 0x1.512322e75c89fp+12, 0x1.4b772d5d65266p+14, 0x1.3317caa64f4bep+15,
                                 0x1.c0e457cb1ae76p+14, 0x1.46a7eca984b6ap+12);
    return centered * num / den;
}

__device__ __forceinline__ double as241_tail(double p, double centered) {
    const double tail = centered < 0.0 ? p : 1.0 - p;
    const double r = sqrt(-log(tail));
    double m;
    if (r <= 5.0) {
        const double a = r - 1.6;
        m = poly8(a, 0x1.6c665fde9526ap+0, 0x1.2857748cab19bp+2, 0x1.713f71462256ap+2,
                  0x1.d2ecb1a3d02c4p+1, 0x1.453cc085375b2p+0, 0x1.ef2abb9b85c37p-3,
                  0x1.744eb6c45ec67p-6, 0x1.9615ac0b7ace9p-11) /
            poly8(a, 1.0, 0x1.06cefbb46a449p+1, 0x1.ad278e6526633p+0, 0x1.61292f23385c9p-1,
                  0x1.2f5123394f040p-3, 0x1.f207a7eab17bfp-7, 0x1.1f18cbfdf2728p-11,
                  0x1.20d3f686439e4p-30);
    } else {
        const double a = r - 5.0;
        m = poly8(a, 0x1.aa1b1c13ee527p+2, 0x1.5daea6e875003p+2, 0x1.c8ea6461fa445p+0,
                  0x1.2fad9315255d0p-2, 0x1.b2b41193b4ee7p-6, 0x1.45c1908425345p-10,
                  0x1.c6ec6cc59e02ap-16, 0x1.afb74d693bf93p-23) /
            poly8(a, 1.0, 0x1.331d34fc7d77ep-1, 0x1.186eb183443fbp-3, 0x1.e76f93215462ap-7,
                  0x1.9c8bc979dc5d7p-11, 0x1.35c2c494cf5d0p-16, 0x1.31446f740bfc3p-23,
                  0x1.269bff1f8c190p-49);
    }
    return centered < 0.0 ? -m : m;
}

__device__ __forceinline__ double as241(double p) {
    const double centered = p - 0.5;
    if (fabs(centered) <= 0.425) return as241_central(centered);
    return as241_tail(p, centered);
}

// Single-precision AS241 for the FP32 bulk path (same branches, FP32 rounding).
__device__ __forceinline__ float as241f(float p) {
    const float centered = p - 0.5f;
    if (fabsf(centered) <= 0.425f) {
        const float a = 0.180625f - centered * centered;
        const float num =
            ((((((2509.0809287301227f * a + 33430.575583588128f) * a + 67265.770927008700f) * a +
                 45921.953931549871f) * a + 13731.693765509461f) * a + 1971.5909503065514f) * a +
             133.14166789178438f) * a + 3.3871328727963666f;
        const float den =
            ((((((5226.4952788528545f * a + 28729.085735721943f) * a + 39307.895800092710f) * a +
                 21213.794301586596f) * a + 5394.1960214247511f) * a + 687.18700749205790f) * a +
             42.313330701600911f) * a + 1.0f;
        return centered * num / den;
    }
    const float tail = centered < 0.0f ? p : 1.0f - p;
    const float r = sqrtf(-logf(tail));
    float m;
    if (r <= 5.0f) {
        const float a = r - 1.6f;
        m = ((((((7.74545014278341407640e-4f * a + 2.27238449892691845833e-2f) * a +
                 2.41780725177450611770e-1f) * a + 1.27045825245236838258f) * a +
               3.64784832476320460504f) * a + 5.76949722146069140550f) * a +
             4.63033784615654529590f) * a + 1.42343711074968357734f;
        m /= ((((((1.05075007164441684324e-9f * a + 5.47593808499534494600e-4f) * a +
                  1.51986665636164571966e-2f) * a + 1.48103976427480074590e-1f) * a +
                6.89767334985100004550e-1f) * a + 1.67638483018380384940f) * a +
              2.05319162663775882187f) * a + 1.0f;
    } else {
        const float a = r - 5.0f;
        m = ((((((2.01033439929228813265e-7f * a + 2.71155556874348757815e-5f) * a +
                 1.24266094738807843860e-3f) * a + 2.65321895265761230930e-2f) * a +
               2.96560571828504891230e-1f) * a + 1.78482653991729133580f) * a +
             5.46378491116411436990f) * a + 6.65790464350110377720f;
        m /= ((((((2.04426310338993978564e-15f * a + 1.42151175831644588870e-7f) * a +
                  1.84631831751005468180e-5f) * a + 7.86869131145613259100e-4f) * a +
                1.48753612908506148525e-2f) * a + 1.36929880922735805310e-1f) * a +
              5.99832206555887937690e-1f) * a + 1.0f;
    }
    return centered < 0.0f ? -m : m;
}

// ------------------------------------------------------------ total order

// Key with Rust f64::total_cmp order (-0.0 < +0.0).
__device__ __forceinline__ long long total_key(double x) {
    const long long b = __double_as_longlong(x);
    return b ^ static_cast<long long>(static_cast<unsigned long long>(b >> 63) >> 1);
}

// ------------------------------------------------------------- smoothing

// f64::is_normal by the exponent field: neither zero/subnormal nor inf/NaN.
// (The C library's isnormal is a host function; this one runs on both sides.)
MCG_HD bool is_normal(double x) {
#ifdef __CUDA_ARCH__
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
#else
    unsigned long long b;
    __builtin_memcpy(&b, &x, 8);
#endif
    const unsigned e = static_cast<unsigned>(b >> 52) & 0x7ffu;
    return e != 0u && e != 0x7ffu;
}

// CompactC2Smoothing, crates/pricing/src/product/smoothing.rs:29-198.
struct SmoothD {
    double value, first;
};

MCG_HD double transition_coordinate(double input, double h) {
    const double full = 2.0 * h;
    if (isfinite(full)) return (input + h) / full;
    if (input < 0.0) return 0.5 * ((input + h) / h);
    return 0.5 * (input / h + 1.0);
}

MCG_HD double quintic(double u) {
    return u * u * u * (10.0 + u * (-15.0 + 6.0 * u));
}

MCG_HD SmoothD interior_indicator(double input, double h, double u,
                                                      double& complement) {
    const double hit = quintic(u);
    const double safety = 1.0 - hit;
    double z, value;
    if (safety <= 32.0 * 2.220446049250313e-16) {
        z = transition_coordinate(-input, h);
        const double tail = quintic(z);
        value = 1.0 - tail;
        complement = tail;
    } else {
        z = u;
        value = hit;
        complement = safety;
    }
    const double z2 = z * z;
    const double omz = 1.0 - z;
    return {value, 15.0 * z2 * omz * omz / h};
}

MCG_HD SmoothD smooth_indicator(double h, double input, double& complement) {
    if (input <= -h) {
        complement = 1.0;
        return {0.0, 0.0};
    }
    if (input >= h) {
        complement = 0.0;
        return {1.0, 0.0};
    }
    return interior_indicator(input, h, transition_coordinate(input, h), complement);
}

MCG_HD SmoothD smooth_positive_part(double h, double input) {
    if (input <= -h) return {0.0, 0.0};
    if (input >= h) return {input, 1.0};
    const double u = transition_coordinate(input, h);
    const double u2 = u * u;
    const double u4 = u2 * u2;
    double comp;
    const SmoothD ind = interior_indicator(input, h, u, comp);
    const double scaled_u4 = 2.0 * h * u4;
    const double poly = 2.5 + u * (-3.0 + u);
    const double value = is_normal(scaled_u4) ? scaled_u4 * poly : (2.0 * u4 * poly) * h;
    return {value, ind.value};
}

// Smooth maximum of the compact-C2 smoothing, right + positive_part(left -
// right) (CompactC2Smoothing::maximum, crates/pricing/src/product/smoothing.rs:136-160),
// with its partial derivatives d/dleft (the indicator) and d/dright (its
// complement).
MCG_HD double smooth_maximum(double h, double left, double right, double& d_left, double& d_right) {
    const double diff = left - right;
    if (diff >= h) {
        d_left = 1.0;
        d_right = 0.0;
        return left;
    }
    if (diff <= -h) {
        d_left = 0.0;
        d_right = 1.0;
        return right;
    }
    const double u = transition_coordinate(diff, h);
    const double u2 = u * u;
    const double u4 = u2 * u2;
    double comp;
    const SmoothD ind = interior_indicator(diff, h, u, comp);
    const double scaled_u4 = 2.0 * h * u4;
    const double poly = 2.5 + u * (-3.0 + u);
    const double value = is_normal(scaled_u4) ? scaled_u4 * poly : (2.0 * u4 * poly) * h;
    d_left = ind.value;
    d_right = comp;
    return right + value;
}

// ------------------------------------------------------------- dividends

// AffineDividendCoordinate (crates/pricing/src/market/dividend.rs:137-181):
// the observed spot a S0 + b f of the canonical state f, and the spot-bump
// derivative scale.  A plan stores each observation's coordinate at its own
// spot as double4 {a, b, spot_scale, flag}; at_spot refits it to a bumped
// spot with the cash held fixed.
struct DivCoord {
    double a, b, spot_scale;
};

MCG_HD DivCoord div_at_spot(const double4& c, double original, double spot) {
    if (original == spot) return {c.x, c.y, c.z};
    return {c.x * original / spot, c.z - (c.z - c.y) * original / spot, c.z};
}

// ------------------------------------------------------------ statistics

// One DeterministicStatistics record: NeumaierSum + CenteredMoment,
// crates/pricing-numerics/src/reduction.rs:3-170.
struct Stat {
    double sum, corr;
    double count;  // exact integer below 2^53
    double mean, m2;
};

__device__ __forceinline__ void neumaier_add(double& sum, double& corr, double value) {
    const double updated = sum + value;
    if (fabs(sum) >= fabs(value)) corr += (sum - updated) + value;
    else corr += (value - updated) + sum;
    sum = updated;
}

// NeumaierSum::merged and CenteredMoment::merged (Chan--Golub--LeVeque).
__device__ __forceinline__ Stat stat_merge(const Stat& l, const Stat& r) {
    Stat m;
    m.sum = 0.0;
    m.corr = 0.0;
    neumaier_add(m.sum, m.corr, l.sum);
    neumaier_add(m.sum, m.corr, l.corr);
    neumaier_add(m.sum, m.corr, r.sum);
    neumaier_add(m.sum, m.corr, r.corr);
    if (l.count == 0.0) {
        m.count = r.count;
        m.mean = r.mean;
        m.m2 = r.m2;
    } else if (r.count == 0.0) {
        m.count = l.count;
        m.mean = l.mean;
        m.m2 = l.m2;
    } else {
        m.count = l.count + r.count;
        const double delta = r.mean - l.mean;
        m.mean = l.mean + delta * (r.count / m.count);
        m.m2 = (l.m2 + r.m2) + delta * delta * (l.count * r.count / m.count);
    }
    return m;
}

__device__ __forceinline__ Stat stat_of(double v, bool valid) {
    if (!valid) return {0.0, 0.0, 0.0, 0.0, 0.0};
    return {v, 0.0, 1.0, v, 0.0};
}

__device__ __forceinline__ Stat shfl_down_stat(const Stat& s, int offset) {
    Stat r;
    r.sum = __shfl_down_sync(0xffffffffu, s.sum, offset);
    r.corr = __shfl_down_sync(0xffffffffu, s.corr, offset);
    r.count = __shfl_down_sync(0xffffffffu, s.count, offset);
    r.mean = __shfl_down_sync(0xffffffffu, s.mean, offset);
    r.m2 = __shfl_down_sync(0xffffffffu, s.m2, offset);
    return r;
}

// Fixed-shape warp tree: lane i merges lane i+off (left = lower lane); the
// result is in lane 0 and independent of scheduling.
__device__ __forceinline__ Stat warp_reduce_stat(Stat s) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const Stat o = shfl_down_stat(s, off);
        if ((threadIdx.x & (2 * off - 1)) == 0) s = stat_merge(s, o);
    }
    return s;
}

}  // namespace mcg

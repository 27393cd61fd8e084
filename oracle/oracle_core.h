// oracle_core.h -- CPU restatement of the reference's Monte Carlo hot path.
//
// TEST INFRASTRUCTURE ONLY.  This code is the oracle the CUDA engine is
// compared against: only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg may load it.  It is never linked into the engine.
//
// It restates, in plain C++ compiled with -O2 -ffp-contract=off against the
// platform libm, the arithmetic of msfmfjt/rust-pricing-library (paths relative
// to that project).  Each function cites the file:line it follows.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- sampling

// Philox4x32-10 with the Random123 constants and round schedule,
// crates/pricing/src/engine/sampling/random.rs:4-8,82-137.
struct Block4 {
    uint32_t v[4];
};

inline Block4 philox_generate(uint64_t seed, Block4 counter) {
    uint32_t k0 = static_cast<uint32_t>(seed);
    uint32_t k1 = static_cast<uint32_t>(seed >> 32);
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = static_cast<uint64_t>(0xd2511f53u) * counter.v[0];
        const uint64_t p1 = static_cast<uint64_t>(0xcd9e8d57u) * counter.v[2];
        const uint32_t h0 = static_cast<uint32_t>(p0 >> 32);
        const uint32_t h1 = static_cast<uint32_t>(p1 >> 32);
        Block4 next;
        next.v[0] = h1 ^ counter.v[1] ^ k0;
        next.v[1] = static_cast<uint32_t>(p1);
        next.v[2] = h0 ^ counter.v[3] ^ k1;
        next.v[3] = static_cast<uint32_t>(p0);
        counter = next;
        if (round + 1 < 10) {
            k0 += 0x9e3779b9u;
            k1 += 0xbb67ae85u;
        }
    }
    return counter;
}

// RandomCoordinate counter/lane layout, random.rs:63-75.
inline uint32_t philox_word(uint64_t seed, uint64_t path, uint32_t dimension, uint32_t domain) {
    Block4 c{{static_cast<uint32_t>(path), static_cast<uint32_t>(path >> 32), dimension / 4u,
              domain}};
    return philox_generate(seed, c).v[dimension % 4u];
}

// Bin midpoint, random.rs:139-143.
inline double open_unit_interval(uint32_t word) {
    return (static_cast<double>(word) + 0.5) * (1.0 / 4294967296.0);
}

double inverse_standard_normal(double probability);  // AS241, random.rs:176-277

inline double philox_normal(uint64_t seed, uint64_t path, uint32_t dimension, uint32_t domain) {
    return inverse_standard_normal(open_unit_interval(philox_word(seed, path, dimension, domain)));
}

// Sobol word by Gray-code XOR, qmc.rs:71-84.  `directions` holds 32 words.
inline uint32_t sobol_word(const uint32_t* directions, uint32_t point) {
    uint32_t gray = point ^ (point >> 1);
    uint32_t word = 0;
    int bit = 0;
    while (gray != 0) {
        if (gray & 1u) word ^= directions[bit];
        gray >>= 1;
        ++bit;
    }
    return word;
}

// Linear matrix scramble plus digital shift, qmc.rs:107-132,348-369.
struct Scramble {
    uint32_t shift;
    uint32_t rows[32];
    uint32_t apply(uint32_t input) const {
        uint32_t out = 0;
        for (int r = 0; r < 32; ++r) {
            const uint32_t parity = static_cast<uint32_t>(__builtin_popcount(input & rows[r])) & 1u;
            out |= parity << (31 - r);
        }
        return out ^ shift;
    }
};

Scramble compile_scramble(uint64_t seed, uint64_t scramble, uint32_t dimension);

// -------------------------------------------------------- Brownian bridge

// BrownianBridgePlan, crates/pricing/src/engine/sampling/bridge.rs:163-311,395-467.
struct BridgeInstruction {
    bool terminal;
    uint32_t node, left, right, rank;
    double left_weight, right_weight, standard_deviation;
};

struct BridgePlan {
    std::vector<double> times;
    std::vector<double> inverse_sqrt_dt;
    std::vector<BridgeInstruction> instructions;
    // Returns false on an invalid grid (BrownianBridgeError).
    bool compile(const std::vector<double>& node_times);
    // apply_one_factor: normals by rank -> normalised increments by interval.
    void apply(const double* normals, double* increments, std::vector<double>& scratch) const;
    // reverse_one_factor: increment adjoints -> normal adjoints.
    void reverse(const double* increment_adjoints, double* normal_adjoints,
                 std::vector<double>& scratch) const;
};

// ------------------------------------------------------------- reductions

// NeumaierSum and CenteredMoment, crates/pricing-numerics/src/reduction.rs:3-170.
struct NeumaierSum {
    double sum = 0.0;
    double correction = 0.0;
    void add(double value) {
        const double updated = sum + value;
        if (std::fabs(sum) >= std::fabs(value)) {
            correction += (sum - updated) + value;
        } else {
            correction += (value - updated) + sum;
        }
        sum = updated;
    }
    double total() const { return sum + correction; }
    static NeumaierSum merged(const NeumaierSum& l, const NeumaierSum& r) {
        NeumaierSum m;
        m.add(l.sum);
        m.add(l.correction);
        m.add(r.sum);
        m.add(r.correction);
        return m;
    }
};

struct CenteredMoment {
    uint64_t count = 0;
    double mean = 0.0;
    double second_moment = 0.0;
    void add(double value) {
        const uint64_t next_count = count + 1;
        const double delta = value - mean;
        const double next_mean = mean + delta / static_cast<double>(next_count);
        second_moment += delta * (value - next_mean);
        mean = next_mean;
        count = next_count;
    }
    static CenteredMoment merged(const CenteredMoment& l, const CenteredMoment& r) {
        if (l.count == 0) return r;
        if (r.count == 0) return l;
        CenteredMoment m;
        m.count = l.count + r.count;
        const double delta = r.mean - l.mean;
        const double lw = static_cast<double>(l.count);
        const double rw = static_cast<double>(r.count);
        const double n = static_cast<double>(m.count);
        m.mean = l.mean + delta * (rw / n);
        const double between = delta * delta * (lw * rw / n);
        m.second_moment = (l.second_moment + r.second_moment) + between;
        return m;
    }
    static CenteredMoment two_pass(const std::vector<double>& values);
};

struct Statistics {
    NeumaierSum sum;
    CenteredMoment moments;
    void add(double v) {
        sum.add(v);
        moments.add(v);
    }
};

// fixed_tree_reduce, reduction.rs:257-272: pairwise levels, odd tail carried.
template <class T, class Merge>
T fixed_tree_reduce(std::vector<T> level, Merge merge) {
    if (level.empty()) return T{};
    while (level.size() > 1) {
        std::vector<T> next;
        next.reserve((level.size() + 1) / 2);
        size_t i = 0;
        for (; i + 1 < level.size(); i += 2) next.push_back(merge(level[i], level[i + 1]));
        if (i < level.size()) next.push_back(level[i]);
        level.swap(next);
    }
    return level[0];
}

// ----------------------------------------------------------------- market

// LogLinearDiscountCurve::evaluate, crates/pricing/src/market/curve.rs:156-200.
struct Curve {
    std::vector<double> times, logs;
    void set(const double* t, const double* df, uint32_t n) {
        times.assign(t, t + n);
        logs.resize(n);
        for (uint32_t i = 0; i < n; ++i) logs[i] = std::log(df[i]);
    }
    double log_discount(double time) const;
};

// total_cmp key of an f64: orders -0.0 below +0.0, like Rust's f64::total_cmp.
inline int64_t total_key(double x) {
    int64_t b;
    std::memcpy(&b, &x, 8);
    return b ^ static_cast<int64_t>((static_cast<uint64_t>(b >> 63)) >> 1);
}

// LocalVarianceGrid interpolation, crates/pricing/src/market/local_variance.rs:273-414.
struct Interpolation {
    double value;
    uint32_t time_cell, x_cell;
    double time_weight, x_weight;
    bool in_range;
};

struct Grid {
    std::vector<double> t, x, v;
    double floor = 0.0, cap = 0.0;
    uint32_t nt() const { return static_cast<uint32_t>(t.size()); }
    uint32_t nx() const { return static_cast<uint32_t>(x.size()); }
    // Returns false for an out-of-range time or non-finite x (InvalidSurfaceQuery).
    bool interpolate(double time, double log_moneyness, Interpolation& out) const;
    double x_derivative(const Interpolation& in) const;
    void transpose_accumulate(const Interpolation& in, double seed, double* adjoints) const;
};

uint32_t lower_cell(const std::vector<double>& nodes, double value);

}  // namespace oracle

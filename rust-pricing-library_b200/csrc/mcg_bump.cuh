// mcg_bump.cuh -- the scenario sides of a bump-and-revalue request: launch
// interface shared by the kernels (mcg_bump.cu) and the host (mcg_host.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mcg_book.cuh"
#include "mcg_plan.h"

namespace mcg {

struct ErrorWord;

// One launch prices every side: CTA (tile, scramble, side) evaluates 128 units
// of one scramble of one side's plan.  All sides are the same kind of path
// (they are one plan with an input moved), so the kernel is specialised on it.
struct ScenarioLaunch {
    const DevicePlan* plans;   // [sides]
    const uint32_t* masks;     // [sides]
    uint32_t sides, scrambles, tiles;
    uint32_t path;             // BookPath of every side
    int evolutions;            // local volatility: 1, or 2 with antithetic pairs
    StatRecord* partials;      // [side][scramble][tile][kComponents]
    double* unit_prices;       // pseudo-MC: [side][unit] discounted unit prices; RQMC: null
    uint64_t units;            // units per scramble
    ErrorWord* errors;         // [sides]
    uint32_t max_nodes, max_slots;
};

// One paired difference: (up - down) / 2h, or ((up - base) + (down - base)) / h^2.
struct BumpPair {
    uint32_t up, down, base;
    int32_t second;
    double h;
};

size_t scenario_smem_bytes(uint32_t max_nodes, uint32_t max_slots);
cudaError_t launch_scenarios(const ScenarioLaunch& L, size_t smem, cudaStream_t stream);
// Tile records [pair][tile] of the paired per-unit differences (pseudo-MC).
cudaError_t launch_bump_pairs(const double* unit_prices, uint64_t units, const BumpPair* pairs, uint32_t pair_count,
                              StatRecord* partials, cudaStream_t stream);

}  // namespace mcg

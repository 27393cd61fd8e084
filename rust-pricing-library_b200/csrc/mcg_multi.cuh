// mcg_multi.cuh -- device layout of a correlated multi-asset plan, shared by
// the host compiler (mcg_host.cu) and the kernel (mcg_multi.cu).
#pragma once

#include "mcg_kernels.cuh"

namespace mcg {

constexpr int kMaxAssets = MCG_MAX_ASSETS;

// Flat device arrays plus this POD header, passed to the kernel by value.
struct MultiAssetDev {
    uint32_t n, steps, dimension;
    int32_t engine, antithetic, bridge, rank_major;
    uint64_t seed, units;
    // per step of the common time grid
    const double* dt;
    const double* sqrt_dt;
    const double* inv_sqrt_dt;
    const int32_t* step_entry;  // correlation entry of the interval
    const double* lower;        // entries x n x n lower Cholesky factors
    // per asset (index i), per step arrays at [i * steps + s]
    int32_t model[kMaxAssets];
    double vol[kMaxAssets], spot[kMaxAssets];
    const double* ratio;        // forward ratios F_{s+1} / F_s
    const int32_t* time_cell;   // local volatility: grid time cell of the step
    const double* time_weight;
    int32_t nx[kMaxAssets];
    const double2* bounds[kMaxAssets];  // local volatility: cell bounds {x[c], x[c+1]}
    const double2* cells[kMaxAssets];   // local volatility: {v[t][c], slope} per row and cell
    double x_first[kMaxAssets], x_last[kMaxAssets];
    // the dimensions of the unit's normals in the order the kernel consumes
    // them (per step: the bridge nodes' ranks x factors, or the step x factors)
    const uint32_t* z_dims;
    uint32_t z_count;
    // the one-factor bridge program of the common grid
    const int4* step_prog;
    const BridgeNode* bridge_nodes;
    int32_t zero_slot;
    uint32_t slot_count;
    // RQMC: scrambled direction table [scramble][dim][32], shifts, low words
    const uint32_t* scr_dirs;
    const uint32_t* scr_shift;
    const uint32_t* scr_low;
    // product
    int32_t product, side;
    double strike, notional, smoothing, df;
    double weights[kMaxAssets], scales[kMaxAssets];
};

size_t multi_asset_smem(const MultiAssetDev& M);
cudaError_t launch_multi_asset(const MultiAssetDev& M, uint32_t scrambles, StatRecord* partials, ErrorWord* err,
                               cudaStream_t stream);

}  // namespace mcg

// mcg_plan.h -- device-resident plan layout shared by the host compiler
// (mcg_host.cu) and the path kernels.
//
// A compiled plan is a set of flat device arrays plus this POD header, passed
// to every kernel by value.  The layout follows the reference's immutable
// SimulationPlan (crates/pricing/src/engine/plan/simulation.rs:73-119) and
// LocalVolRuntime (:129-140), re-laid out for one-thread-per-path kernels:
// per-step constants are structure-of-arrays in global memory (read uniformly
// by a warp), the local-variance grid is staged in shared memory.
#pragma once

#include <cstdint>

#include "../../include/mcg.h"

namespace mcg {

constexpr int kMaxProducts = MCG_MAX_PRODUCTS;
constexpr int kComponents = MCG_PATHWISE_COMPONENTS;
constexpr int kMaxBridgeSlots = 32;

// Path program opcodes.  A Brownian-bridge plan is compiled into a
// time-ordered program: node values are produced just before the step that
// needs them and live in a few shared-memory slots (crates/pricing/src/engine/sampling/bridge.rs:272-311
// evaluates the same linear map in heap order over a full array).
enum OpKind : int32_t {
    kOpTerminal = 0,  // W[out] = sd * z[rank]
    kOpInterior = 1,  // W[out] = wl * W[left] + wr * W[right] + sd * z[rank]
    kOpStep = 2,      // shock = (W[right] - W[left]) * inv_sqrt_dt[step]; evolve one step
    kOpStepDirect = 3, // shock = z[rank]; evolve one step
    kOpZero = 4        // W[out] = 0 (the bridge's time-zero node)
};

struct Op {
    int32_t kind;
    int32_t out;    // slot written (terminal/interior)
    int32_t left;   // slot read
    int32_t right;  // slot read
    int32_t rank;   // normal dimension
    int32_t step;   // step index (step ops)
    double wl, wr, sd;
};

// Per-step constants of the base runtime, one 48-byte record per step (three
// 16-byte loads, read uniformly by a warp).
struct __align__(16) LvStep {
    double dt, sqrt_dt, inv_sqrt_dt, time_weight, ratio;
    int32_t time_cell;
    int32_t obs_next;  // observation index of node s + 1, or -1
};

// The path tiles' program, one int4 per step: the Brownian-bridge nodes
// produced just before the step, bridge_nodes[x, x + y), and the slots of the
// step's two bracketing values W(t_s), W(t_{s+1}) in z, w (-1: the step takes
// its normal directly, dimension s).  The tiles walk the steps with no
// per-op dispatch, reading this record before the nodes and the step's
// constants after them.
// One Brownian-bridge node of the path tiles: W[out] = wl W[left] + wr W[right]
// + sd z[rank].  The terminal node is the same form with wl = wr = 0 and both
// reads from the W(0) slot, which holds 0.0 when the terminal is produced
// (it is the first node of every program), so it is sd z bit for bit.
struct __align__(16) BridgeNode {
    double wl, wr, sd;
    int32_t out, left, right, rank;
};

struct ProductParams {
    int32_t kind, side;
    double strike, notional;
    int32_t digital_payout;
    double payout;
    int32_t barrier_direction, barrier_style, has_rebate;
    double barrier, rebate;
    const double* weights;  // device, one per observation (Asian weights; barrier/lookback monitoring flags)
    int32_t has_initial;    // seasoned state (Asian known-fixing sum, lookback extremum, barrier hit)
    double initial;
};

struct DevicePlan {
    int32_t model, engine, precision;
    int32_t antithetic;
    uint64_t seed;
    uint64_t units;          // pseudo: units; rqmc: points per scramble
    uint32_t scramble_count;
    uint32_t steps;          // time steps of one path
    uint32_t observation_count;
    uint32_t product_count;
    uint32_t dimension;      // Sobol / Philox dimensions per path
    int32_t zero_variance;   // BS with total variance 0: normals are zero

    // program
    const Op* ops;
    uint32_t op_count;
    const uint32_t* z_ranks;  // local volatility: the normal ranks the program consumes, in order
    uint32_t z_count;
    uint32_t slot_count;

    // per-step constants (steps entries unless noted)
    const double* node_time;     // steps + 1
    const double* dt;
    const double* sqrt_dt;
    const double* inv_sqrt_dt;
    const int32_t* obs_of_node;  // steps + 1: observation index or -1
    const int32_t* time_cell;    // LV: grid time cell per step
    const double* time_weight;   // LV: grid time weight per step
    const double* fwd;           // LV: 3 x (steps + 1) forward normalizers (base, down, up)
    const double* ratio;         // LV: 3 x steps forward ratios F[i+1]/F[i]
    const float* fwd_f;          // FP32 bulk: reciprocal base forward normalisers 1/F_i (steps + 1)
    const float* ratio_f;        // FP32 bulk: base forward ratios F_{i+1}/F_i (steps)
    const float4* step_f;        // FP32 bulk: per step {dt, sqrt(dt), time weight, 1/sqrt(dt)}
    const LvStep* lv_steps;      // LV: the base runtime's per-step constants, packed
    const int4* step_prog;       // LV: the path tiles' program, one record per step
    const BridgeNode* bridge_nodes;  // LV: the bridge nodes of the path tiles, in program order
    int32_t zero_slot;           // LV bridge: the slot holding W(0) = 0 at the start of a path

    // Black--Scholes observation data (observation_count entries)
    const double* obs_time;
    const double* obs_fwd;
    const double* obs_sqrt_step;
    double spot, vol, discount, expiry;
    double spot_variant[3];      // base, down, up spots

    // local-variance grid
    const double* grid_t;
    const double* grid_x;
    const double* grid_v;
    const double* grid_vol2;     // 2 sqrt(v) of every grid value (local Vega per node adjoint)
    // Per row t and x cell c: {v[t][c], (v[t][c+1] - v[t][c]) / (x[c+1] - x[c])}, the
    // path tiles' form of the grid (nt x (nx - 1) entries, read through L1)
    const double2* grid_cells;
    const float* grid_v_f;
    uint32_t nt, nx;

    // RQMC: scrambled direction table [scramble][dim][32] and shifts [scramble][dim]
    const uint32_t* scr_dirs;
    const uint32_t* scr_shift;
    // RQMC: per-lane low Gray-code words [scramble][dim][32]: for lane l the
    // XOR of the table words of the set bits of gray(l)
    const uint32_t* scr_low;

    // risk
    int32_t risk;          // BS: pathwise values with bumps
    int32_t req_gamma;
    int32_t lv_bumps;      // LV: CRN delta/gamma evolutions
    double gamma_bump, spot_bump, vol_bump;
    double smoothing;
    // Discrete dividends (escrowed affine model; null without dividends): per
    // observation its coordinate {a, b, spot_scale, 1 when the observation is
    // an ex-date} at the plan's spot and the coordinate just before that
    // ex-date's dividend {a, b, spot_scale, 0}; local volatility: per spot
    // runtime (base, down, up) and observation {a, b, pre a, pre b} at the
    // runtime's spot, observation i of runtime w at lv_obs_div[w * n + i].
    int32_t dividends;
    const double4* obs_div;
    const double4* obs_div_pre;
    const double4* lv_obs_div;
    // BS pathwise risk of a multi-observation product: per-thread scratch of
    // `bs_tape_units` threads x bs_tape_rows rows ([row][thread]).
    double* bs_tape;
    int32_t bs_sweep;  // 1: the single-sweep kernel (no tape) prices this plan's path risk
    uint64_t bs_tape_units;
    uint32_t bs_tape_rows;

    ProductParams products[kMaxProducts];
};

// Per-CTA statistics record of one component.
struct StatRecord {
    double sum, corr, count, mean, m2;
};

}  // namespace mcg

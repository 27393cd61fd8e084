// mcg_host.cu -- plan compiler and C ABI of the B200 Monte Carlo engine.
//
// mcg_plan_create turns an mcg_plan_desc into device-resident plan data:
//   * the local-volatility time grid (LocalVolTimeGrid::compile,
//     crates/pricing/src/engine/processes/local_vol.rs:167-237) and forward
//     normalisers for the base and the two bumped spots
//     (crates/pricing/src/engine/compile/local_vol.rs:14-102,
//      crates/pricing/src/engine/processes/local_vol_valuation.rs:24-68),
//   * the Brownian-bridge plan (crates/pricing/src/engine/sampling/bridge.rs:177-208,395-467)
//     recompiled into a time-ordered program with a handful of live slots,
//   * the RQMC scramble table, pre-applied to the Joe--Kuo directions on the device,
//   * per-step constants (dt, sqrt(dt), grid time cell and weight, forward ratios).
// mcg_plan_evaluate launches the path kernel and the tile reduction, merges
// the per-scramble records and builds the estimates of
// crates/pricing/src/engine/risk/report.rs:454-473.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <cstdio>
#include <cstring>
#include <limits>
#include <queue>
#include <string>
#include <vector>

#include "mcg_kernels.cuh"
#include "mcg_lsm.cuh"
#include "mcg_mlp.cuh"
#include "mcg_book.cuh"
#include "mcg_surface.cuh"
#include "mcg_dividends.h"
#include "mcg_multi.cuh"
#include "mcg_bump.cuh"

namespace mcg {
cudaError_t launch_lv_path(const DevicePlan& P, uint64_t unit_begin, uint64_t units, uint32_t scrambles,
                           StatRecord* partials, uint32_t mask, ErrorWord* err, int detail,
                           cudaStream_t stream, int& evolutions_out);
cudaError_t launch_lv32_path(const DevicePlan& P, StatRecord* partials, uint32_t mask, ErrorWord* err,
                             cudaStream_t stream);
cudaError_t launch_bs_path(const DevicePlan& P, bool single_terminal, uint64_t unit_begin, uint64_t units,
                           uint32_t scrambles, StatRecord* partials, uint32_t mask, ErrorWord* err,
                           int detail, cudaStream_t stream);
__global__ void scramble_table_kernel(const uint32_t*, uint32_t, uint32_t, uint32_t, uint64_t, uint32_t*,
                                      uint32_t*);
__global__ void reduce_tiles_kernel(const StatRecord*, uint32_t, uint32_t, StatRecord*);
__global__ void scramble_low_kernel(const uint32_t*, uint32_t, uint32_t*);
__global__ void philox_normals_kernel(uint64_t, uint64_t, uint64_t, uint32_t, uint32_t, double*);
__global__ void rqmc_words_kernel(const uint32_t*, const uint32_t*, uint32_t, uint32_t, uint64_t,
                                  uint64_t, uint32_t*);
__global__ void rqmc_words_warp_kernel(const uint32_t*, const uint32_t*, const uint32_t*, uint32_t, uint32_t,
                                       uint64_t, uint64_t, uint32_t*);
__global__ void fp64_peak_kernel(double*, int);
struct AdjointArgs {
    int32_t which;
    double sign;
    double node_weight;
    int32_t node_add;
    uint32_t scramble;
    uint64_t unit_begin;
    uint64_t units;
    uint32_t tile_offset;
    double* tape_f;
    double* tape_z;
    double* out_vega;
    double* out_delta;
    double* node_tiles;
    double* out_price;
    double* out_diag;
    const uint32_t* stops;
    uint32_t stop_stride;
    const double* exercise_df;
};
cudaError_t launch_lv_adjoint_price(const double* price, const double* diag, uint64_t units, int pairs,
                                    uint32_t tile_offset, uint32_t mask, StatRecord* partials, cudaStream_t stream);
cudaError_t launch_lv_fixed_policy_combine(const double* price, const double* vega, uint64_t units, int pairs,
                                           int crn, int gamma, int want_vega, double h, uint32_t tile_offset,
                                           StatRecord* partials, cudaStream_t stream);
size_t lv_adjoint_smem(const DevicePlan& P);
cudaError_t launch_lv_adjoint(const DevicePlan& P, const AdjointArgs& A, ErrorWord* err, cudaStream_t stream);
cudaError_t launch_lv_adjoint_combine(const double* vega, const double* delta, uint64_t units, int pairs,
                                      int have_gamma, double h, uint32_t tile_offset, StatRecord* partials,
                                      cudaStream_t stream);
cudaError_t launch_lv_node_reduce(const double* node_tiles, uint32_t tiles_per_scramble, uint32_t scrambles,
                                  uint32_t nv, StatRecord* out, cudaStream_t stream);
}  // namespace mcg

using namespace mcg;

namespace {

thread_local std::string g_last_error;

mcg_status fail(mcg_status code, const std::string& message) {
    g_last_error = message;
    return code;
}

uint64_t bits_of(double v) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
}

int64_t host_total_key(double x) {
    int64_t b;
    std::memcpy(&b, &x, 8);
    return b ^ static_cast<int64_t>(static_cast<uint64_t>(b >> 63) >> 1);
}

// Index of the first element whose total-order key is >= key.
size_t lower_bound_key(const std::vector<double>& v, int64_t key) {
    size_t lo = 0, hi = v.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (host_total_key(v[mid]) < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Log-linear discount curve (crates/pricing/src/market/curve.rs:156-205).
struct HostCurve {
    std::vector<double> t, logs;
    double log_discount(double time) const {
        if (time == 0.0) time = 0.0;
        const int64_t key = host_total_key(time);
        const size_t lo = lower_bound_key(t, key);
        if (lo < t.size() && host_total_key(t[lo]) == key) return logs[lo];
        const size_t right = lo < t.size() ? lo : t.size() - 1;
        const size_t left = right - 1;
        const double w = (time - t[left]) / (t[right] - t[left]);
        return logs[left] + w * (logs[right] - logs[left]);
    }
};

bool load_curve(const mcg_curve& c, HostCurve& out, const char* name, std::string& why) {
    if (c.pillar_count < 2 || !c.times || !c.discount_factors) {
        why = std::string(name) + ": needs at least two pillars";
        return false;
    }
    if (c.times[0] != 0.0 || c.discount_factors[0] != 1.0) {
        why = std::string(name) + ": the first pillar must be time 0 with discount 1";
        return false;
    }
    for (uint32_t i = 0; i < c.pillar_count; ++i) {
        if (!std::isfinite(c.times[i]) || !std::isfinite(c.discount_factors[i]) ||
            c.discount_factors[i] <= 0.0 || (i > 0 && !(c.times[i] > c.times[i - 1]))) {
            why = std::string(name) + ": pillar " + std::to_string(i) + " is invalid";
            return false;
        }
    }
    out.t.assign(c.times, c.times + c.pillar_count);
    out.t[0] = 0.0;
    out.logs.resize(c.pillar_count);
    for (uint32_t i = 0; i < c.pillar_count; ++i) out.logs[i] = std::log(c.discount_factors[i]);
    return true;
}

// ---------------------------------------------------------- bridge plan

struct BridgeInstr {
    bool terminal;
    uint32_t node, left, right, rank;
    double wl, wr, sd;
};

struct Candidate {
    double variance, time;
    uint32_t node, left, right;
};

// IntervalCandidate's order (bridge.rs:149-160): variance, then the earlier
// time, then the smaller node wins.
bool candidate_less(const Candidate& a, const Candidate& b) {
    const int64_t va = host_total_key(a.variance), vb = host_total_key(b.variance);
    if (va != vb) return va < vb;
    const int64_t ta = host_total_key(a.time), tb = host_total_key(b.time);
    if (ta != tb) return ta > tb;
    return a.node > b.node;
}

bool best_candidate(const std::vector<double>& t, uint32_t left, uint32_t right, Candidate& best,
                    bool& any) {
    any = false;
    if (right <= left + 1) return true;
    const double den = t[right] - t[left];
    for (uint32_t node = left + 1; node < right; ++node) {
        const double variance = ((t[node] - t[left]) * (t[right] - t[node])) / den;
        if (!std::isfinite(variance) || variance <= 0.0) return false;
        const Candidate c{variance, t[node], node, left, right};
        if (!any || candidate_less(best, c)) best = c;
        any = true;
    }
    return true;
}

bool compile_bridge(const std::vector<double>& t, std::vector<BridgeInstr>& out) {
    out.clear();
    const uint32_t terminal = static_cast<uint32_t>(t.size() - 1);
    out.push_back({true, terminal, 0, 0, 0, 0.0, 0.0, std::sqrt(t[terminal])});
    auto cmp = [](const Candidate& a, const Candidate& b) { return candidate_less(a, b); };
    std::priority_queue<Candidate, std::vector<Candidate>, decltype(cmp)> heap(cmp);
    Candidate c;
    bool any;
    if (!best_candidate(t, 0, terminal, c, any)) return false;
    if (any) heap.push(c);
    uint32_t rank = 1;
    while (!heap.empty()) {
        const Candidate top = heap.top();
        heap.pop();
        const double den = t[top.right] - t[top.left];
        out.push_back({false, top.node, top.left, top.right, rank++,
                       (t[top.right] - t[top.node]) / den, (t[top.node] - t[top.left]) / den,
                       std::sqrt(top.variance)});
        if (!best_candidate(t, top.left, top.node, c, any)) return false;
        if (any) heap.push(c);
        if (!best_candidate(t, top.node, top.right, c, any)) return false;
        if (any) heap.push(c);
    }
    return true;
}

// Time-ordered program of a bridge: node values are produced on demand (the
// right bracketing node first), each value lives in a slot from its
// computation to its last read.  Returns false when more than kMaxBridgeSlots
// values would be live at once.
bool bridge_program(const std::vector<double>& t, const std::vector<BridgeInstr>& instrs,
                    std::vector<Op>& ops, uint32_t& slot_count) {
    const uint32_t n = static_cast<uint32_t>(t.size());  // nodes 0..n-1
    std::vector<int> by_node(n, -1);
    for (size_t i = 0; i < instrs.size(); ++i) by_node[instrs[i].node] = static_cast<int>(i);
    std::vector<char> done(n, 0);
    done[0] = 1;
    // (kind, node or step) in execution order
    struct Raw {
        int kind;
        uint32_t a;
    };
    std::vector<Raw> order;
    std::vector<uint32_t> stack;
    for (uint32_t s = 0; s + 1 < n; ++s) {
        // ensure(s + 1): walk up the right brackets until a computed node.
        stack.clear();
        uint32_t m = s + 1;
        while (!done[m]) {
            stack.push_back(m);
            const BridgeInstr& in = instrs[by_node[m]];
            if (in.terminal) break;
            m = in.right;
        }
        while (!stack.empty()) {
            const uint32_t node = stack.back();
            stack.pop_back();
            order.push_back({0, node});
            done[node] = 1;
        }
        order.push_back({1, s});
    }
    // last use of every node value
    std::vector<int> last(n, -1);
    for (size_t i = 0; i < order.size(); ++i) {
        if (order[i].kind == 0) {
            const BridgeInstr& in = instrs[by_node[order[i].a]];
            if (!in.terminal) {
                last[in.left] = static_cast<int>(i);
                last[in.right] = static_cast<int>(i);
            }
        } else {
            last[order[i].a] = static_cast<int>(i);
            last[order[i].a + 1] = static_cast<int>(i);
        }
    }
    std::vector<int> slot_of(n, -1);
    std::vector<int> free_slots;
    uint32_t used = 0;
    auto take = [&]() -> int {
        if (!free_slots.empty()) {
            const int sl = free_slots.back();
            free_slots.pop_back();
            return sl;
        }
        return static_cast<int>(used++);
    };
    slot_of[0] = take();  // W(0) = 0
    ops.clear();
    ops.push_back({kOpZero, slot_of[0], 0, 0, 0, 0, 0.0, 0.0, 0.0});  // W(0) = 0
    for (size_t i = 0; i < order.size(); ++i) {
        if (order[i].kind == 0) {
            const uint32_t node = order[i].a;
            const BridgeInstr& in = instrs[by_node[node]];
            const int out = take();
            slot_of[node] = out;
            Op op{};
            op.kind = in.terminal ? kOpTerminal : kOpInterior;
            op.out = out;
            op.left = in.terminal ? 0 : slot_of[in.left];
            op.right = in.terminal ? 0 : slot_of[in.right];
            op.rank = static_cast<int32_t>(in.rank);
            op.wl = in.wl;
            op.wr = in.wr;
            op.sd = in.sd;
            ops.push_back(op);
        } else {
            const uint32_t s = order[i].a;
            Op op{};
            op.kind = kOpStep;
            op.left = slot_of[s];
            op.right = slot_of[s + 1];
            op.step = static_cast<int32_t>(s);
            ops.push_back(op);
        }
        // release values whose last read was this op
        auto release = [&](uint32_t node) {
            if (last[node] == static_cast<int>(i) && slot_of[node] >= 0) {
                free_slots.push_back(slot_of[node]);
                slot_of[node] = -1;
            }
        };
        if (order[i].kind == 0) {
            const BridgeInstr& in = instrs[by_node[order[i].a]];
            if (!in.terminal) {
                release(in.left);
                release(in.right);
            }
        } else {
            release(order[i].a);
            release(order[i].a + 1);
        }
    }
    slot_count = used;
    return used <= static_cast<uint32_t>(kMaxBridgeSlots);
}

// The path tiles' form of a program: per step, the bridge nodes produced just
// before it (the terminal as a node with zero weights reading the W(0) slot)
// and its bracketing slots.  False if the steps are not in order.
bool step_program(const std::vector<Op>& ops, uint32_t steps, std::vector<int4>& prog,
                  std::vector<BridgeNode>& bnodes, int32_t& zero_slot) {
    prog.assign(steps, make_int4(0, 0, -1, -1));
    bnodes.clear();
    zero_slot = 0;
    size_t pending = 0;
    uint32_t next_step = 0;
    for (const Op& op : ops) {
        if (op.kind == kOpZero) {
            zero_slot = op.out;
        } else if (op.kind == kOpTerminal) {
            bnodes.push_back(BridgeNode{0.0, 0.0, op.sd, op.out, zero_slot, zero_slot, op.rank});
        } else if (op.kind == kOpInterior) {
            bnodes.push_back(BridgeNode{op.wl, op.wr, op.sd, op.out, op.left, op.right, op.rank});
        } else {
            if (op.step != static_cast<int32_t>(next_step) || next_step >= steps) return false;
            int4& r = prog[next_step++];
            r.x = static_cast<int32_t>(pending);
            r.y = static_cast<int32_t>(bnodes.size() - pending);
            pending = bnodes.size();
            if (op.kind == kOpStep) {
                r.z = op.left;
                r.w = op.right;
            }
        }
    }
    return next_step == steps && pending == bnodes.size();
}

template <class T>
struct DeviceArray {
    T* ptr = nullptr;
    size_t count = 0;
    cudaError_t upload(const std::vector<T>& v) {
        count = v.size();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&ptr, count * sizeof(T));
        if (e != cudaSuccess) return e;
        return cudaMemcpy(ptr, v.data(), count * sizeof(T), cudaMemcpyHostToDevice);
    }
    cudaError_t alloc(size_t n) {
        count = n;
        return n ? cudaMalloc(&ptr, n * sizeof(T)) : cudaSuccess;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
    }
};

}  // namespace

struct mcg_plan {
    DevicePlan dp{};
    bool single_terminal = false;
    uint32_t product_count = 0;
    uint32_t mask = 1u;  // components reduced on the device
    uint32_t slots = 1;  // popcount(mask)
    double total_variance = 0.0;
    uint32_t grid_values = 0;
    std::vector<ProductParams> products;
    // device storage
    DeviceArray<Op> ops;
    DeviceArray<uint32_t> z_ranks;
    DeviceArray<double> node_time, dt, sqrt_dt, inv_sqrt_dt, time_weight, fwd, ratio, obs_time,
        obs_fwd, obs_sqrt_step, grid_t, grid_x, grid_v, grid_vol2, weights;
    DeviceArray<int32_t> obs_of_node, time_cell;
    DeviceArray<double4> obs_div, obs_div_pre, lv_obs_div;
    DeviceArray<LvStep> lv_steps;
    DeviceArray<int4> step_prog;
    DeviceArray<BridgeNode> bridge_nodes;
    DeviceArray<double2> grid_cells;
    DeviceArray<uint32_t> scr_dirs, scr_shift, scr_low, directions;
    DeviceArray<StatRecord> partials, records;
    DeviceArray<ErrorWord> error;
    uint32_t tiles = 0;
    // local-volatility adjoint (Vega, adjoint Delta/Gamma, node sensitivities)
    bool adjoint = false, adjoint_nodes = false, adjoint_gamma = false;
    bool price_from_adjoint = false;  // no CRN runtimes: the sweeps' forward passes give the price
    uint64_t chunk_units = 0;
    DeviceArray<double> tape, adj_vega, adj_delta, node_tiles, adj_price, adj_diag;
    DeviceArray<StatRecord> adj_partials, adj_records, node_records;
    DeviceArray<float> fwd_f, ratio_f;
    DeviceArray<float4> step_f;

    ~mcg_plan() {
        fwd_f.release();
        ratio_f.release();
        step_f.release();
        ops.release();
        z_ranks.release();
        node_time.release();
        dt.release();
        sqrt_dt.release();
        inv_sqrt_dt.release();
        time_weight.release();
        fwd.release();
        ratio.release();
        obs_time.release();
        obs_fwd.release();
        obs_sqrt_step.release();
        grid_t.release();
        grid_x.release();
        grid_v.release();
        grid_vol2.release();
        weights.release();
        obs_of_node.release();
        time_cell.release();
        obs_div.release();
        obs_div_pre.release();
        lv_obs_div.release();
        lv_steps.release();
        step_prog.release();
        bridge_nodes.release();
        grid_cells.release();
        scr_dirs.release();
        scr_shift.release();
        scr_low.release();
        directions.release();
        partials.release();
        records.release();
        error.release();
        tape.release();
        adj_vega.release();
        adj_delta.release();
        adj_price.release();
        adj_diag.release();
        node_tiles.release();
        adj_partials.release();
        adj_records.release();
        node_records.release();
    }
};

namespace {

#define MCG_CUDA(call)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? MCG_ERR_ALLOCATION : MCG_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

// LocalVolTimeGrid::compile, local_vol.rs:167-237.
void compile_time_grid(std::vector<double> events, double maximum_step, std::vector<double>& nodes) {
    std::sort(events.begin(), events.end(),
              [](double a, double b) { return host_total_key(a) < host_total_key(b); });
    events.erase(std::unique(events.begin(), events.end(),
                             [](double a, double b) { return bits_of(a) == bits_of(b); }),
                 events.end());
    if (bits_of(events[0]) != 0) events.insert(events.begin(), 0.0);
    nodes.assign(1, 0.0);
    for (size_t i = 0; i + 1 < events.size(); ++i) {
        const double left = events[i], right = events[i + 1];
        if (right <= left) continue;
        const double interval = right - left;
        const double steps_f = std::ceil(interval / maximum_step);
        const size_t steps = steps_f < 1.0 ? 1 : static_cast<size_t>(steps_f);
        const double sub = interval / static_cast<double>(steps);
        for (size_t k = 1; k < steps; ++k) nodes.push_back(left + sub * static_cast<double>(k));
        nodes.push_back(right);
    }
}

mcg_status validate_products(const mcg_plan_desc* d, std::vector<ProductParams>& out, bool& single) {
    if (d->product_count == 0 || d->product_count > MCG_MAX_PRODUCTS || !d->products)
        return fail(MCG_ERR_INVALID_ARGUMENT, "product_count must be 1..8");
    single = d->observation_count == 1;
    for (uint32_t i = 0; i < d->product_count; ++i) {
        const mcg_product_desc& p = d->products[i];
        ProductParams q{};
        q.kind = p.kind;
        q.side = p.side;
        q.strike = p.strike;
        q.notional = p.notional;
        q.digital_payout = p.digital_payout;
        q.payout = p.payout;
        q.barrier_direction = p.barrier_direction;
        q.barrier_style = p.barrier_style;
        q.has_rebate = p.has_rebate;
        q.barrier = p.barrier;
        q.rebate = p.rebate;
        q.has_initial = p.has_initial_state != 0;
        q.initial = p.initial_state;
        if (p.kind < MCG_PRODUCT_EUROPEAN || p.kind > MCG_PRODUCT_CONTINUOUS_BARRIER)
            return fail(MCG_ERR_UNSUPPORTED, "product kind " + std::to_string(p.kind));
        if (!(p.notional > 0.0) || !std::isfinite(p.strike) || p.strike <= 0.0)
            return fail(MCG_ERR_INVALID_ARGUMENT, "product strike/notional must be positive");
        if ((p.kind == MCG_PRODUCT_DISCRETE_BARRIER || p.kind == MCG_PRODUCT_CONTINUOUS_BARRIER) &&
            !(p.barrier > 0.0))
            return fail(MCG_ERR_INVALID_ARGUMENT, "barrier level must be positive");
        if (p.kind == MCG_PRODUCT_ASIAN && !p.observation_weights)
            return fail(MCG_ERR_INVALID_ARGUMENT, "Asian product needs observation weights");
        if (p.has_initial_state) {
            if (p.kind != MCG_PRODUCT_ASIAN && p.kind != MCG_PRODUCT_LOOKBACK &&
                p.kind != MCG_PRODUCT_DISCRETE_BARRIER)
                return fail(MCG_ERR_UNSUPPORTED, "seasoned state of a product without observation history");
            if (!std::isfinite(p.initial_state) ||
                (p.kind == MCG_PRODUCT_DISCRETE_BARRIER && p.initial_state != 0.0 && p.initial_state != 1.0))
                return fail(MCG_ERR_INVALID_ARGUMENT, "initial_state");
        }
        if (p.kind != MCG_PRODUCT_EUROPEAN && p.kind != MCG_PRODUCT_DIGITAL) single = false;
        out.push_back(q);
    }
    return MCG_OK;
}

double resolve_gamma_bump(const mcg_plan_desc* d) {
    return d->gamma_bump_relative ? d->spot * d->gamma_bump : d->gamma_bump;
}

mcg_status build(const mcg_plan_desc* d, mcg_plan& plan, bool reduction_buffers = true) {
    if (!d) return fail(MCG_ERR_INVALID_ARGUMENT, "null descriptor");
    if (d->abi_version != MCG_ABI_VERSION) return fail(MCG_ERR_INVALID_ARGUMENT, "abi_version mismatch");
    if (d->model != MCG_MODEL_BLACK_SCHOLES && d->model != MCG_MODEL_LOCAL_VOLATILITY)
        return fail(MCG_ERR_UNSUPPORTED, "model");
    if (d->engine != MCG_ENGINE_PSEUDO && d->engine != MCG_ENGINE_RQMC)
        return fail(MCG_ERR_UNSUPPORTED, "engine");
    if (d->precision != MCG_PRECISION_F64 && d->precision != MCG_PRECISION_F32_BULK)
        return fail(MCG_ERR_INVALID_ARGUMENT, "precision");
    if (d->precision == MCG_PRECISION_F32_BULK &&
        (d->model != MCG_MODEL_LOCAL_VOLATILITY || d->request_delta || d->request_gamma || d->request_vega ||
         d->request_local_vega_nodes))
        return fail(MCG_ERR_UNSUPPORTED, "the FP32 path bulk prices local-volatility plans without risk");
    if (!(d->spot > 0.0) || !std::isfinite(d->spot)) return fail(MCG_ERR_INVALID_ARGUMENT, "spot");
    if (d->observation_count == 0 || !d->observation_times)
        return fail(MCG_ERR_INVALID_ARGUMENT, "observation_times");
    // A Black-Scholes path may observe the valuation date itself (time 0: a
    // zero-length step that still takes its normal, as the reference's
    // path_observations_from_normals does); every other plan starts after it.
    bool time_zero_ok = d->model == MCG_MODEL_BLACK_SCHOLES && d->observation_count > 1;
    for (uint32_t i = 0; i < d->product_count && d->products; ++i)
        time_zero_ok &= d->products[i].kind != MCG_PRODUCT_AMERICAN;
    for (uint32_t i = 0; i < d->observation_count; ++i) {
        const double t = d->observation_times[i];
        const bool zero_first = i == 0 && t == 0.0 && time_zero_ok;
        if (!std::isfinite(t) || (t <= 0.0 && !zero_first) || (i && !(t > d->observation_times[i - 1])))
            return fail(MCG_ERR_INVALID_ARGUMENT, "observation_times must be positive and increasing");
    }
    if (d->sampling_units == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "sampling_units");
    if (d->engine == MCG_ENGINE_RQMC) {
        if (d->scramble_count == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "scramble_count");
        if ((d->sampling_units & (d->sampling_units - 1)) != 0 || d->sampling_units > (1ull << 32))
            return fail(MCG_ERR_INVALID_ARGUMENT, "points_per_scramble must be a power of two <= 2^32");
    }
    HostCurve rc, qc;
    std::string why;
    if (!load_curve(d->discount_curve, rc, "discount_curve", why)) return fail(MCG_ERR_MARKET, why);
    if (!load_curve(d->dividend_curve, qc, "dividend_curve", why)) return fail(MCG_ERR_MARKET, why);
    auto forward = [&](double spot, double t) {
        return spot * std::exp(qc.log_discount(t) - rc.log_discount(t));
    };
    bool single;
    mcg_status st = validate_products(d, plan.products, single);
    if (st != MCG_OK) return st;
    const uint32_t n = d->observation_count;
    const double expiry = d->observation_times[n - 1];
    const bool lv = d->model == MCG_MODEL_LOCAL_VOLATILITY;
    // Discrete dividends: the escrowed affine transform at the plan's spot.
    HostDividends<HostCurve> divs;
    const bool dividends = d->discrete_dividends.count > 0;
    double residual_spot = d->spot;
    if (dividends) {
        if (!divs.compile(d->discrete_dividends, d->spot, rc, qc, why)) return fail(MCG_ERR_MARKET, why);
        residual_spot = d->spot - divs.reserve;
        for (uint32_t i = 0; i < d->product_count; ++i)
            if (d->products[i].kind == MCG_PRODUCT_CONTINUOUS_BARRIER || d->products[i].kind == MCG_PRODUCT_AMERICAN)
                return fail(MCG_ERR_UNSUPPORTED, "discrete dividends with a continuous barrier or early exercise");
        if (d->precision != MCG_PRECISION_F64)
            return fail(MCG_ERR_UNSUPPORTED, "discrete dividends in the FP32 path bulk");
        if (lv && (d->request_vega || d->request_local_vega_nodes))
            return fail(MCG_ERR_UNSUPPORTED, "local-volatility Vega and node sensitivities with discrete dividends");
    }

    DevicePlan& P = plan.dp;
    P.model = d->model;
    P.engine = d->engine;
    P.precision = d->precision;
    P.antithetic = d->antithetic != 0;
    P.seed = d->master_seed;
    P.units = d->sampling_units;
    P.scramble_count = d->engine == MCG_ENGINE_RQMC ? d->scramble_count : 1;
    P.observation_count = n;
    P.product_count = d->product_count;
    P.spot = d->spot;
    P.vol = d->volatility;
    P.expiry = expiry;
    P.discount = std::exp(rc.log_discount(d->payment_time));
    P.smoothing = d->smoothing_half_width;
    if (!(P.smoothing >= 0.0) || !std::isfinite(P.smoothing))
        return fail(MCG_ERR_INVALID_ARGUMENT, "smoothing_half_width");
    const bool risk = d->request_delta || d->request_gamma || d->request_vega;
    // Bumps, crates/pricing/src/engine/compile/simulation.rs:481-502.
    P.req_gamma = d->request_gamma != 0;
    P.gamma_bump = resolve_gamma_bump(d);
    // With dividends the bumps stay below the escrowed spot S0 - R (compile/simulation.rs:473-489).
    if (d->request_gamma && (!std::isfinite(P.gamma_bump) || P.gamma_bump >= residual_spot || P.gamma_bump <= 0.0))
        return fail(MCG_ERR_INVALID_ARGUMENT, "gamma bump must be positive and below the (escrowed) spot");
    P.spot_bump = d->request_gamma ? P.gamma_bump : std::min(d->spot * 1.0e-4, 0.5 * residual_spot);
    P.spot_variant[0] = d->spot;
    P.spot_variant[1] = d->spot - P.spot_bump;
    P.spot_variant[2] = d->spot + P.spot_bump;
    bool has_continuous = false;
    for (auto& q : plan.products) has_continuous |= q.kind == MCG_PRODUCT_CONTINUOUS_BARRIER;

    uint32_t steps;
    if (!lv) {
        if (!(d->volatility >= 0.0) || !std::isfinite(d->volatility))
            return fail(MCG_ERR_INVALID_ARGUMENT, "volatility");
        P.vol_bump = d->volatility == 0.0 ? 0.0 : std::min(1.0e-4, d->volatility * 0.5);
        plan.total_variance = d->volatility * d->volatility * expiry;
        P.zero_variance = plan.total_variance == 0.0;
        P.risk = risk;
        if (risk && !single && d->product_count != 1)
            return fail(MCG_ERR_UNSUPPORTED, "Black-Scholes path risk prices one product per plan");
        std::vector<double> of(n), ot(n), sq(n);
        double prev = 0.0;
        for (uint32_t i = 0; i < n; ++i) {
            ot[i] = d->observation_times[i];
            of[i] = forward(d->spot, ot[i]);
            sq[i] = std::sqrt(std::max(ot[i] - prev, 0.0));
            prev = ot[i];
        }
        MCG_CUDA(plan.obs_time.upload(ot));
        MCG_CUDA(plan.obs_fwd.upload(of));
        MCG_CUDA(plan.obs_sqrt_step.upload(sq));
        P.obs_time = plan.obs_time.ptr;
        P.obs_fwd = plan.obs_fwd.ptr;
        P.obs_sqrt_step = plan.obs_sqrt_step.ptr;
        if (dividends) {
            // path_observation (black_scholes.rs:335-354): the observations'
            // coordinates and, on an ex-date, the one before its dividend
            std::vector<double4> post(n), pre(n);
            for (uint32_t i = 0; i < n; ++i) {
                const HostCoord c = divs.after_time(ot[i]);
                const long e = divs.event_at(ot[i]);
                const HostCoord b = e >= 0 ? divs.before_event(static_cast<size_t>(e)) : c;
                post[i] = make_double4(c.a, c.b, c.spot_scale, e >= 0 ? 1.0 : 0.0);
                pre[i] = make_double4(b.a, b.b, b.spot_scale, 0.0);
            }
            MCG_CUDA(plan.obs_div.upload(post));
            MCG_CUDA(plan.obs_div_pre.upload(pre));
            P.obs_div = plan.obs_div.ptr;
            P.obs_div_pre = plan.obs_div_pre.ptr;
            P.dividends = 1;
        }
        steps = n;
        P.steps = n;
        P.dimension = n;
        plan.single_terminal = single;
        plan.mask = 1u;
        if (risk) plan.mask = 0x3ffu;
        if (has_continuous) plan.mask |= 0xffu << 10;
    } else {
        // exercise-date times, for the early-exercise engine's network inputs
        MCG_CUDA(plan.obs_time.upload(std::vector<double>(d->observation_times, d->observation_times + n)));
        P.obs_time = plan.obs_time.ptr;
        plan.adjoint = d->request_vega || d->request_local_vega_nodes;
        plan.adjoint_nodes = d->request_local_vega_nodes != 0;
        plan.adjoint_gamma = plan.adjoint && d->request_delta && d->request_gamma;
        if (plan.adjoint) {
            if (d->product_count != 1)
                return fail(MCG_ERR_UNSUPPORTED, "local-volatility Vega prices one product per plan");
            if (d->products[0].kind == MCG_PRODUCT_DISCRETE_BARRIER && d->smoothing_half_width > 0.0)
                return fail(MCG_ERR_UNSUPPORTED, "local-volatility Vega of a smoothed discrete barrier");
        }
        const mcg_local_variance_grid& g = d->local_variance;
        if (g.time_count < 2 || g.log_moneyness_count < 2 || !g.time_nodes || !g.log_moneyness_nodes || !g.values)
            return fail(MCG_ERR_MARKET, "local variance grid needs at least 2x2 nodes");
        std::vector<double> gt(g.time_nodes, g.time_nodes + g.time_count);
        std::vector<double> gx(g.log_moneyness_nodes, g.log_moneyness_nodes + g.log_moneyness_count);
        std::vector<double> gv(g.values, g.values + static_cast<size_t>(g.time_count) * g.log_moneyness_count);
        for (size_t i = 0; i < gt.size(); ++i)
            if (!std::isfinite(gt[i]) || gt[i] < 0.0 || (i && !(gt[i] > gt[i - 1])))
                return fail(MCG_ERR_MARKET, "grid time nodes must be finite, non-negative and increasing");
        for (size_t i = 0; i < gx.size(); ++i)
            if (!std::isfinite(gx[i]) || (i && !(gx[i] > gx[i - 1])))
                return fail(MCG_ERR_MARKET, "grid log-moneyness nodes must be finite and increasing");
        for (size_t i = 0; i < gv.size(); ++i)
            if (!std::isfinite(gv[i]) || gv[i] < g.floor || gv[i] > g.cap)
                return fail(MCG_ERR_MARKET, "grid value " + std::to_string(i) + " outside [floor, cap]");
        if (bits_of(gt[0]) != 0 || bits_of(gt.back()) != bits_of(expiry))
            return fail(MCG_ERR_MARKET, "grid time nodes must start at +0.0 and end at the expiry time");
        double maximum_step = 0.0;
        for (size_t i = 0; i + 1 < gt.size(); ++i) maximum_step = std::max(maximum_step, gt[i + 1] - gt[i]);
        std::vector<double> events = gt;
        events.insert(events.end(), d->observation_times, d->observation_times + n);
        // ex-dividend times up to expiry are time-grid events (compile/local_vol.rs:38-52)
        for (const auto& e : divs.ev)
            if (e.t <= expiry) events.push_back(e.t);
        std::vector<double> nodes;
        compile_time_grid(events, maximum_step, nodes);
        steps = static_cast<uint32_t>(nodes.size() - 1);
        P.steps = steps;
        P.dimension = steps;
        plan.total_variance = nodes.back() * g.cap;
        std::vector<double> dtv(steps), sq(steps), isq(steps), tw(steps), fw(3 * (steps + 1)), ra(3 * steps);
        std::vector<int32_t> tc(steps), oon(steps + 1, -1);
        for (uint32_t s = 0; s < steps; ++s) {
            dtv[s] = nodes[s + 1] - nodes[s];
            sq[s] = std::sqrt(dtv[s]);
            isq[s] = 1.0 / std::sqrt(dtv[s]);
            // lower_cell under total_cmp, local_variance.rs:629-634
            const int64_t key = host_total_key(nodes[s]);
            const size_t lo = lower_bound_key(gt, key);
            size_t c = (lo < gt.size() && host_total_key(gt[lo]) == key) ? lo : (lo == 0 ? 0 : lo - 1);
            c = std::min(c, gt.size() - 2);
            tc[s] = static_cast<int32_t>(c);
            tw[s] = (nodes[s] - gt[c]) / (gt[c + 1] - gt[c]);
        }
        for (int k = 0; k < 3; ++k)
            for (uint32_t i = 0; i <= steps; ++i) {
                fw[k * (steps + 1) + i] = forward(P.spot_variant[k], nodes[i]);
                if (!std::isfinite(fw[k * (steps + 1) + i]) || fw[k * (steps + 1) + i] <= 0.0)
                    return fail(MCG_ERR_MARKET, "non-finite forward normaliser");
            }
        for (int k = 0; k < 3; ++k)
            for (uint32_t s = 0; s < steps; ++s)
                ra[k * steps + s] = fw[k * (steps + 1) + s + 1] / fw[k * (steps + 1) + s];
        for (uint32_t i = 0; i < n; ++i) {
            const uint64_t b = bits_of(d->observation_times[i]);
            uint32_t k = 0;
            while (k <= steps && bits_of(nodes[k]) != b) ++k;
            if (k > steps) return fail(MCG_ERR_MARKET, "observation time missing from the time grid");
            oon[k] = static_cast<int32_t>(i);
        }
        if (dividends) {
            // Every spot runtime's transform recompiled at its spot
            // (local_vol_runtime_for_spot, risk/pathwise_local_vol.rs:51-69); the
            // observations' node coordinates (local_vol_valuation.rs:221-247).
            std::vector<double4> lvc(3 * static_cast<size_t>(n)), post(n), pre(n);
            for (int k = 0; k < 3; ++k) {
                HostDividends<HostCurve> dk;
                if (!dk.compile(d->discrete_dividends, P.spot_variant[k], rc, qc, why))
                    return fail(MCG_ERR_MARKET, why + " (bumped spot)");
                for (uint32_t i = 0; i < n; ++i) {
                    const double t = d->observation_times[i];
                    const HostCoord c = dk.after_time(t);
                    const long e = dk.event_at(t);
                    const HostCoord b = e >= 0 ? dk.before_event(static_cast<size_t>(e)) : c;
                    lvc[k * static_cast<size_t>(n) + i] = make_double4(c.a, c.b, b.a, b.b);
                    if (k == 0) {
                        post[i] = make_double4(c.a, c.b, c.spot_scale, e >= 0 ? 1.0 : 0.0);
                        pre[i] = make_double4(b.a, b.b, b.spot_scale, 0.0);
                    }
                }
                // The post-dividend spot A S + B f of an ex-date node (its check,
                // dividend.rs:557-583) is positive for every positive f when A >= 0.
                for (const auto& e : dk.ev)
                    if (e.t <= expiry && dk.after_time(e.t).a < 0.0)
                        return fail(MCG_ERR_UNSUPPORTED, "discrete dividends: a negative cash reserve after an ex-date");
            }
            MCG_CUDA(plan.lv_obs_div.upload(lvc));
            MCG_CUDA(plan.obs_div.upload(post));
            MCG_CUDA(plan.obs_div_pre.upload(pre));
            P.lv_obs_div = plan.lv_obs_div.ptr;
            P.obs_div = plan.obs_div.ptr;
            P.obs_div_pre = plan.obs_div_pre.ptr;
            P.dividends = 1;
        }
        if (d->precision == MCG_PRECISION_F32_BULK) {
            std::vector<float> inv_f(steps + 1), ra_f(steps);
            std::vector<float4> sk(steps);
            for (uint32_t i = 0; i <= steps; ++i) inv_f[i] = static_cast<float>(1.0 / fw[i]);
            for (uint32_t i = 0; i < steps; ++i) {
                ra_f[i] = static_cast<float>(ra[i]);
                sk[i] = make_float4(static_cast<float>(dtv[i]), static_cast<float>(sq[i]), static_cast<float>(tw[i]),
                                    static_cast<float>(isq[i]));
            }
            MCG_CUDA(plan.fwd_f.upload(inv_f));
            MCG_CUDA(plan.ratio_f.upload(ra_f));
            MCG_CUDA(plan.step_f.upload(sk));
            P.fwd_f = plan.fwd_f.ptr;
            P.ratio_f = plan.ratio_f.ptr;
            P.step_f = plan.step_f.ptr;
        }
        {
            std::vector<LvStep> packed(steps);
            for (uint32_t s = 0; s < steps; ++s)
                packed[s] = LvStep{dtv[s], sq[s], isq[s], tw[s], ra[s], tc[s], oon[s + 1]};
            MCG_CUDA(plan.lv_steps.upload(packed));
            P.lv_steps = plan.lv_steps.ptr;
        }
        {
            // {v[t][c], slope of cell c} per row: the path tiles' bilinear form.
            const uint32_t ncell = g.log_moneyness_count - 1;
            std::vector<double2> cells(static_cast<size_t>(g.time_count) * ncell);
            for (uint32_t t = 0; t < g.time_count; ++t)
                for (uint32_t c = 0; c < ncell; ++c) {
                    const double* row = gv.data() + static_cast<size_t>(t) * g.log_moneyness_count;
                    const double inv = 1.0 / (gx[c + 1] - gx[c]);
                    cells[static_cast<size_t>(t) * ncell + c] = make_double2(row[c], (row[c + 1] - row[c]) * inv);
                }
            MCG_CUDA(plan.grid_cells.upload(cells));
            P.grid_cells = plan.grid_cells.ptr;
        }
        MCG_CUDA(plan.node_time.upload(nodes));
        MCG_CUDA(plan.dt.upload(dtv));
        MCG_CUDA(plan.sqrt_dt.upload(sq));
        MCG_CUDA(plan.inv_sqrt_dt.upload(isq));
        MCG_CUDA(plan.time_weight.upload(tw));
        MCG_CUDA(plan.time_cell.upload(tc));
        MCG_CUDA(plan.fwd.upload(fw));
        MCG_CUDA(plan.ratio.upload(ra));
        MCG_CUDA(plan.obs_of_node.upload(oon));
        MCG_CUDA(plan.grid_t.upload(gt));
        MCG_CUDA(plan.grid_x.upload(gx));
        MCG_CUDA(plan.grid_v.upload(gv));
        {
            std::vector<double> v2(gv.size());
            for (size_t i = 0; i < gv.size(); ++i) v2[i] = 2.0 * std::sqrt(gv[i]);
            MCG_CUDA(plan.grid_vol2.upload(v2));
        }
        P.node_time = plan.node_time.ptr;
        P.dt = plan.dt.ptr;
        P.sqrt_dt = plan.sqrt_dt.ptr;
        P.inv_sqrt_dt = plan.inv_sqrt_dt.ptr;
        P.time_weight = plan.time_weight.ptr;
        P.time_cell = plan.time_cell.ptr;
        P.fwd = plan.fwd.ptr;
        P.ratio = plan.ratio.ptr;
        P.obs_of_node = plan.obs_of_node.ptr;
        P.grid_t = plan.grid_t.ptr;
        P.grid_x = plan.grid_x.ptr;
        P.grid_v = plan.grid_v.ptr;
        P.grid_vol2 = plan.grid_vol2.ptr;
        P.nt = g.time_count;
        P.nx = g.log_moneyness_count;
        plan.grid_values = static_cast<uint32_t>(gv.size());
        P.lv_bumps = d->request_delta || d->request_gamma;
        plan.mask = 1u;
        if (P.lv_bumps) plan.mask |= (1u << MCG_DELTA) | (1u << MCG_BUMP_DELTA);
        if (d->request_gamma) plan.mask |= (1u << MCG_GAMMA) | (1u << MCG_BUMP_GAMMA);
        if (has_continuous) plan.mask |= 0xffu << 10;
        // Program: Brownian bridge on the time grid, or steps in order.
        std::vector<Op> ops;
        uint32_t slots = 1;
        if (d->brownian_bridge) {
            std::vector<BridgeInstr> instrs;
            if (!compile_bridge(nodes, instrs)) return fail(MCG_ERR_BRIDGE, "invalid bridge grid");
            if (!bridge_program(nodes, instrs, ops, slots))
                return fail(MCG_ERR_UNSUPPORTED, "bridge needs more than 32 live values");
        } else {
            for (uint32_t s = 0; s < steps; ++s) {
                Op op{};
                op.kind = kOpStepDirect;
                op.rank = static_cast<int32_t>(s);
                op.step = static_cast<int32_t>(s);
                ops.push_back(op);
            }
        }
        // Every index a kernel reads from the program stays inside its buffer.
        for (const Op& op : ops) {
            const bool slots_ok = op.out >= 0 && op.out < static_cast<int32_t>(slots) && op.left >= 0 &&
                                  op.left < static_cast<int32_t>(slots) && op.right >= 0 &&
                                  op.right < static_cast<int32_t>(slots);
            const bool rank_ok = op.rank >= 0 && op.rank < static_cast<int32_t>(steps);
            const bool step_ok = op.step >= 0 && op.step < static_cast<int32_t>(steps);
            if (!slots_ok || !rank_ok || !step_ok)
                return fail(MCG_ERR_BRIDGE, "internal: path program index out of range");
        }
        MCG_CUDA(plan.ops.upload(ops));
        P.ops = plan.ops.ptr;
        P.op_count = static_cast<uint32_t>(ops.size());
        {
            std::vector<int4> prog;
            std::vector<BridgeNode> bnodes;
            int32_t zero_slot = 0;
            if (!step_program(ops, steps, prog, bnodes, zero_slot))
                return fail(MCG_ERR_BRIDGE, "internal: path program steps out of order");
            MCG_CUDA(plan.step_prog.upload(prog));
            P.step_prog = plan.step_prog.ptr;
            MCG_CUDA(plan.bridge_nodes.upload(bnodes));
            P.bridge_nodes = plan.bridge_nodes.ptr;
            P.zero_slot = zero_slot;
        }
        std::vector<uint32_t> ranks;
        for (const Op& op : ops)
            if (op.kind == kOpTerminal || op.kind == kOpInterior || op.kind == kOpStepDirect)
                ranks.push_back(static_cast<uint32_t>(op.rank));
        MCG_CUDA(plan.z_ranks.upload(ranks));
        P.z_ranks = plan.z_ranks.ptr;
        P.z_count = static_cast<uint32_t>(ranks.size());
        P.slot_count = slots;
        const size_t smem = (gv.size() + 2 * gx.size()) * sizeof(double) +
                            static_cast<size_t>(slots) * kThreads * sizeof(double) +
                            4 * kComponents * sizeof(Stat);
        if (smem > 200 * 1024) return fail(MCG_ERR_UNSUPPORTED, "local-variance grid too large for shared memory");
    }
    // Asian weights: one device array per product, concatenated.
    {
        std::vector<double> w;
        std::vector<size_t> offsets;
        for (uint32_t i = 0; i < d->product_count; ++i) {
            offsets.push_back(w.size());
            if (d->products[i].observation_weights)
                w.insert(w.end(), d->products[i].observation_weights, d->products[i].observation_weights + n);
        }
        MCG_CUDA(plan.weights.upload(w));
        for (uint32_t i = 0; i < d->product_count; ++i) {
            plan.products[i].weights = d->products[i].observation_weights ? plan.weights.ptr + offsets[i] : nullptr;
            P.products[i] = plan.products[i];
        }
    }
    plan.product_count = d->product_count;
    plan.slots = static_cast<uint32_t>(__builtin_popcount(plan.mask));
    // RQMC scramble table.
    if (d->engine == MCG_ENGINE_RQMC) {
        if (P.dimension > MCG_MAX_SOBOL_DIMENSION)
            return fail(MCG_ERR_SOBOL_DIMENSION, "effective Sobol dimension exceeds 21201");
        if (!d->sobol_directions || d->sobol_dimension_count < P.dimension)
            return fail(MCG_ERR_SOBOL_DIMENSION, "sobol_directions cover fewer dimensions than the plan needs");
        std::vector<uint32_t> dirs(d->sobol_directions, d->sobol_directions + static_cast<size_t>(P.dimension) * 32u);
        MCG_CUDA(plan.directions.upload(dirs));
        MCG_CUDA(plan.scr_dirs.alloc(static_cast<size_t>(P.scramble_count) * P.dimension * 32u));
        MCG_CUDA(plan.scr_shift.alloc(static_cast<size_t>(P.scramble_count) * P.dimension));
        const uint32_t total = P.scramble_count * P.dimension;
        scramble_table_kernel<<<(total + 127) / 128, 128>>>(plan.directions.ptr, P.dimension, P.scramble_count,
                                                           d->scramble_begin, P.seed, plan.scr_dirs.ptr,
                                                           plan.scr_shift.ptr);
        MCG_CUDA(cudaGetLastError());
        MCG_CUDA(cudaDeviceSynchronize());
        P.scr_dirs = plan.scr_dirs.ptr;
        P.scr_shift = plan.scr_shift.ptr;
        {
            const uint32_t rows = P.scramble_count * P.dimension;
            MCG_CUDA(plan.scr_low.alloc(static_cast<size_t>(rows) * 32u));
            scramble_low_kernel<<<(rows * 32u + 127) / 128, 128>>>(plan.scr_dirs.ptr, rows, plan.scr_low.ptr);
            MCG_CUDA(cudaGetLastError());
            P.scr_low = plan.scr_low.ptr;
        }
    }
    (void)steps;
    // Reduction buffers (a book trade shares the book's).
    plan.tiles = static_cast<uint32_t>((P.units + kThreads - 1) / kThreads);
    if (!reduction_buffers) return MCG_OK;
    MCG_CUDA(plan.partials.alloc(static_cast<size_t>(P.scramble_count) * plan.tiles * plan.product_count * kComponents));
    MCG_CUDA(plan.records.alloc(static_cast<size_t>(P.scramble_count) * plan.product_count * kComponents));
    MCG_CUDA(plan.error.alloc(1));
    const bool sweep = !lv && P.risk && !plan.single_terminal && plan.product_count == 1 && !P.dividends &&
                       plan.products[0].kind != MCG_PRODUCT_CONTINUOUS_BARRIER &&
                       !(plan.products[0].kind == MCG_PRODUCT_DISCRETE_BARRIER && P.smoothing > 0.0);
    P.bs_sweep = sweep ? 1 : 0;
    if (!lv && P.risk && !plan.single_terminal && !sweep) {
        // Scratch of the path-risk kernel (at most 2 GiB): W_k and the path's
        // exponentials per thread, plus the hit state, weight and slope per
        // observation for a smoothed discrete barrier, or the observed states
        // for a continuous barrier.
        const bool smooth_barrier =
            plan.products[0].kind == MCG_PRODUCT_DISCRETE_BARRIER && P.smoothing > 0.0;
        const bool continuous = plan.products[0].kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
        P.bs_tape_rows = smooth_barrier ? (P.dividends ? 7u : 5u) * P.observation_count
                                        : (continuous ? 3u : 2u) * P.observation_count;
        const uint64_t budget = (2048ull << 20) / (sizeof(double) * P.bs_tape_rows * P.scramble_count);
        const uint64_t units_rounded = (P.units + kThreads - 1) / kThreads * kThreads;
        const uint64_t per_scramble =
            std::min<uint64_t>(units_rounded, std::max<uint64_t>(kThreads, budget / kThreads * kThreads));
        P.bs_tape_units = per_scramble * P.scramble_count;
        MCG_CUDA(plan.tape.alloc(static_cast<size_t>(P.bs_tape_rows) * P.bs_tape_units));
        P.bs_tape = plan.tape.ptr;
    }
    if (plan.adjoint) {
        // Per-step checkpoints of one chunk of units: states (steps + 1) and shocks (steps).
        plan.chunk_units = std::min<uint64_t>(P.units, 1ull << 20);
        MCG_CUDA(plan.tape.alloc(static_cast<size_t>(2 * P.steps + 1) * plan.chunk_units));
        MCG_CUDA(plan.adj_vega.alloc(6 * plan.chunk_units));
        MCG_CUDA(plan.adj_delta.alloc(6 * plan.chunk_units));
        // Without CRN Delta/Gamma the base sweeps' forward passes are the
        // plan's paths: they give the price and no separate price pass runs.
        plan.price_from_adjoint = !P.lv_bumps && P.precision == MCG_PRECISION_F64;
        if (plan.price_from_adjoint) {
            MCG_CUDA(plan.adj_price.alloc(2 * plan.chunk_units));
            if (plan.mask & (0xffu << 10)) MCG_CUDA(plan.adj_diag.alloc(2 * 8 * plan.chunk_units));
        }
        MCG_CUDA(plan.adj_partials.alloc(static_cast<size_t>(P.scramble_count) * plan.tiles * 3));
        MCG_CUDA(plan.adj_records.alloc(static_cast<size_t>(P.scramble_count) * 3));
        if (plan.adjoint_nodes) {
            MCG_CUDA(plan.node_tiles.alloc(static_cast<size_t>(P.scramble_count) * plan.tiles * plan.grid_values));
            MCG_CUDA(plan.node_records.alloc(static_cast<size_t>(P.scramble_count) * plan.grid_values));
        }
        if (lv_adjoint_smem(P) > 200 * 1024)
            return fail(MCG_ERR_UNSUPPORTED, "local-variance grid too large for the adjoint kernel's shared memory");
    }
    return MCG_OK;
}

// Statistics over ordered values, two passes
// (CenteredMoment::from_ordered_values_two_pass, reduction.rs:99-122).
struct HostStat {
    double sum = 0.0, corr = 0.0;
    uint64_t count = 0;
    double mean = 0.0, m2 = 0.0;
    double total() const { return sum + corr; }
};

void neumaier(double& s, double& c, double v) {
    const double u = s + v;
    if (std::fabs(s) >= std::fabs(v)) c += (s - u) + v;
    else c += (v - u) + s;
    s = u;
}

HostStat two_pass(const std::vector<double>& values) {
    HostStat h;
    if (values.empty()) return h;
    double s = 0.0, c = 0.0;
    for (double v : values) neumaier(s, c, v);
    h.sum = s;
    h.corr = c;
    const double mean = (s + c) / static_cast<double>(values.size());
    double qs = 0.0, qc = 0.0;
    for (double v : values) {
        const double dv = v - mean;
        neumaier(qs, qc, dv * dv);
    }
    h.count = values.size();
    h.mean = mean;
    h.m2 = qs + qc;
    return h;
}

// Statistics of grid node k from the per-scramble node records: pseudo-MC
// from the 128-path tile sums (batch means), RQMC from the scramble means.
HostStat node_statistics(const std::vector<StatRecord>& node_rec, uint32_t nv, uint32_t k, uint64_t units,
                         uint32_t scrambles, bool rqmc) {
    HostStat h;
    if (!rqmc) {
        const StatRecord& x = node_rec[k];
        const double total = x.sum + x.corr;
        const double n = static_cast<double>(units);
        const double tiles = x.count;
        const double batch = n / tiles;
        const double s2 = tiles > 1.0 ? x.m2 / (tiles - 1.0) / (batch * batch) : 0.0;
        h.sum = x.sum;
        h.corr = x.corr;
        h.count = units;
        h.mean = total / n;
        h.m2 = (s2 / tiles) * n * (n - 1.0);
    } else {
        std::vector<double> reps(scrambles);
        for (uint32_t sc = 0; sc < scrambles; ++sc)
            reps[sc] = (node_rec[static_cast<size_t>(sc) * nv + k].sum + node_rec[static_cast<size_t>(sc) * nv + k].corr) /
                       static_cast<double>(units);
        h = two_pass(reps);
    }
    return h;
}

mcg_estimate make_estimate(const HostStat& s, uint64_t units, double scale) {
    const double inv = 1.0 / static_cast<double>(units);
    const double value = s.total() * inv * scale;
    const double var = s.count > 1 ? s.m2 / static_cast<double>(s.count - 1) : 0.0;
    const double se = std::sqrt(var * inv) * std::fabs(scale);
    const double hw = 1.959963984540054 * se;
    return {value, se, value - hw, value + hw, units};
}

mcg_status evaluate(mcg_plan* plan, cudaStream_t stream, mcg_result* result) {
    if (!plan || !result) return fail(MCG_ERR_INVALID_ARGUMENT, "null plan or result");
    if (result->product_capacity < plan->product_count || !result->products)
        return fail(MCG_ERR_INVALID_ARGUMENT, "result has too few product slots");
    std::memset(&result->error, 0, sizeof(result->error));
    DevicePlan& P = plan->dp;
    const uint32_t slots = plan->slots;
    ErrorWord init{~0ull, 0, 0, 0, 0};
    MCG_CUDA(cudaMemcpyAsync(plan->error.ptr, &init, sizeof(init), cudaMemcpyHostToDevice, stream));
    cudaEvent_t t0, t1, tp;
    MCG_CUDA(cudaEventCreate(&t0));
    MCG_CUDA(cudaEventCreate(&t1));
    MCG_CUDA(cudaEventCreate(&tp));
    MCG_CUDA(cudaEventRecord(t0, stream));
    // Kernels write records in compact (slot) order: remap through the mask.
    uint32_t launches = 0;
    cudaError_t e;
    // Per-product partials use kComponents stride; reduce only masked slots below.
    if (P.model == MCG_MODEL_LOCAL_VOLATILITY && P.precision == MCG_PRECISION_F32_BULK) {
        e = launch_lv32_path(P, plan->partials.ptr, plan->mask, plan->error.ptr, stream);
    } else if (P.model == MCG_MODEL_LOCAL_VOLATILITY && plan->price_from_adjoint) {
        e = cudaSuccess;  // the price comes from the adjoint sweeps below
    } else if (P.model == MCG_MODEL_LOCAL_VOLATILITY) {
        int evolutions;
        e = launch_lv_path(P, 0, P.units, P.scramble_count, plan->partials.ptr, plan->mask, plan->error.ptr, 0,
                           stream, evolutions);
    } else {
        e = launch_bs_path(P, plan->single_terminal, 0, P.units, P.scramble_count, plan->partials.ptr,
                           plan->mask, plan->error.ptr, 0, stream);
    }
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("path kernel: ") + cudaGetErrorString(e));
    const uint32_t width = plan->product_count * kComponents;
    if (P.bs_tape) {
        // the path-risk kernel runs in scratch-sized chunks of units
        const uint64_t per_launch = P.bs_tape_units / P.scramble_count / kThreads * kThreads;
        launches += static_cast<uint32_t>((P.units + per_launch - 1) / per_launch) - 1;
    }
    if (!plan->price_from_adjoint) {
        ++launches;
        MCG_CUDA(cudaEventRecord(tp, stream));
        reduce_tiles_kernel<<<dim3(width, P.scramble_count), 256, 0, stream>>>(plan->partials.ptr, plan->tiles,
                                                                               width, plan->records.ptr);
        MCG_CUDA(cudaGetLastError());
        ++launches;
    }
    std::vector<StatRecord> adj_rec, node_rec;
    if (plan->adjoint) {
        const int pairs = P.antithetic ? 2 : 1;
        const uint32_t tiles_chunk = static_cast<uint32_t>((plan->chunk_units + kThreads - 1) / kThreads);
        for (uint32_t sc = 0; sc < P.scramble_count; ++sc) {
            for (uint64_t begin = 0; begin < P.units; begin += plan->chunk_units) {
                const uint64_t n = std::min<uint64_t>(plan->chunk_units, P.units - begin);
                const uint32_t tile_offset = sc * plan->tiles + static_cast<uint32_t>(begin / kThreads);
                for (int pr = 0; pr < pairs; ++pr) {
                    for (int which : {1, 2, 0}) {
                        if (which != 0 && !plan->adjoint_gamma) continue;
                        AdjointArgs A{};
                        A.which = which;
                        A.sign = pr == 0 ? 1.0 : -1.0;
                        A.node_weight = pairs == 2 ? 0.5 : 1.0;
                        A.node_add = pr;
                        A.scramble = sc;
                        A.unit_begin = begin;
                        A.units = n;
                        A.tile_offset = tile_offset;
                        A.tape_f = plan->tape.ptr;
                        A.tape_z = plan->tape.ptr + static_cast<size_t>(P.steps + 1) * plan->chunk_units;
                        A.out_vega = plan->adj_vega.ptr + static_cast<size_t>(pr * 3 + which) * n;
                        A.out_delta = plan->adj_delta.ptr + static_cast<size_t>(pr * 3 + which) * n;
                        A.node_tiles = (which == 0 && plan->adjoint_nodes) ? plan->node_tiles.ptr : nullptr;
                        if (which == 0 && plan->price_from_adjoint) {
                            A.out_price = plan->adj_price.ptr + static_cast<size_t>(pr) * n;
                            A.out_diag = plan->adj_diag.ptr ? plan->adj_diag.ptr + static_cast<size_t>(pr) * 8 * n
                                                            : nullptr;
                        }
                        e = launch_lv_adjoint(P, A, plan->error.ptr, stream);
                        if (e != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("adjoint kernel: ") + cudaGetErrorString(e));
                        ++launches;
                    }
                }
                e = launch_lv_adjoint_combine(plan->adj_vega.ptr, plan->adj_delta.ptr, n, pairs,
                                              plan->adjoint_gamma ? 1 : 0, P.spot_bump, tile_offset,
                                              plan->adj_partials.ptr, stream);
                if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
                ++launches;
                if (plan->price_from_adjoint) {
                    e = launch_lv_adjoint_price(plan->adj_price.ptr, plan->adj_diag.ptr, n, pairs, tile_offset,
                                                plan->mask, plan->partials.ptr, stream);
                    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
                    ++launches;
                }
                (void)tiles_chunk;
            }
        }
        reduce_tiles_kernel<<<dim3(3, P.scramble_count), 256, 0, stream>>>(plan->adj_partials.ptr, plan->tiles, 3,
                                                                          plan->adj_records.ptr);
        MCG_CUDA(cudaGetLastError());
        ++launches;
        if (plan->price_from_adjoint) {
            MCG_CUDA(cudaEventRecord(tp, stream));
            reduce_tiles_kernel<<<dim3(width, P.scramble_count), 256, 0, stream>>>(plan->partials.ptr, plan->tiles,
                                                                                   width, plan->records.ptr);
            MCG_CUDA(cudaGetLastError());
            ++launches;
        }
        adj_rec.resize(static_cast<size_t>(P.scramble_count) * 3);
        if (plan->adjoint_nodes) {
            e = launch_lv_node_reduce(plan->node_tiles.ptr, plan->tiles, P.scramble_count, plan->grid_values,
                                      plan->node_records.ptr, stream);
            if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
            ++launches;
            node_rec.resize(static_cast<size_t>(P.scramble_count) * plan->grid_values);
        }
    }
    MCG_CUDA(cudaEventRecord(t1, stream));
    if (!adj_rec.empty())
        MCG_CUDA(cudaMemcpyAsync(adj_rec.data(), plan->adj_records.ptr, adj_rec.size() * sizeof(StatRecord),
                                 cudaMemcpyDeviceToHost, stream));
    if (!node_rec.empty())
        MCG_CUDA(cudaMemcpyAsync(node_rec.data(), plan->node_records.ptr, node_rec.size() * sizeof(StatRecord),
                                 cudaMemcpyDeviceToHost, stream));
    std::vector<StatRecord> rec(static_cast<size_t>(P.scramble_count) * width);
    ErrorWord ew;
    MCG_CUDA(cudaMemcpyAsync(rec.data(), plan->records.ptr, rec.size() * sizeof(StatRecord),
                             cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaMemcpyAsync(&ew, plan->error.ptr, sizeof(ew), cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.0f, path_ms = 0.0f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventElapsedTime(&path_ms, t0, tp);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaEventDestroy(tp);
    result->device_ms = ms;
    result->path_kernel_ms = path_ms;
    result->kernel_launches = launches;
    if (ew.key != ~0ull && P.precision == MCG_PRECISION_F32_BULK) {
        result->error.code = static_cast<int32_t>(ew.key & 0xff);
        result->error.sampling_unit = ew.key >> 8;
        return fail(static_cast<mcg_status>(result->error.code),
                    "sampling unit " + std::to_string(result->error.sampling_unit) + " failed (FP32 path bulk)");
    }
    if (ew.key != ~0ull) {
        // Re-run the first failing unit alone to recover step and value bits.
        const uint64_t unit = ew.key >> 8;
        const uint32_t scrambles_for_detail = 1;
        (void)scrambles_for_detail;
        MCG_CUDA(cudaMemcpyAsync(plan->error.ptr, &init, sizeof(init), cudaMemcpyHostToDevice, stream));
        if (P.model == MCG_MODEL_LOCAL_VOLATILITY) {
            int ev;
            e = launch_lv_path(P, unit, 1, P.scramble_count, plan->partials.ptr, plan->mask, plan->error.ptr, 1,
                               stream, ev);
        } else {
            e = launch_bs_path(P, plan->single_terminal, unit, 1, P.scramble_count, plan->partials.ptr,
                               plan->mask, plan->error.ptr, 1, stream);
        }
        MCG_CUDA(cudaMemcpyAsync(&ew, plan->error.ptr, sizeof(ew), cudaMemcpyDeviceToHost, stream));
        MCG_CUDA(cudaStreamSynchronize(stream));
        result->error.code = static_cast<int32_t>(ew.key & 0xff);
        result->error.sampling_unit = ew.key >> 8;
        result->error.step = ew.step;
        result->error.value_bits = ew.value_bits;
        return fail(static_cast<mcg_status>(result->error.code),
                    "sampling unit " + std::to_string(result->error.sampling_unit) + " failed");
    }
    const bool rqmc = P.engine == MCG_ENGINE_RQMC;
    const uint64_t independent = rqmc ? P.scramble_count : P.units;
    result->independent_sampling_units = independent;
    result->evaluated_paths = P.units * (rqmc ? P.scramble_count : 1) * (P.antithetic ? 2 : 1);
    result->time_steps = P.steps;
    result->effective_dimension = P.dimension;
    result->reduction_records = plan->tiles * P.scramble_count;
    const bool want_replicates = rqmc && result->replicate_means &&
                                 result->replicate_capacity >=
                                     static_cast<uint64_t>(P.scramble_count) * plan->product_count * kComponents;
    for (uint32_t k = 0; k < plan->product_count; ++k) {
        mcg_product_result& r = result->products[k];
        HostStat stats[kComponents];
        for (int c = 0; c < kComponents; ++c) {
            const bool active = plan->mask & (1u << c);
            HostStat h;
            if (!rqmc) {
                if (active) {
                    const StatRecord& s = rec[static_cast<size_t>(k) * kComponents + c];
                    h = {s.sum, s.corr, static_cast<uint64_t>(s.count), s.mean, s.m2};
                } else {
                    h.count = P.units;
                }
            } else {
                std::vector<double> reps(P.scramble_count, 0.0);
                if (active)
                    for (uint32_t s = 0; s < P.scramble_count; ++s) {
                        const StatRecord& x = rec[(static_cast<size_t>(s) * plan->product_count + k) * kComponents + c];
                        reps[s] = (x.sum + x.corr) / static_cast<double>(P.units);
                    }
                h = two_pass(reps);
                if (want_replicates)
                    for (uint32_t s = 0; s < P.scramble_count; ++s)
                        result->replicate_means[(static_cast<size_t>(s) * plan->product_count + k) * kComponents + c] =
                            reps[s];
            }
            stats[c] = h;
            r.components[c] = {h.sum, h.corr, h.count, h.mean, h.m2};
        }
        if (plan->adjoint) {
            // Vega and the adjoint Delta/Gamma come from the reverse sweep.
            HostStat adj[3];
            for (int c = 0; c < 3; ++c) {
                if (!rqmc) {
                    const StatRecord& x = adj_rec[c];
                    adj[c] = {x.sum, x.corr, static_cast<uint64_t>(x.count), x.mean, x.m2};
                } else {
                    std::vector<double> reps(P.scramble_count);
                    for (uint32_t sc = 0; sc < P.scramble_count; ++sc)
                        reps[sc] = (adj_rec[sc * 3 + c].sum + adj_rec[sc * 3 + c].corr) / static_cast<double>(P.units);
                    adj[c] = two_pass(reps);
                }
            }
            stats[MCG_VEGA] = adj[0];
            r.components[MCG_VEGA] = {adj[0].sum, adj[0].corr, adj[0].count, adj[0].mean, adj[0].m2};
            for (int c = 0; c < 2; ++c)
                r.adjoint_components[c] = {adj[c + 1].sum, adj[c + 1].corr, adj[c + 1].count, adj[c + 1].mean,
                                           adj[c + 1].m2};
            r.adjoint_delta = make_estimate(adj[1], independent, 1.0);
            r.adjoint_gamma = make_estimate(adj[2], independent, 1.0);
        }
        r.price = make_estimate(stats[MCG_PRICE], independent, 1.0);
        r.delta = make_estimate(stats[MCG_DELTA], independent, 1.0);
        r.gamma = make_estimate(stats[MCG_GAMMA], independent, 1.0);
        r.vega = make_estimate(stats[MCG_VEGA], independent, 1.0);
        r.bump_delta = make_estimate(stats[MCG_BUMP_DELTA], independent, 1.0);
        r.bump_gamma = make_estimate(stats[MCG_BUMP_GAMMA], independent, 1.0);
        r.bump_vega = make_estimate(stats[MCG_BUMP_VEGA], independent, 1.0);
        const HostStat& pr = stats[MCG_PRICE];
        const double sv = pr.count > 1 ? pr.m2 / static_cast<double>(pr.count - 1) : 0.0;
        r.sampling_variance = plan->total_variance == 0.0 ? 0.0 : sv;
        r.estimator_variance = r.sampling_variance / static_cast<double>(independent);
    }
    if (!node_rec.empty() && result->local_vega_nodes && result->node_capacity >= plan->grid_values) {
        // Node sensitivities: exact means; pseudo-MC standard errors from the
        // batch means of the 128-unit CTA tiles, RQMC from the scramble means.
        const uint32_t nv = plan->grid_values;
        for (uint32_t k = 0; k < nv; ++k) {
            const HostStat h = node_statistics(node_rec, nv, k, P.units, P.scramble_count, rqmc);
            result->local_vega_nodes[k] = {h.sum, h.corr, h.count, h.mean, h.m2};
            if (result->local_vega_node_estimates)
                result->local_vega_node_estimates[k] = make_estimate(h, independent, 1.0);
        }
    }
    if (plan->total_variance > 0.0 && independent < 2)
        return fail(MCG_ERR_INSUFFICIENT_UNITS, "at least two independent sampling units are required");
    return MCG_OK;
}

// ------------------------------------------------------------ early exercise

// Device buffers of one mcg_lsm_price call, released on every return path.
struct LsmBuffers {
    DeviceArray<double> spots, cf, df, unit_values, means, centers, cf_mlp, centers_mlp;
    DeviceArray<float> mlp_params, mlp_moments, mlp_partials, mlp_loss, mlp_snapshots;
    DeviceArray<uint32_t> stop_mlp;
    cudaEvent_t mlp_ev[2] = {nullptr, nullptr};
    DeviceArray<uint32_t> stop, vstops;
    DeviceArray<mcg_lsm_date_model> models;
    DeviceArray<DD> partials, group_partials, sums;
    DeviceArray<unsigned int> tickets;
    DeviceArray<unsigned long long> counts, words;
    DeviceArray<StatRecord> risk_partials, risk_records;
    DeviceArray<double> risk_price;  // local volatility: exercise-value prices [pair][runtime][unit]
    DeviceArray<double> vspots;      // local volatility: valuation path store (when the training one is too small)
    DeviceArray<ErrorWord> path_errors;  // local volatility: [0] training, [1] valuation
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    ~LsmBuffers() {
        vspots.release();
        path_errors.release();
        risk_partials.release();
        risk_records.release();
        risk_price.release();
        spots.release();
        cf.release();
        df.release();
        unit_values.release();
        means.release();
        centers.release();
        cf_mlp.release();
        centers_mlp.release();
        mlp_params.release();
        mlp_moments.release();
        mlp_partials.release();
        mlp_loss.release();
        mlp_snapshots.release();
        stop_mlp.release();
        for (cudaEvent_t& e : mlp_ev)
            if (e) cudaEventDestroy(e);
        stop.release();
        vstops.release();
        models.release();
        partials.release();
        group_partials.release();
        sums.release();
        tickets.release();
        counts.release();
        words.release();
        for (cudaEvent_t& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

mcg_status validate_lsm(const mcg_plan_desc* d, const mcg_lsm_desc* l, const mcg_lsm_result* r) {
    if (!d || !l || !r) return fail(MCG_ERR_INVALID_ARGUMENT, "null argument");
    if (d->abi_version != MCG_ABI_VERSION) return fail(MCG_ERR_INVALID_ARGUMENT, "abi_version mismatch");
    if (d->product_count != 1 || !d->products || d->products[0].kind != MCG_PRODUCT_AMERICAN)
        return fail(MCG_ERR_INVALID_ARGUMENT, "an early-exercise plan holds exactly one American product");
    if (d->model != MCG_MODEL_BLACK_SCHOLES && d->model != MCG_MODEL_LOCAL_VOLATILITY)
        return fail(MCG_ERR_INVALID_ARGUMENT, "model");
    if (d->request_local_vega_nodes && d->model != MCG_MODEL_LOCAL_VOLATILITY)
        return fail(MCG_ERR_UNSUPPORTED, "local vega nodes need a local-volatility plan");
    if (d->model == MCG_MODEL_LOCAL_VOLATILITY && d->precision != MCG_PRECISION_F64 &&
        (d->request_delta || d->request_gamma || d->request_vega || d->request_local_vega_nodes))
        return fail(MCG_ERR_UNSUPPORTED, "early-exercise risk runs in FP64");
    if (d->request_gamma) {
        const double b = resolve_gamma_bump(d);
        if (!std::isfinite(b) || b <= 0.0 || b >= d->spot)
            return fail(MCG_ERR_INVALID_ARGUMENT, "gamma bump must lie in (0, spot)");
    }
    if (l->continuation != MCG_CONTINUATION_POLYNOMIAL && l->continuation != MCG_CONTINUATION_MLP)
        return fail(MCG_ERR_UNSUPPORTED, "continuation kind");
    if (l->continuation == MCG_CONTINUATION_MLP &&
        (!std::isfinite(l->mlp_learning_rate) || l->mlp_learning_rate < 0.0f || l->mlp_epochs > 1000u))
        return fail(MCG_ERR_INVALID_ARGUMENT, "mlp_learning_rate / mlp_epochs");
    if (l->max_degree < 1 || l->max_degree > MCG_LSM_MAX_DEGREE)
        return fail(MCG_ERR_INVALID_ARGUMENT, "max_degree must be 1..7");
    // validate_tolerance, lsm.rs:2295-2302
    for (double t : {l->itm_abs_tolerance, l->cpqr_abs_tolerance, l->cpqr_rel_tolerance})
        if (!std::isfinite(t) || t < 0.0) return fail(MCG_ERR_LSM, "tolerances must be finite and non-negative");
    if (l->max_matrix_elements == 0) return fail(MCG_ERR_LSM, "max_matrix_elements must be positive");
    if (l->training_units == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "training_units");
    if (d->engine == MCG_ENGINE_RQMC && l->training_scramble_count == 0)
        return fail(MCG_ERR_INVALID_ARGUMENT, "training_scramble_count");
    const uint32_t dates = d->observation_count;
    if (dates == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "observation_times");
    if (r->date_capacity < dates || !r->exercise_counts || (dates > 1 && !r->models))
        return fail(MCG_ERR_INVALID_ARGUMENT, "result needs date_capacity >= exercise dates");
    return MCG_OK;
}

mcg_status lsm_price(const mcg_plan_desc* d, const mcg_lsm_desc* l, cudaStream_t stream, mcg_lsm_result* r) {
    mcg_status st = validate_lsm(d, l, r);
    if (st != MCG_OK) return st;
    std::memset(&r->error, 0, sizeof(r->error));
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
        return fail(MCG_ERR_CUDA, "no CUDA device is visible");
    if (d->discrete_dividends.count)
        return fail(MCG_ERR_UNSUPPORTED, "early exercise with discrete dividends");
    // The path plans of both engines: the American product prices nothing by
    // itself, so each plan carries a European placeholder of the same contract.
    mcg_product_desc placeholder = d->products[0];
    placeholder.kind = MCG_PRODUCT_EUROPEAN;
    mcg_plan_desc vd = *d;
    vd.products = &placeholder;
    vd.payment_time = d->observation_times[d->observation_count - 1];
    // Risk is taken by the fixed-policy pass below, not by the path plans.
    const bool risk = d->request_delta || d->request_gamma || d->request_vega || d->request_local_vega_nodes;
    vd.request_delta = vd.request_gamma = vd.request_vega = vd.request_local_vega_nodes = 0;
    mcg_plan_desc td = vd;
    td.master_seed = l->training_seed;
    td.sampling_units = l->training_units;
    td.scramble_count = l->training_scramble_count;
    td.scramble_begin = 0;
    td.antithetic = l->training_antithetic;
    td.brownian_bridge = l->training_brownian_bridge;
    mcg_plan vplan, tplan;
    if ((st = build(&vd, vplan)) != MCG_OK) return st;
    if ((st = build(&td, tplan)) != MCG_OK) return st;
    const DevicePlan& TP = tplan.dp;
    const DevicePlan& VP = vplan.dp;
    const uint32_t dates = d->observation_count;
    const bool rqmc = d->engine == MCG_ENGINE_RQMC;
    const uint64_t t_units = TP.units * TP.scramble_count, v_units = VP.units * VP.scramble_count;
    const uint64_t t_paths = t_units * (TP.antithetic ? 2 : 1), v_paths = v_units * (VP.antithetic ? 2 : 1);
    HostCurve rc;
    std::string why;
    if (!load_curve(d->discount_curve, rc, "discount_curve", why)) return fail(MCG_ERR_MARKET, why);
    std::vector<double> df(dates);
    for (uint32_t i = 0; i < dates; ++i) {
        df[i] = std::exp(rc.log_discount(d->observation_times[i]));
        if (!std::isfinite(df[i]) || df[i] <= 0.0) return fail(MCG_ERR_LSM, "invalid discount factor");
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const unsigned ctas = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>((t_paths + 255) / 256, 2ull * static_cast<uint64_t>(sms))));
    const unsigned group_ctas = static_cast<unsigned>(std::max(1, sms));
    const uint32_t t_groups = rqmc ? TP.scramble_count : 1, v_groups = rqmc ? VP.scramble_count : 1;

    LsmBuffers B;
    MCG_CUDA(B.spots.alloc(static_cast<size_t>(dates) * t_paths));
    MCG_CUDA(B.cf.alloc(t_paths));
    MCG_CUDA(B.stop.alloc(t_paths));
    MCG_CUDA(B.df.upload(df));
    MCG_CUDA(B.centers.upload(std::vector<double>(dates, d->products[0].strike)));
    MCG_CUDA(B.models.alloc(std::max<uint32_t>(dates - 1, 1)));
    MCG_CUDA(B.partials.alloc(static_cast<size_t>(ctas) * lsm_partial_stride()));
    MCG_CUDA(B.tickets.alloc(3));
    MCG_CUDA(B.words.alloc(2));  // [0] first non-finite training unit, [1] first failing date
    MCG_CUDA(B.unit_values.alloc(v_units));
    MCG_CUDA(B.counts.alloc(dates));
    const bool want_stops = r->stopping_indices && r->stopping_capacity >= v_paths;
    if (want_stops || risk) MCG_CUDA(B.vstops.alloc(v_paths));
    const uint32_t max_groups = std::max(t_groups, v_groups);
    MCG_CUDA(B.group_partials.alloc(static_cast<size_t>(max_groups) * group_ctas));
    MCG_CUDA(B.sums.alloc(4 * static_cast<size_t>(max_groups)));  // in-sample, valuation, squares, network in-sample
    MCG_CUDA(B.means.alloc(static_cast<size_t>(max_groups)));
    MCG_CUDA(cudaMemsetAsync(B.tickets.ptr, 0, 3 * sizeof(unsigned int), stream));
    MCG_CUDA(cudaMemsetAsync(B.words.ptr, 0xff, 2 * sizeof(unsigned long long), stream));
    MCG_CUDA(cudaMemsetAsync(B.counts.ptr, 0, dates * sizeof(unsigned long long), stream));
    MCG_CUDA(cudaMemsetAsync(B.models.ptr, 0, std::max<uint32_t>(dates - 1, 1) * sizeof(mcg_lsm_date_model), stream));
    for (cudaEvent_t& e : B.ev) MCG_CUDA(cudaEventCreate(&e));
    uint32_t launches = 0;

    // Training: path matrix, then the backward induction.
    MCG_CUDA(cudaEventRecord(B.ev[0], stream));
    const bool lv = d->model == MCG_MODEL_LOCAL_VOLATILITY;
    if (lv) {
        const ErrorWord init[2] = {{~0ull, 0, 0, 0, 0}, {~0ull, 0, 0, 0, 0}};
        MCG_CUDA(B.path_errors.alloc(2));
        MCG_CUDA(cudaMemcpyAsync(B.path_errors.ptr, init, sizeof(init), cudaMemcpyHostToDevice, stream));
        MCG_CUDA(launch_lsm_lv_spots(TP, /*LsmTrain*/ 1u, B.spots.ptr, t_paths, &B.path_errors.ptr[0], stream));
    } else {
        MCG_CUDA(launch_lsm_bs_spots(TP, /*LsmTrain*/ 1u, B.spots.ptr, t_paths, &B.words.ptr[0], stream));
    }
    ++launches;
    MCG_CUDA(cudaEventRecord(B.ev[1], stream));
    LsmArgs A{};
    A.spots = B.spots.ptr;
    A.paths = t_paths;
    A.dates = dates;
    A.nb = l->max_degree + 1;
    A.side = d->products[0].side;
    A.strike = d->products[0].strike;
    A.notional = d->products[0].notional;
    A.itm_tol = l->itm_abs_tolerance;
    A.abs_tol = l->cpqr_abs_tolerance;
    A.rel_tol = l->cpqr_rel_tolerance;
    A.max_elements = l->max_matrix_elements;
    A.df = B.df.ptr;
    A.cf = B.cf.ptr;
    A.stop = B.stop.ptr;
    A.models = B.models.ptr;
    A.centers = B.centers.ptr;
    A.partials = B.partials.ptr;
    A.tickets = B.tickets.ptr;
    A.lsm_error = &B.words.ptr[1];
    const int last = static_cast<int>(dates) - 1;
    MCG_CUDA(launch_lsm_init(A, ctas, stream));
    ++launches;
    if (last >= 1) {
        MCG_CUDA(launch_lsm_step(A, ctas, -1, last - 1, stream));
        ++launches;
    }
    for (int date = last - 1; date >= 0; --date) {
        MCG_CUDA(launch_lsm_step(A, ctas, date, date - 1, stream));
        ++launches;
    }
    // In-sample value of the training paths under their own policy.
    DD* s_in = B.sums.ptr;
    DD* s_val = B.sums.ptr + max_groups;
    DD* s_sq = B.sums.ptr + 2 * max_groups;
    MCG_CUDA(launch_lsm_group_sum(B.cf.ptr, TP.units, t_groups, TP.antithetic, nullptr, B.group_partials.ptr,
                                  group_ctas, s_in, nullptr, stream));
    launches += 2;
    MCG_CUDA(cudaEventRecord(B.ev[2], stream));

    // In-sample value from the group sums: mean of the collapsed training values
    // (pseudo) or of the per-scramble replicates (RQMC), risk/early_exercise.rs:100-110,300-313.
    auto in_sample_of = [&](const std::vector<DD>& sums, size_t base) {
        if (rqmc) {
            double s = 0.0, c = 0.0;
            for (uint32_t g = 0; g < t_groups; ++g)
                neumaier(s, c, (sums[base + g].hi + sums[base + g].lo) / static_cast<double>(TP.units));
            return (s + c) / static_cast<double>(t_groups);
        }
        return (sums[base].hi + sums[base].lo) / static_cast<double>(TP.units);
    };

    // Learned continuation: the network's own backward induction on the same
    // training paths, then the choice between the two policies.
    bool use_mlp = false;
    r->continuation_used = MCG_CONTINUATION_POLYNOMIAL;
    r->mlp_steps = 0;
    r->mlp_ms = 0.f;
    r->mlp_final_loss = 0.f;
    r->polynomial_in_sample = 0.0;
    r->mlp_in_sample = 0.0;
    if (l->continuation == MCG_CONTINUATION_MLP && dates > 1) {
        const uint64_t batch = l->mlp_batch ? l->mlp_batch : 16384u;
        const uint32_t epochs = l->mlp_epochs ? l->mlp_epochs : 1u;
        const float lr = l->mlp_learning_rate > 0.0f ? l->mlp_learning_rate : 2e-3f;
        // Glorot-uniform initial weights from a splitmix64 stream, zero biases.
        std::vector<float> params(kMlpParams, 0.0f);
        uint64_t state = l->mlp_seed;
        auto uniform = [&]() {
            uint64_t z = (state += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            return static_cast<double>(z >> 11) * 0x1.0p-53 * 2.0 - 1.0;
        };
        const double a1 = std::sqrt(6.0 / (2 + kMlpHidden)), a2 = std::sqrt(6.0 / (2 * kMlpHidden)),
                     a3 = std::sqrt(6.0 / (kMlpHidden + 1));
        for (int i = 0; i < 2 * kMlpHidden; ++i) params[kMlpW1 + i] = static_cast<float>(a1 * uniform());
        for (int i = 0; i < kMlpHidden * kMlpHidden; ++i) params[kMlpW2 + i] = static_cast<float>(a2 * uniform());
        for (int i = 0; i < kMlpHidden; ++i) params[kMlpW3 + i] = static_cast<float>(a3 * uniform());
        MCG_CUDA(B.mlp_params.upload(params));
        MCG_CUDA(B.mlp_moments.alloc(2 * static_cast<size_t>(kMlpParams)));
        MCG_CUDA(cudaMemsetAsync(B.mlp_moments.ptr, 0, 2 * kMlpParams * sizeof(float), stream));
        MCG_CUDA(B.mlp_partials.alloc(static_cast<size_t>(std::max(sms, 1)) * kMlpPartial));
        MCG_CUDA(B.mlp_loss.alloc(1));
        // the weights each date was decided with, for the valuation
        MCG_CUDA(B.mlp_snapshots.alloc(static_cast<size_t>(dates - 1) * kMlpParams));
        MCG_CUDA(B.cf_mlp.alloc(t_paths));
        MCG_CUDA(B.stop_mlp.alloc(t_paths));
        MCG_CUDA(B.centers_mlp.upload(std::vector<double>(dates, d->products[0].strike)));
        for (cudaEvent_t& e : B.mlp_ev) MCG_CUDA(cudaEventCreate(&e));
        LsmArgs AM = A;
        AM.cf = B.cf_mlp.ptr;
        AM.stop = B.stop_mlp.ptr;
        AM.centers = B.centers_mlp.ptr;
        MCG_CUDA(cudaEventRecord(B.mlp_ev[0], stream));
        MCG_CUDA(launch_lsm_init(AM, ctas, stream));
        ++launches;
        const double horizon = d->observation_times[last];
        const uint64_t nbatch = (t_paths + batch - 1) / batch;
        uint32_t step = 0;
        for (int date = last - 1; date >= 0; --date) {
            const double tin = 2.0 * d->observation_times[date] / horizon - 1.0;
            // Default schedule: at least 400 Adam steps at the first (from-scratch)
            // date and 50 at the warm-started ones; an explicit epoch count gives
            // exactly epochs x batches (4x at the first date).
            const uint64_t first = date == last - 1 ? 4u : 1u;
            const uint64_t steps = l->mlp_epochs
                                       ? first * static_cast<uint64_t>(epochs) * nbatch
                                       : std::max<uint64_t>(nbatch, date == last - 1 ? 400u : 50u);
            // the date's Adam steps in one cooperative launch (gradient pass,
            // grid barrier, update, grid barrier per step)
            MlpRows rows{};
            rows.spots = B.spots.ptr + static_cast<size_t>(date) * t_paths;
            rows.cf = B.cf_mlp.ptr;
            rows.df = df[date];
            rows.time_input = tin;
            rows.side = A.side;
            rows.strike = A.strike;
            rows.notional = A.notional;
            rows.itm_tol = A.itm_tol;
            MCG_CUDA(launch_mlp_train(B.mlp_params.ptr, B.mlp_moments.ptr, B.mlp_partials.ptr, rows, t_paths, batch,
                                      static_cast<uint32_t>(steps), step, lr, B.mlp_loss.ptr, stream));
            step += static_cast<uint32_t>(steps);
            ++launches;
            MCG_CUDA(cudaMemcpyAsync(B.mlp_snapshots.ptr + static_cast<size_t>(date) * kMlpParams, B.mlp_params.ptr,
                                     kMlpParams * sizeof(float), cudaMemcpyDeviceToDevice, stream));
            MlpDecision dec{};
            dec.spots = B.spots.ptr + static_cast<size_t>(date) * t_paths;
            dec.cf = B.cf_mlp.ptr;
            dec.stop = B.stop_mlp.ptr;
            dec.paths = t_paths;
            dec.date = static_cast<uint32_t>(date);
            dec.df = df[date];
            dec.time_input = tin;
            dec.side = A.side;
            dec.strike = A.strike;
            dec.notional = A.notional;
            dec.itm_tol = A.itm_tol;
            MCG_CUDA(launch_mlp_decide(B.mlp_params.ptr, dec, stream));
            ++launches;
        }
        MCG_CUDA(cudaEventRecord(B.mlp_ev[1], stream));
        DD* s_in_mlp = B.sums.ptr + 3 * max_groups;
        MCG_CUDA(launch_lsm_group_sum(B.cf_mlp.ptr, TP.units, t_groups, TP.antithetic, nullptr,
                                      B.group_partials.ptr, group_ctas, s_in_mlp, nullptr, stream));
        launches += 2;
        std::vector<DD> early(4 * static_cast<size_t>(max_groups));
        float loss = 0.f;
        MCG_CUDA(cudaMemcpyAsync(early.data(), B.sums.ptr, early.size() * sizeof(DD), cudaMemcpyDeviceToHost,
                                 stream));
        MCG_CUDA(cudaMemcpyAsync(params.data(), B.mlp_params.ptr, kMlpParams * sizeof(float),
                                 cudaMemcpyDeviceToHost, stream));
        MCG_CUDA(cudaMemcpyAsync(&loss, B.mlp_loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, stream));
        MCG_CUDA(cudaStreamSynchronize(stream));
        bool finite = std::isfinite(loss);
        for (float v : params) finite &= std::isfinite(v);
        r->polynomial_in_sample = in_sample_of(early, 0);
        r->mlp_in_sample = in_sample_of(early, 3 * static_cast<size_t>(max_groups));
        r->mlp_steps = step;
        r->mlp_final_loss = loss;
        cudaEventElapsedTime(&r->mlp_ms, B.mlp_ev[0], B.mlp_ev[1]);
        use_mlp = finite && r->mlp_in_sample >= r->polynomial_in_sample;
        if (use_mlp) r->continuation_used = MCG_CONTINUATION_MLP;
        if (r->mlp_params && r->mlp_param_capacity >= static_cast<uint32_t>(kMlpParams))
            std::memcpy(r->mlp_params, params.data(), kMlpParams * sizeof(float));
    }

    // Valuation: fresh paths under the fitted policy.
    LsmValueArgs V{};
    V.df = B.df.ptr;
    V.models = B.models.ptr;
    V.dates = dates;
    V.nb = A.nb;
    V.side = A.side;
    V.strike = A.strike;
    V.notional = A.notional;
    V.unit_values = B.unit_values.ptr;
    V.stops = want_stops || risk ? B.vstops.ptr : nullptr;
    V.counts = B.counts.ptr;
    if (lv) {
        // Local volatility stores the valuation paths too (the training store
        // is free once the policy is fitted), then applies the policy to them.
        double* vs = B.spots.ptr;
        if (v_paths > t_paths) {
            MCG_CUDA(B.vspots.alloc(static_cast<size_t>(dates) * v_paths));
            vs = B.vspots.ptr;
        }
        MCG_CUDA(launch_lsm_lv_spots(VP, /*Valuation*/ 0u, vs, v_paths, &B.path_errors.ptr[1], stream));
        ++launches;
        V.spots = vs;
        V.paths = v_paths;
    }
    if (use_mlp) {
        MCG_CUDA(launch_lsm_bs_value_mlp(VP, V, B.mlp_snapshots.ptr, 1.0 / d->observation_times[last], stream));
    } else {
        MCG_CUDA(launch_lsm_bs_value(VP, V, stream));
    }
    ++launches;
    MCG_CUDA(launch_lsm_group_sum(B.unit_values.ptr, VP.units, v_groups, 0, nullptr, B.group_partials.ptr,
                                  group_ctas, s_val, B.means.ptr, stream));
    launches += 2;
    if (!rqmc) {
        MCG_CUDA(launch_lsm_group_sum(B.unit_values.ptr, VP.units, 1, 0, B.means.ptr, B.group_partials.ptr,
                                      group_ctas, s_sq, nullptr, stream));
        launches += 2;
    }
    // Fixed-policy risk: the valuation stopping dates held, per-tile records
    // of the pathwise components merged per scramble.
    const uint32_t risk_tiles = lsm_risk_tiles(VP.units);
    // Local volatility: the fixed-policy risk runs the adjoint sweeps of a risk
    // plan (the valuation plan with the requests) in exercise-value mode, one
    // per spot runtime (base for the price, Vega and nodes; down and up for
    // the CRN Delta/Gamma), every path paying at its own stopping date.
    mcg_plan rplan;
    std::vector<StatRecord> lv_node_rec;
    if (risk && lv) {
        mcg_plan_desc rd = vd;
        rd.request_delta = d->request_delta;
        rd.request_gamma = d->request_gamma;
        rd.request_vega = 1;
        rd.request_local_vega_nodes = d->request_local_vega_nodes;
        if ((st = build(&rd, rplan)) != MCG_OK) return st;
        const DevicePlan& RP = rplan.dp;
        const int pairs = RP.antithetic ? 2 : 1;
        const bool crn = RP.lv_bumps != 0;
        const uint64_t chunk = rplan.chunk_units;
        MCG_CUDA(B.risk_partials.alloc(static_cast<size_t>(v_groups) * rplan.tiles * kComponents));
        MCG_CUDA(B.risk_records.alloc(static_cast<size_t>(v_groups) * kComponents));
        MCG_CUDA(B.risk_price.alloc(6 * chunk));
        const ErrorWord init{~0ull, 0, 0, 0, 0};
        MCG_CUDA(cudaMemcpyAsync(rplan.error.ptr, &init, sizeof(init), cudaMemcpyHostToDevice, stream));
        for (uint32_t sc = 0; sc < RP.scramble_count; ++sc)
            for (uint64_t begin = 0; begin < RP.units; begin += chunk) {
                const uint64_t n = std::min<uint64_t>(chunk, RP.units - begin);
                const uint32_t tile_offset = sc * rplan.tiles + static_cast<uint32_t>(begin / kThreads);
                for (int pr = 0; pr < pairs; ++pr)
                    for (int which : {1, 2, 0}) {
                        if (which != 0 && !crn) continue;
                        AdjointArgs AA{};
                        AA.which = which;
                        AA.sign = pr == 0 ? 1.0 : -1.0;
                        AA.node_weight = pairs == 2 ? 0.5 : 1.0;
                        AA.node_add = pr;
                        AA.scramble = sc;
                        AA.unit_begin = begin;
                        AA.units = n;
                        AA.tile_offset = tile_offset;
                        AA.tape_f = rplan.tape.ptr;
                        AA.tape_z = rplan.tape.ptr + static_cast<size_t>(RP.steps + 1) * chunk;
                        AA.out_vega = rplan.adj_vega.ptr + static_cast<size_t>(pr * 3 + which) * n;
                        AA.out_delta = rplan.adj_delta.ptr + static_cast<size_t>(pr * 3 + which) * n;
                        AA.node_tiles = (which == 0 && rplan.adjoint_nodes) ? rplan.node_tiles.ptr : nullptr;
                        AA.out_price = B.risk_price.ptr + static_cast<size_t>(pr * 3 + which) * n;
                        AA.stops = B.vstops.ptr + ((static_cast<uint64_t>(sc) * RP.units + begin) * pairs + pr);
                        AA.stop_stride = static_cast<uint32_t>(pairs);
                        AA.exercise_df = B.df.ptr;
                        MCG_CUDA(launch_lv_adjoint(RP, AA, rplan.error.ptr, stream));
                        ++launches;
                    }
                MCG_CUDA(launch_lv_fixed_policy_combine(B.risk_price.ptr, rplan.adj_vega.ptr, n, pairs, crn ? 1 : 0,
                                                        d->request_gamma ? 1 : 0, 1, RP.spot_bump, tile_offset,
                                                        B.risk_partials.ptr, stream));
                ++launches;
            }
        reduce_tiles_kernel<<<dim3(kComponents, v_groups), 256, 0, stream>>>(B.risk_partials.ptr, rplan.tiles,
                                                                            kComponents, B.risk_records.ptr);
        MCG_CUDA(cudaGetLastError());
        ++launches;
        if (rplan.adjoint_nodes && r->local_vega_nodes && r->node_capacity >= rplan.grid_values) {
            MCG_CUDA(launch_lv_node_reduce(rplan.node_tiles.ptr, rplan.tiles, RP.scramble_count, rplan.grid_values,
                                           rplan.node_records.ptr, stream));
            ++launches;
            lv_node_rec.resize(static_cast<size_t>(RP.scramble_count) * rplan.grid_values);
            MCG_CUDA(cudaMemcpyAsync(lv_node_rec.data(), rplan.node_records.ptr, lv_node_rec.size() * sizeof(StatRecord),
                                     cudaMemcpyDeviceToHost, stream));
        }
    } else if (risk) {
        MCG_CUDA(B.risk_partials.alloc(static_cast<size_t>(v_groups) * risk_tiles * kComponents));
        MCG_CUDA(B.risk_records.alloc(static_cast<size_t>(v_groups) * kComponents));
        LsmRiskArgs R{};
        R.df = B.df.ptr;
        R.stops = B.vstops.ptr;
        R.side = A.side;
        R.strike = A.strike;
        R.notional = A.notional;
        R.gamma = d->request_gamma ? 1 : 0;
        R.gamma_bump = resolve_gamma_bump(d);
        // validation bumps, crates/pricing/src/engine/compile/simulation.rs:481-502
        R.spot_bump = d->request_gamma ? R.gamma_bump : std::min(d->spot * 1.0e-4, 0.5 * d->spot);
        R.vol_bump = d->volatility == 0.0 ? 0.0 : std::min(1.0e-4, d->volatility * 0.5);
        MCG_CUDA(launch_lsm_bs_risk(VP, R, B.risk_partials.ptr, stream));
        reduce_tiles_kernel<<<dim3(kComponents, v_groups), 256, 0, stream>>>(B.risk_partials.ptr, risk_tiles,
                                                                            kComponents, B.risk_records.ptr);
        MCG_CUDA(cudaGetLastError());
        launches += 2;
    }
    MCG_CUDA(cudaEventRecord(B.ev[3], stream));

    std::vector<DD> sums(4 * static_cast<size_t>(max_groups));
    unsigned long long words[2];
    std::vector<unsigned long long> counts(dates);
    MCG_CUDA(cudaMemcpyAsync(sums.data(), B.sums.ptr, sums.size() * sizeof(DD), cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaMemcpyAsync(words, B.words.ptr, sizeof(words), cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaMemcpyAsync(counts.data(), B.counts.ptr, dates * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, stream));
    if (dates > 1)
        MCG_CUDA(cudaMemcpyAsync(r->models, B.models.ptr, (dates - 1) * sizeof(mcg_lsm_date_model),
                                 cudaMemcpyDeviceToHost, stream));
    if (want_stops)
        MCG_CUDA(cudaMemcpyAsync(r->stopping_indices, B.vstops.ptr, v_paths * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, stream));
    std::vector<StatRecord> risk_rec(risk ? static_cast<size_t>(v_groups) * kComponents : 0);
    if (risk)
        MCG_CUDA(cudaMemcpyAsync(risk_rec.data(), B.risk_records.ptr, risk_rec.size() * sizeof(StatRecord),
                                 cudaMemcpyDeviceToHost, stream));
    ErrorWord path_errors[2] = {{~0ull, 0, 0, 0, 0}, {~0ull, 0, 0, 0, 0}};
    if (lv)
        MCG_CUDA(cudaMemcpyAsync(path_errors, B.path_errors.ptr, sizeof(path_errors), cudaMemcpyDeviceToHost,
                                 stream));
    MCG_CUDA(cudaStreamSynchronize(stream));
    for (int k = 0; k < 2; ++k)
        if (path_errors[k].key != ~0ull) {
            // LocalVolError::NonFiniteState of the Log-Euler step (local_vol.rs:24-73)
            r->error.code = static_cast<int32_t>(path_errors[k].key & 0xff);
            r->error.sampling_unit = path_errors[k].key >> 8;
            return fail(static_cast<mcg_status>(r->error.code),
                        std::string(k ? "valuation" : "training") + " path of sampling unit " +
                            std::to_string(r->error.sampling_unit) + " left the positive finite states");
        }
    if (words[0] != ~0ull) {
        r->error.code = MCG_ERR_LSM;
        r->error.sampling_unit = words[0];
        return fail(MCG_ERR_LSM, "non-finite training spot (NonFiniteFeature) in sampling unit " +
                                     std::to_string(words[0]));
    }
    if (words[1] != ~0ull) {
        const uint32_t date = static_cast<uint32_t>(words[1] >> 8);
        r->error.code = MCG_ERR_LSM;
        r->error.step = date;
        return fail(MCG_ERR_LSM, "regression of exercise date " + std::to_string(date) +
                                     " exceeds max_matrix_elements or is not finite");
    }
    float ms[3] = {0.f, 0.f, 0.f};
    cudaEventElapsedTime(&ms[0], B.ev[0], B.ev[1]);
    cudaEventElapsedTime(&ms[1], B.ev[1], B.ev[2]);
    cudaEventElapsedTime(&ms[2], B.ev[2], B.ev[3]);
    r->path_kernel_ms = ms[0];
    r->regression_ms = ms[1];
    r->valuation_ms = ms[2];
    r->device_ms = ms[0] + ms[1] + ms[2];
    for (uint32_t i = 0; i < dates; ++i) r->exercise_counts[i] = counts[i];

    r->in_sample_value = in_sample_of(sums, use_mlp ? 3 * static_cast<size_t>(max_groups) : 0);
    HostStat hs;
    uint64_t independent;
    if (rqmc) {
        std::vector<double> reps(v_groups);
        for (uint32_t g = 0; g < v_groups; ++g)
            reps[g] = (sums[max_groups + g].hi + sums[max_groups + g].lo) / static_cast<double>(VP.units);
        hs = two_pass(reps);
        independent = v_groups;
    } else {
        const DD tv = sums[max_groups], sq = sums[2 * static_cast<size_t>(max_groups)];
        hs.sum = tv.hi;
        hs.corr = tv.lo;
        hs.count = VP.units;
        hs.mean = (tv.hi + tv.lo) / static_cast<double>(VP.units);
        hs.m2 = sq.hi + sq.lo;
        independent = VP.units;
    }
    r->price_statistics = {hs.sum, hs.corr, hs.count, hs.mean, hs.m2};
    r->price = make_estimate(hs, independent, 1.0);
    r->sampling_variance = hs.count > 1 ? hs.m2 / static_cast<double>(hs.count - 1) : 0.0;
    r->estimator_variance = r->sampling_variance / static_cast<double>(independent);
    r->training_paths = t_paths;
    r->valuation_paths = v_paths;
    r->independent_sampling_units = independent;
    r->date_count = dates;
    r->kernel_launches = launches;
    // Fixed-policy Greeks: pseudo statistics over sampling units, RQMC over
    // the per-scramble replicate means (early_exercise.rs:454-600).
    std::memset(r->risk_components, 0, sizeof(r->risk_components));
    r->delta = r->gamma = r->vega = mcg_estimate{};
    r->bump_delta = r->bump_gamma = r->bump_vega = mcg_estimate{};
    if (risk && lv) {
        ErrorWord ew{~0ull, 0, 0, 0, 0};
        MCG_CUDA(cudaMemcpy(&ew, rplan.error.ptr, sizeof(ew), cudaMemcpyDeviceToHost));
        if (ew.key != ~0ull) {
            r->error.code = static_cast<int32_t>(ew.key & 0xff);
            r->error.sampling_unit = ew.key >> 8;
            return fail(static_cast<mcg_status>(r->error.code),
                        "fixed-policy risk: sampling unit " + std::to_string(r->error.sampling_unit) + " failed");
        }
        const uint32_t nv = rplan.grid_values;
        for (uint32_t k = 0; k < nv && !lv_node_rec.empty(); ++k) {
            const HostStat h = node_statistics(lv_node_rec, nv, k, VP.units, VP.scramble_count, rqmc);
            r->local_vega_nodes[k] = {h.sum, h.corr, h.count, h.mean, h.m2};
            if (r->local_vega_node_estimates) r->local_vega_node_estimates[k] = make_estimate(h, independent, 1.0);
        }
    }
    if (risk) {
        HostStat rs[kComponents];
        for (int c = 0; c < kComponents; ++c) {
            if (c >= 10) {
                rs[c].count = independent;
            } else if (!rqmc) {
                const StatRecord& x = risk_rec[c];
                rs[c] = {x.sum, x.corr, static_cast<uint64_t>(x.count), x.mean, x.m2};
            } else {
                std::vector<double> reps(v_groups);
                for (uint32_t g = 0; g < v_groups; ++g) {
                    const StatRecord& x = risk_rec[static_cast<size_t>(g) * kComponents + c];
                    reps[g] = (x.sum + x.corr) / static_cast<double>(VP.units);
                }
                rs[c] = two_pass(reps);
            }
            r->risk_components[c] = {rs[c].sum, rs[c].corr, rs[c].count, rs[c].mean, rs[c].m2};
        }
        r->delta = make_estimate(rs[MCG_DELTA], independent, 1.0);
        r->gamma = make_estimate(rs[MCG_GAMMA], independent, 1.0);
        r->vega = make_estimate(rs[MCG_VEGA], independent, 1.0);
        r->bump_delta = make_estimate(rs[MCG_BUMP_DELTA], independent, 1.0);
        r->bump_gamma = make_estimate(rs[MCG_BUMP_GAMMA], independent, 1.0);
        r->bump_vega = make_estimate(rs[MCG_BUMP_VEGA], independent, 1.0);
    }
    return MCG_OK;
}

// AndersenBroadiePlan::compile/evaluate (crates/pricing/src/engine/risk/dual.rs:140-404):
// the policy trained and the outer paths valued by lsm_price, then the
// nested simulation of mcg_dual.cu around that policy.
mcg_status lsm_dual(const mcg_plan_desc* d, const mcg_lsm_desc* l, const mcg_dual_desc* x, cudaStream_t stream,
                    mcg_dual_result* r) {
    if (!d || !l || !x || !r) return fail(MCG_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(r, 0, sizeof(*r));
    if (d->product_count != 1 || !d->products || d->products[0].kind != MCG_PRODUCT_AMERICAN)
        return fail(MCG_ERR_INVALID_ARGUMENT, "the dual prices exactly one American product");
    if (d->model != MCG_MODEL_BLACK_SCHOLES)
        return fail(MCG_ERR_UNSUPPORTED, "the dual upper bound runs under Black-Scholes");
    if (d->engine != MCG_ENGINE_PSEUDO)
        return fail(MCG_ERR_UNSUPPORTED, "the dual upper bound needs pseudo-MC training and valuation engines");
    if (l->continuation != MCG_CONTINUATION_POLYNOMIAL)
        return fail(MCG_ERR_UNSUPPORTED, "the dual upper bound uses the polynomial policy");
    if (d->request_delta || d->request_gamma || d->request_vega || d->request_local_vega_nodes)
        return fail(MCG_ERR_UNSUPPORTED, "Greeks of the dual (use a fixed-policy risk request)");
    if (x->continuation_inner_paths == 0 || x->exercise_inner_paths == 0)
        return fail(MCG_ERR_INVALID_ARGUMENT, "inner path counts must be positive");
    const uint32_t dates = d->observation_count;
    const uint64_t lanes = d->antithetic ? 2 : 1;
    const uint64_t stride = std::max(x->continuation_inner_paths, x->exercise_inner_paths);
    const uint64_t trajectories = d->sampling_units * lanes;
    if (d->sampling_units == 0 || trajectories / lanes != d->sampling_units ||
        trajectories > std::numeric_limits<uint64_t>::max() / stride ||
        static_cast<uint64_t>(dates) * dates > 0xffffffffull)
        return fail(MCG_ERR_INVALID_ARGUMENT, "random-coordinate count overflows");
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    struct EventGuard {
        cudaEvent_t* e;
        ~EventGuard() {
            for (int i = 0; i < 4; ++i)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    } guard{ev};
    for (cudaEvent_t& e : ev) MCG_CUDA(cudaEventCreate(&e));
    MCG_CUDA(cudaEventRecord(ev[0], stream));
    // The policy (and the lower bound's valuation, the same outer paths).
    std::vector<mcg_lsm_date_model> models(std::max<uint32_t>(dates - 1, 1));
    std::vector<uint64_t> counts(dates);
    mcg_lsm_result lr{};
    lr.date_capacity = dates;
    lr.models = models.data();
    lr.exercise_counts = counts.data();
    mcg_status st = lsm_price(d, l, stream, &lr);
    if (st != MCG_OK) {
        r->error = lr.error;
        return st;
    }
    mcg_product_desc placeholder = d->products[0];
    placeholder.kind = MCG_PRODUCT_EUROPEAN;
    mcg_plan_desc vd = *d;
    vd.products = &placeholder;
    vd.payment_time = d->observation_times[dates - 1];
    mcg_plan vplan;
    if ((st = build(&vd, vplan)) != MCG_OK) return st;
    const DevicePlan& P = vplan.dp;
    HostCurve rc;
    std::string why;
    if (!load_curve(d->discount_curve, rc, "discount_curve", why)) return fail(MCG_ERR_MARKET, why);
    std::vector<double> df(dates), sq(dates, 0.0);
    for (uint32_t i = 0; i < dates; ++i) df[i] = std::exp(rc.log_discount(d->observation_times[i]));
    for (uint32_t i = 1; i < dates; ++i) sq[i] = std::sqrt(d->observation_times[i] - d->observation_times[i - 1]);
    DeviceArray<mcg_lsm_date_model> dmodels;
    DeviceArray<double> ddf, dsq, spot, brownian, continuation;
    DeviceArray<uint8_t> exercise;
    DeviceArray<unsigned long long> words;
    DeviceArray<StatRecord> partials, records;
    MCG_CUDA(dmodels.upload(models));
    MCG_CUDA(ddf.upload(df));
    MCG_CUDA(dsq.upload(sq));
    const size_t cells = static_cast<size_t>(dates) * trajectories;
    MCG_CUDA(spot.alloc(cells));
    MCG_CUDA(brownian.alloc(cells));
    MCG_CUDA(continuation.alloc(cells));
    MCG_CUDA(exercise.alloc(cells));
    MCG_CUDA(words.alloc(2));
    const uint32_t tiles = static_cast<uint32_t>((P.units + kThreads - 1) / kThreads);
    MCG_CUDA(partials.alloc(static_cast<size_t>(tiles) * 3));
    MCG_CUDA(records.alloc(3));
    const unsigned long long init[2] = {~0ull, 0ull};
    MCG_CUDA(cudaMemcpyAsync(words.ptr, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    DualArgs A{};
    A.models = dmodels.ptr;
    A.nb = l->max_degree + 1;
    A.df = ddf.ptr;
    A.sqrt_step = dsq.ptr;
    A.side = d->products[0].side;
    A.strike = d->products[0].strike;
    A.notional = d->products[0].notional;
    A.trajectories = trajectories;
    A.path_stride = stride;
    A.continuation_inner_paths = x->continuation_inner_paths;
    A.exercise_inner_paths = x->exercise_inner_paths;
    A.inner_seed = x->inner_seed;
    A.spot = spot.ptr;
    A.brownian = brownian.ptr;
    A.exercise = exercise.ptr;
    A.continuation = continuation.ptr;
    A.failure = &words.ptr[0];
    A.inner_count = &words.ptr[1];
    uint32_t launches = lr.kernel_launches;
    MCG_CUDA(launch_dual(P, A, partials.ptr, stream, ev[1], ev[2], launches));
    reduce_tiles_kernel<<<dim3(3, 1), 256, 0, stream>>>(partials.ptr, tiles, 3, records.ptr);
    MCG_CUDA(cudaGetLastError());
    ++launches;
    MCG_CUDA(cudaEventRecord(ev[3], stream));
    StatRecord rec[3];
    unsigned long long w[2];
    MCG_CUDA(cudaMemcpyAsync(rec, records.ptr, sizeof(rec), cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaMemcpyAsync(w, words.ptr, sizeof(w), cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaStreamSynchronize(stream));
    if (w[0] != ~0ull) {
        r->error.code = MCG_ERR_LSM;
        r->error.sampling_unit = w[0] / lanes;
        return fail(MCG_ERR_LSM, "non-finite dual intermediate on outer trajectory " + std::to_string(w[0]));
    }
    mcg_estimate* est[3] = {&r->lower_bound, &r->upper_bound, &r->duality_gap};
    for (int c = 0; c < 3; ++c) {
        const HostStat h{rec[c].sum, rec[c].corr, static_cast<uint64_t>(rec[c].count), rec[c].mean, rec[c].m2};
        r->components[c] = {h.sum, h.corr, h.count, h.mean, h.m2};
        *est[c] = make_estimate(h, P.units, 1.0);
    }
    r->price_confidence_interval_95[0] = r->lower_bound.confidence_lower;
    r->price_confidence_interval_95[1] = r->upper_bound.confidence_upper;
    r->outer_trajectories = trajectories;
    r->inner_paths = w[1];
    r->exercise_date_count = dates;
    r->kernel_launches = launches;
    float ms = 0.f, nested = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[3]);
    cudaEventElapsedTime(&nested, ev[1], ev[2]);
    r->device_ms = ms;
    r->nested_ms = nested;
    return MCG_OK;
}

// --------------------------------------------------------------- book of trades

}  // namespace

struct mcg_book {
    std::vector<mcg_plan*> plans;
    std::vector<uint32_t> trade_family, trade_path, trade_steps;
    std::vector<BookItem> host_items[kBookFamilies];
    DeviceArray<DevicePlan> dplans;
    DeviceArray<uint32_t> masks;
    DeviceArray<BookItem> items[kBookFamilies];
    DeviceArray<unsigned int> cursor;  // one per family
    DeviceArray<StatRecord> partials, records;
    DeviceArray<ErrorWord> errors;
    uint32_t trades = 0, tiles = 0;
    uint32_t max_nodes[kBookFamilies] = {0, 0, 0, 0}, max_slots[kBookFamilies] = {1, 1, 1, 1};
    size_t smem[kBookFamilies] = {0, 0, 0, 0};
    int fit[kBookFamilies] = {1, 1, 1, 1};
    uint32_t ctas[kBookFamilies] = {0, 0, 0, 0};
    uint64_t family_cost[kBookFamilies] = {0, 0, 0, 0};
    uint32_t tiles_per_item = 4, ctas_per_sm = 0;  // 0: every family at its own occupancy
    uint64_t units = 0, path_steps = 0;
    int sms = 148;
    float autotune_ms = 0.f;
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    ~mcg_book() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (capture_stream) cudaStreamDestroy(capture_stream);
        for (mcg_plan* p : plans) delete p;
        dplans.release();
        masks.release();
        for (auto& it : items) it.release();
        cursor.release();
        partials.release();
        records.release();
        errors.release();
    }
};

namespace {

// Work items of `tiles_per_item` tiles (even in the two-path family, from even
// first tiles), per family ordered heaviest first (cost = tiles x steps, local
// volatility weighted 3x for its interpolation); ties keep trade order, so the
// queues are deterministic.
void book_items(mcg_book& b, uint32_t tiles_per_item, const std::vector<uint32_t>& trades) {
    for (uint32_t f = 0; f < kBookFamilies; ++f) {
        std::vector<std::pair<uint64_t, BookItem>> order;
        for (uint32_t t : trades) {
            if (b.trade_family[t] != f) continue;
            const uint32_t step = f == kFamilyLvDiscrete ? (tiles_per_item + 1) & ~1u : tiles_per_item;
            for (uint32_t first = 0; first < b.tiles; first += step) {
                const uint32_t n = std::min(step, b.tiles - first);
                const BookItem it{t, first, n, b.trade_path[t]};
                order.emplace_back(static_cast<uint64_t>(n) * b.trade_steps[t] * (it.path == kBookLocalVol ? 3 : 1), it);
            }
        }
        std::stable_sort(order.begin(), order.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        b.host_items[f].clear();
        b.family_cost[f] = 0;
        for (auto& o : order) {
            b.host_items[f].push_back(o.second);
            b.family_cost[f] += o.first;
        }
    }
}

BookLaunch book_launch(mcg_book& b, uint32_t f) {
    BookLaunch L{};
    L.plans = b.dplans.ptr;
    L.masks = b.masks.ptr;
    L.items = b.items[f].ptr;
    L.item_count = static_cast<uint32_t>(b.host_items[f].size());
    L.next = b.cursor.ptr + f;
    L.partials = b.partials.ptr;
    L.tiles_per_trade = b.tiles;
    L.errors = b.errors.ptr;
    L.max_nodes = b.max_nodes[f];
    L.max_slots = b.max_slots[f];
    return L;
}

// The families in launch order: heaviest first.
std::vector<uint32_t> book_order(const mcg_book& b) {
    std::vector<uint32_t> order;
    for (uint32_t f = 0; f < kBookFamilies; ++f)
        if (!b.host_items[f].empty()) order.push_back(f);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t x, uint32_t y) { return b.family_cost[x] > b.family_cost[y]; });
    return order;
}

// The evaluation's launches: queue reset, error words, one persistent kernel
// per family, the per-trade reduction.
cudaError_t book_enqueue(mcg_book& b, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(b.cursor.ptr, 0, kBookFamilies * sizeof(unsigned int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.errors.ptr, 0xff, b.trades * sizeof(ErrorWord), stream);
    for (uint32_t f : book_order(b))
        if (e == cudaSuccess) e = launch_book(f, book_launch(b, f), b.ctas[f], b.smem[f], stream);
    if (e == cudaSuccess) {
        reduce_tiles_kernel<<<dim3(kComponents, b.trades), 256, 0, stream>>>(b.partials.ptr, b.tiles, kComponents,
                                                                          b.records.ptr);
        e = cudaGetLastError();
    }
    return e;
}

mcg_status book_set_shape(mcg_book& b, uint32_t tiles_per_item, uint32_t ctas_per_sm,
                          const std::vector<uint32_t>& trades) {
    b.tiles_per_item = tiles_per_item;
    b.ctas_per_sm = ctas_per_sm;
    book_items(b, tiles_per_item, trades);
    for (uint32_t f = 0; f < kBookFamilies; ++f) {
        const int per_sm = ctas_per_sm ? std::min<int>(static_cast<int>(ctas_per_sm), b.fit[f]) : b.fit[f];
        b.ctas[f] = static_cast<uint32_t>(b.sms) * static_cast<uint32_t>(std::max(per_sm, 1));
        b.items[f].release();
        MCG_CUDA(b.items[f].upload(b.host_items[f]));
    }
    return MCG_OK;
}

mcg_status book_create(const mcg_plan_desc* trades, uint32_t n, const mcg_book_options* opt, mcg_book** out) {
    if (!out) return fail(MCG_ERR_INVALID_ARGUMENT, "null out_book");
    *out = nullptr;
    if (!trades || n == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "empty book");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
        return fail(MCG_ERR_CUDA, "no CUDA device is visible");
    std::unique_ptr<mcg_book> b(new (std::nothrow) mcg_book());
    if (!b) return fail(MCG_ERR_ALLOCATION, "book allocation");
    b->trades = n;
    b->units = trades[0].sampling_units;
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, 0);
    std::vector<DevicePlan> dp(n);
    std::vector<uint32_t> masks(n);
    for (uint32_t i = 0; i < n; ++i) {
        const mcg_plan_desc& d = trades[i];
        const std::string who = "trade " + std::to_string(i) + ": ";
        if (d.discrete_dividends.count)
            return fail(MCG_ERR_UNSUPPORTED, who + "a book prices trades without discrete dividends");
        if (d.engine != MCG_ENGINE_PSEUDO || d.product_count != 1 || d.request_delta || d.request_gamma ||
            d.request_vega || d.request_local_vega_nodes)
            return fail(MCG_ERR_UNSUPPORTED, who + "a book trade is pseudo-MC, one product, price only");
        if (d.sampling_units != b->units)
            return fail(MCG_ERR_INVALID_ARGUMENT, who + "every trade of a book has the same sampling_units");
        if (d.model == MCG_MODEL_LOCAL_VOLATILITY && d.antithetic)
            return fail(MCG_ERR_UNSUPPORTED, who + "local-volatility book trades are not antithetic");
        if (d.precision != MCG_PRECISION_F64) return fail(MCG_ERR_UNSUPPORTED, who + "a book prices in FP64");
        auto* plan = new (std::nothrow) mcg_plan();
        if (!plan) return fail(MCG_ERR_ALLOCATION, "plan allocation");
        b->plans.push_back(plan);
        const mcg_status st = build(&d, *plan, false);
        if (st != MCG_OK) return fail(st, who + g_last_error);
        dp[i] = plan->dp;
        masks[i] = plan->mask;
        const bool lv = d.model == MCG_MODEL_LOCAL_VOLATILITY;
        const bool cont = d.products[0].kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
        const uint32_t family = lv ? (cont ? kFamilyLvBarrier : kFamilyLvDiscrete)
                                   : (plan->single_terminal ? kFamilyBsTerminal : kFamilyBsPath);
        b->trade_family.push_back(family);
        b->trade_path.push_back(lv ? kBookLocalVol : (plan->single_terminal ? kBookBsTerminal : kBookBsPath));
        const uint32_t steps = lv ? plan->dp.steps : (plan->single_terminal ? 1u : plan->dp.observation_count);
        b->trade_steps.push_back(steps);
        b->path_steps += b->units * steps * (d.antithetic ? 2u : 1u);
        if (lv) {
            b->max_nodes[family] = std::max(b->max_nodes[family], plan->dp.nx);
            b->max_slots[family] = std::max(b->max_slots[family], plan->dp.slot_count);
        }
    }
    b->tiles = b->plans[0]->tiles;
    for (uint32_t f = 0; f < kBookFamilies; ++f) {
        b->smem[f] = book_smem_bytes(f, b->max_nodes[f], b->max_slots[f]);
        if (b->smem[f] > 200 * 1024) return fail(MCG_ERR_UNSUPPORTED, "book grids too large for shared memory");
        MCG_CUDA(book_prepare(f, b->smem[f]));
        MCG_CUDA(book_occupancy(f, b->smem[f], &b->fit[f]));
        b->fit[f] = std::max(b->fit[f], 1);
    }
    MCG_CUDA(b->dplans.upload(dp));
    MCG_CUDA(b->masks.upload(masks));
    MCG_CUDA(b->cursor.alloc(kBookFamilies));
    MCG_CUDA(b->partials.alloc(static_cast<size_t>(n) * b->tiles * kComponents));
    MCG_CUDA(b->records.alloc(static_cast<size_t>(n) * kComponents));
    MCG_CUDA(b->errors.alloc(n));
    std::vector<uint32_t> all(n);
    for (uint32_t i = 0; i < n; ++i) all[i] = i;
    mcg_book_options o{};
    if (opt) o = *opt;
    uint32_t tpi = o.tiles_per_item ? o.tiles_per_item : 4u;
    const uint32_t cps = o.ctas_per_sm;
    if (o.autotune) {
        // Tiles per work item timed on a stratified sample (every k-th trade of
        // the book, at most 128 trades), the fastest kept; every family runs at
        // its own occupancy (or the caller's cap).
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<uint32_t> sample;
        const uint32_t stride = std::max(1u, n / 128u);
        for (uint32_t i = 0; i < n; i += stride) sample.push_back(i);
        cudaStream_t s;
        MCG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        cudaEvent_t e0, e1;
        MCG_CUDA(cudaEventCreate(&e0));
        MCG_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        uint32_t best_tpi = tpi;
        mcg_status st = MCG_OK;
        for (uint32_t cand_tpi : {2u, 4u, 16u}) {
            if ((st = book_set_shape(*b, cand_tpi, cps, sample)) != MCG_OK) break;
            float ms = 0.f;
            for (int rep = 0; rep < 2; ++rep) {  // the first run warms the caches
                if (cudaEventRecord(e0, s) != cudaSuccess || book_enqueue(*b, s) != cudaSuccess ||
                    cudaEventRecord(e1, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
                    st = fail(MCG_ERR_CUDA, "book autotune launch failed");
                    break;
                }
                cudaEventElapsedTime(&ms, e0, e1);
            }
            if (st != MCG_OK) break;
            if (ms < best) {
                best = ms;
                best_tpi = cand_tpi;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(s);
        if (st != MCG_OK) return st;
        tpi = best_tpi;
        b->autotune_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    mcg_status st = book_set_shape(*b, tpi, cps, all);
    if (st != MCG_OK) return st;
    if (o.use_graph) {
        MCG_CUDA(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking));
        MCG_CUDA(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t ce = book_enqueue(*b, b->capture_stream);
        const cudaError_t ee = cudaStreamEndCapture(b->capture_stream, &b->graph);
        if (ce != cudaSuccess || ee != cudaSuccess)
            return fail(MCG_ERR_CUDA, std::string("book graph capture: ") +
                                          cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        MCG_CUDA(cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
    }
    *out = b.release();
    return MCG_OK;
}

mcg_status book_evaluate(mcg_book* b, cudaStream_t stream, mcg_estimate* prices, mcg_book_report* report) {
    if (!b || !prices) return fail(MCG_ERR_INVALID_ARGUMENT, "null book or prices");
    cudaEvent_t e0, e1;
    MCG_CUDA(cudaEventCreate(&e0));
    MCG_CUDA(cudaEventCreate(&e1));
    MCG_CUDA(cudaEventRecord(e0, stream));
    if (b->graph_exec) {
        MCG_CUDA(cudaGraphLaunch(b->graph_exec, stream));
    } else {
        MCG_CUDA(book_enqueue(*b, stream));
    }
    MCG_CUDA(cudaEventRecord(e1, stream));
    std::vector<StatRecord> rec(static_cast<size_t>(b->trades) * kComponents);
    std::vector<ErrorWord> errs(b->trades);
    MCG_CUDA(cudaMemcpyAsync(rec.data(), b->records.ptr, rec.size() * sizeof(StatRecord), cudaMemcpyDeviceToHost,
                             stream));
    MCG_CUDA(cudaMemcpyAsync(errs.data(), b->errors.ptr, errs.size() * sizeof(ErrorWord), cudaMemcpyDeviceToHost,
                             stream));
    MCG_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (report) {
        std::memset(report, 0, sizeof(*report));
        const std::vector<uint32_t> order = book_order(*b);
        report->trade_count = b->trades;
        for (uint32_t f : order) {
            report->items += static_cast<uint32_t>(b->host_items[f].size());
            report->ctas += b->ctas[f];
        }
        report->tiles_per_item = b->tiles_per_item;
        report->ctas_per_sm = order.empty() ? 0u : b->ctas[order[0]] / static_cast<uint32_t>(b->sms);
        report->kernel_launches = static_cast<uint32_t>(order.size()) + 1u;
        report->graph = b->graph_exec ? 1 : 0;
        report->device_ms = ms;
        report->autotune_ms = b->autotune_ms;
        report->path_steps = b->path_steps;
    }
    for (uint32_t t = 0; t < b->trades; ++t)
        if (errs[t].key != ~0ull) {
            if (report) {
                report->error.code = static_cast<int32_t>(errs[t].key & 0xff);
                report->error.step = t;
                report->error.sampling_unit = errs[t].key >> 8;
            }
            return fail(static_cast<mcg_status>(errs[t].key & 0xff),
                        "trade " + std::to_string(t) + ", sampling unit " + std::to_string(errs[t].key >> 8) +
                            " failed");
        }
    for (uint32_t t = 0; t < b->trades; ++t) {
        const StatRecord& s = rec[static_cast<size_t>(t) * kComponents + MCG_PRICE];
        const HostStat h{s.sum, s.corr, static_cast<uint64_t>(s.count), s.mean, s.m2};
        prices[t] = make_estimate(h, b->units, 1.0);
    }
    return MCG_OK;
}

}  // namespace

namespace mcg {
// Lets other translation units report through mcg_last_error().
void set_last_error(const std::string& message) { g_last_error = message; }
}  // namespace mcg

namespace {

// CorrelationFactor::compile (crates/pricing-numerics/src/correlation.rs:61-180)
// with every tolerance 1e-12: symmetric average, unit diagonal, unpivoted
// lower Cholesky factor of a positive semi-definite matrix whose zero pivots
// leave zero columns (residuals checked against the same tolerance).
bool correlation_lower(const double* raw, uint32_t n, std::vector<double>& lower, std::string& why) {
    const double tol = 1e-12;
    std::vector<double> c(raw, raw + static_cast<size_t>(n) * n);
    for (double v : c)
        if (!std::isfinite(v)) {
            why = "correlation: non-finite entry";
            return false;
        }
    for (uint32_t i = 0; i < n; ++i) {
        if (std::fabs(raw[i * n + i] - 1.0) > tol) {
            why = "correlation: diagonal must be 1";
            return false;
        }
        c[i * n + i] = 1.0;
        for (uint32_t j = i + 1; j < n; ++j) {
            if (std::fabs(raw[i * n + j] - raw[j * n + i]) > tol) {
                why = "correlation: matrix must be symmetric";
                return false;
            }
            const double avg = (raw[i * n + j] + raw[j * n + i]) * 0.5;
            if (!(avg >= -1.0 && avg <= 1.0)) {
                why = "correlation: entries must lie in [-1, 1]";
                return false;
            }
            c[i * n + j] = c[j * n + i] = avg;
        }
    }
    double scale = 1.0;
    for (uint32_t i = 0; i < n; ++i) {
        double row = 0.0;
        for (uint32_t j = 0; j < n; ++j) row = row + std::fabs(c[i * n + j]);
        scale = std::max(scale, row);
    }
    const double threshold = std::max(tol, tol * scale);
    lower.assign(static_cast<size_t>(n) * n, 0.0);
    for (uint32_t j = 0; j < n; ++j) {
        double sum = 0.0;
        for (uint32_t k = 0; k < j; ++k) sum += lower[j * n + k] * lower[j * n + k];
        const double pivot = c[j * n + j] - sum;
        if (!std::isfinite(pivot) || pivot < -threshold) {
            why = "correlation: matrix is not positive semi-definite";
            return false;
        }
        if (pivot > threshold) lower[j * n + j] = std::sqrt(pivot);
        for (uint32_t i = j + 1; i < n; ++i) {
            double s2 = 0.0;
            for (uint32_t k = 0; k < j; ++k) s2 += lower[i * n + k] * lower[j * n + k];
            const double residual = c[i * n + j] - s2;
            if (pivot > threshold) {
                lower[i * n + j] = residual / lower[j * n + j];
            } else if (!std::isfinite(residual) || std::fabs(residual) > threshold) {
                why = "correlation: singular matrix with an inconsistent residual";
                return false;
            }
        }
    }
    return true;
}

// Device arrays of one multi-asset evaluation, released on every exit.
struct MultiArrays {
    DeviceArray<double> dt, sqrt_dt, inv_sqrt_dt, lower, ratio, time_weight;
    DeviceArray<int32_t> step_entry, time_cell;
    DeviceArray<double2> bounds[kMaxAssets], cells[kMaxAssets];
    DeviceArray<int4> step_prog;
    DeviceArray<BridgeNode> bridge_nodes;
    DeviceArray<uint32_t> directions, scr_dirs, scr_shift, scr_low, z_dims;
    DeviceArray<StatRecord> partials, records;
    DeviceArray<ErrorWord> error;
    ~MultiArrays() {
        z_dims.release();
        for (auto* a : {&dt, &sqrt_dt, &inv_sqrt_dt, &lower, &ratio, &time_weight}) a->release();
        step_entry.release();
        time_cell.release();
        for (int i = 0; i < kMaxAssets; ++i) {
            bounds[i].release();
            cells[i].release();
        }
        step_prog.release();
        bridge_nodes.release();
        for (auto* a : {&directions, &scr_dirs, &scr_shift, &scr_low}) a->release();
        partials.release();
        records.release();
        error.release();
    }
};

mcg_status multi_asset_price(const mcg_multi_asset_desc* d, cudaStream_t stream, mcg_multi_asset_result* r) {
    if (!d || !r) return fail(MCG_ERR_INVALID_ARGUMENT, "null descriptor or result");
    std::memset(r, 0, sizeof(*r));
    if (d->abi_version != MCG_ABI_VERSION) return fail(MCG_ERR_INVALID_ARGUMENT, "abi_version mismatch");
    const uint32_t n = d->asset_count;
    if (n == 0 || n > MCG_MAX_ASSETS || !d->assets) return fail(MCG_ERR_INVALID_ARGUMENT, "asset_count must be 1..8");
    const double horizon = d->expiry;
    if (!(horizon > 0.0) || !std::isfinite(horizon)) return fail(MCG_ERR_INVALID_ARGUMENT, "expiry");
    if (!(d->payment_time >= horizon) || !std::isfinite(d->payment_time))
        return fail(MCG_ERR_INVALID_ARGUMENT, "payment_time must not precede the expiry");
    if (!(d->maximum_step > 0.0) || !std::isfinite(d->maximum_step))
        return fail(MCG_ERR_INVALID_ARGUMENT, "maximum_step");
    if (!(d->smoothing_half_width >= 0.0) || !std::isfinite(d->smoothing_half_width))
        return fail(MCG_ERR_INVALID_ARGUMENT, "smoothing_half_width");
    if (d->product != MCG_MULTI_BASKET && d->product != MCG_MULTI_WORST_OF)
        return fail(MCG_ERR_UNSUPPORTED, "product");
    if (!std::isfinite(d->strike) || !(d->notional > 0.0) || !std::isfinite(d->notional) || !d->scales ||
        (d->product == MCG_MULTI_BASKET && !d->weights))
        return fail(MCG_ERR_INVALID_ARGUMENT, "strike, notional, weights and scales");
    for (uint32_t i = 0; i < n; ++i)
        if (!(d->scales[i] > 0.0) || !std::isfinite(d->scales[i]) ||
            (d->product == MCG_MULTI_BASKET && !std::isfinite(d->weights[i])))
            return fail(MCG_ERR_INVALID_ARGUMENT, "basket weights must be finite and scales positive");
    const bool rqmc = d->engine == MCG_ENGINE_RQMC;
    if (!rqmc && d->engine != MCG_ENGINE_PSEUDO) return fail(MCG_ERR_UNSUPPORTED, "engine");
    const uint64_t units = d->sampling_units;
    const uint32_t scrambles = rqmc ? d->scramble_count : 1;
    if (units == 0 || (rqmc && (units & (units - 1)) != 0) || units > (1ull << 32))
        return fail(MCG_ERR_INVALID_ARGUMENT, "sampling_units (RQMC: a power of two)");
    if ((rqmc ? scrambles : units) < 2)
        return fail(MCG_ERR_INSUFFICIENT_UNITS, "at least two independent sampling units are required");
    HostCurve rc;
    std::string why;
    if (!load_curve(d->discount_curve, rc, "discount_curve", why)) return fail(MCG_ERR_MARKET, why);
    // correlation term structure
    if (d->correlation_count == 0 || !d->correlation_times || !d->correlations)
        return fail(MCG_ERR_INVALID_ARGUMENT, "correlation term structure is empty");
    std::vector<double> lower;
    for (uint32_t k = 0; k < d->correlation_count; ++k) {
        if (!std::isfinite(d->correlation_times[k]) || (k && !(d->correlation_times[k] > d->correlation_times[k - 1])))
            return fail(MCG_ERR_INVALID_ARGUMENT, "correlation times must be increasing");
        std::vector<double> l;
        if (!correlation_lower(d->correlations + static_cast<size_t>(k) * n * n, n, l, why))
            return fail(MCG_ERR_INVALID_ARGUMENT, why);
        lower.insert(lower.end(), l.begin(), l.end());
    }
    if (!(d->correlation_times[0] <= 0.0))
        return fail(MCG_ERR_INVALID_ARGUMENT, "the first correlation matrix must be in force at the valuation date");
    // time grid: the expiry, correlation changes, the grids' nodes (compile.rs:285-336)
    std::vector<double> events{horizon};
    for (uint32_t k = 0; k < d->correlation_count; ++k)
        if (d->correlation_times[k] > 0.0 && d->correlation_times[k] < horizon) events.push_back(d->correlation_times[k]);
    for (uint32_t i = 0; i < n; ++i) {
        const mcg_asset_desc& a = d->assets[i];
        if (!(a.spot > 0.0) || !std::isfinite(a.spot)) return fail(MCG_ERR_INVALID_ARGUMENT, "asset spot");
        if (a.model == MCG_MODEL_BLACK_SCHOLES) {
            if (!(a.volatility >= 0.0) || !std::isfinite(a.volatility))
                return fail(MCG_ERR_INVALID_ARGUMENT, "asset volatility");
        } else if (a.model == MCG_MODEL_LOCAL_VOLATILITY) {
            const mcg_local_variance_grid& g = a.local_variance;
            if (g.time_count < 2 || g.log_moneyness_count < 2 || !g.time_nodes || !g.log_moneyness_nodes || !g.values)
                return fail(MCG_ERR_MARKET, "local variance grid needs at least 2x2 nodes");
            for (uint32_t k = 0; k < g.time_count; ++k)
                if (!std::isfinite(g.time_nodes[k]) || (k && !(g.time_nodes[k] > g.time_nodes[k - 1])))
                    return fail(MCG_ERR_MARKET, "grid time nodes must be finite and increasing");
            if (bits_of(g.time_nodes[0]) != 0 || g.time_nodes[g.time_count - 1] < horizon)
                return fail(MCG_ERR_MARKET, "local variance grid must cover [0, expiry]");
            for (uint32_t k = 0; k < g.log_moneyness_count; ++k)
                if (!std::isfinite(g.log_moneyness_nodes[k]) ||
                    (k && !(g.log_moneyness_nodes[k] > g.log_moneyness_nodes[k - 1])))
                    return fail(MCG_ERR_MARKET, "grid log-moneyness nodes must be finite and increasing");
            for (size_t k = 0; k < static_cast<size_t>(g.time_count) * g.log_moneyness_count; ++k)
                if (!std::isfinite(g.values[k]) || g.values[k] < g.floor || g.values[k] > g.cap)
                    return fail(MCG_ERR_MARKET, "grid value outside [floor, cap]");
            for (uint32_t k = 0; k < g.time_count; ++k)
                if (g.time_nodes[k] <= horizon) events.push_back(g.time_nodes[k]);
        } else {
            return fail(MCG_ERR_UNSUPPORTED, "multi-asset models are Black-Scholes and local volatility");
        }
    }
    std::vector<double> nodes;
    compile_time_grid(events, d->maximum_step, nodes);
    const uint32_t steps = static_cast<uint32_t>(nodes.size() - 1);
    MultiAssetDev M{};
    M.n = n;
    M.steps = steps;
    M.dimension = n * steps;
    M.engine = d->engine;
    M.antithetic = d->antithetic != 0;
    M.bridge = d->brownian_bridge != 0;
    M.rank_major = rqmc && M.bridge;
    M.seed = d->master_seed;
    M.units = units;
    MultiArrays A;
    {
        std::vector<double> dtv(steps), sq(steps), isq(steps);
        std::vector<int32_t> entry(steps);
        for (uint32_t s = 0; s < steps; ++s) {
            dtv[s] = nodes[s + 1] - nodes[s];
            sq[s] = std::sqrt(dtv[s]);
            isq[s] = 1.0 / std::sqrt(dtv[s]);
            uint32_t e = 0;
            while (e < d->correlation_count && d->correlation_times[e] <= nodes[s]) ++e;
            entry[s] = static_cast<int32_t>(e) - 1;
        }
        MCG_CUDA(A.dt.upload(dtv));
        MCG_CUDA(A.sqrt_dt.upload(sq));
        MCG_CUDA(A.inv_sqrt_dt.upload(isq));
        MCG_CUDA(A.step_entry.upload(entry));
        MCG_CUDA(A.lower.upload(lower));
        M.dt = A.dt.ptr;
        M.sqrt_dt = A.sqrt_dt.ptr;
        M.inv_sqrt_dt = A.inv_sqrt_dt.ptr;
        M.step_entry = A.step_entry.ptr;
        M.lower = A.lower.ptr;
    }
    {
        std::vector<double> ratio(static_cast<size_t>(n) * steps), tw(static_cast<size_t>(n) * steps, 0.0);
        std::vector<int32_t> tc(static_cast<size_t>(n) * steps, 0);
        for (uint32_t i = 0; i < n; ++i) {
            const mcg_asset_desc& a = d->assets[i];
            HostCurve qc;
            if (!load_curve(a.dividend_curve, qc, "asset dividend_curve", why)) return fail(MCG_ERR_MARKET, why);
            std::vector<double> fw(steps + 1);
            for (uint32_t k = 0; k <= steps; ++k) {
                fw[k] = a.spot * std::exp(qc.log_discount(nodes[k]) - rc.log_discount(nodes[k]));
                if (!std::isfinite(fw[k]) || fw[k] <= 0.0) return fail(MCG_ERR_MARKET, "non-finite forward");
            }
            for (uint32_t s = 0; s < steps; ++s) ratio[static_cast<size_t>(i) * steps + s] = fw[s + 1] / fw[s];
            M.model[i] = a.model;
            M.vol[i] = a.volatility;
            M.spot[i] = a.spot;
            M.weights[i] = d->product == MCG_MULTI_BASKET ? d->weights[i] : 0.0;
            M.scales[i] = d->scales[i];
            if (a.model == MCG_MODEL_LOCAL_VOLATILITY) {
                const mcg_local_variance_grid& g = a.local_variance;
                std::vector<double> gt(g.time_nodes, g.time_nodes + g.time_count);
                const uint32_t nx = g.log_moneyness_count, ncell = nx - 1;
                for (uint32_t s = 0; s < steps; ++s) {
                    const int64_t key = host_total_key(nodes[s]);
                    const size_t lo = lower_bound_key(gt, key);
                    size_t c = (lo < gt.size() && host_total_key(gt[lo]) == key) ? lo : (lo == 0 ? 0 : lo - 1);
                    c = std::min(c, gt.size() - 2);
                    tc[static_cast<size_t>(i) * steps + s] = static_cast<int32_t>(c);
                    tw[static_cast<size_t>(i) * steps + s] = (nodes[s] - gt[c]) / (gt[c + 1] - gt[c]);
                }
                std::vector<double2> bounds(ncell), cells(static_cast<size_t>(g.time_count) * ncell);
                for (uint32_t c = 0; c < ncell; ++c)
                    bounds[c] = make_double2(g.log_moneyness_nodes[c], g.log_moneyness_nodes[c + 1]);
                for (uint32_t t = 0; t < g.time_count; ++t)
                    for (uint32_t c = 0; c < ncell; ++c) {
                        const double* row = g.values + static_cast<size_t>(t) * nx;
                        const double inv = 1.0 / (g.log_moneyness_nodes[c + 1] - g.log_moneyness_nodes[c]);
                        cells[static_cast<size_t>(t) * ncell + c] = make_double2(row[c], (row[c + 1] - row[c]) * inv);
                    }
                MCG_CUDA(A.bounds[i].upload(bounds));
                MCG_CUDA(A.cells[i].upload(cells));
                M.bounds[i] = A.bounds[i].ptr;
                M.cells[i] = A.cells[i].ptr;
                M.nx[i] = static_cast<int32_t>(nx);
                M.x_first[i] = g.log_moneyness_nodes[0];
                M.x_last[i] = g.log_moneyness_nodes[nx - 1];
            }
        }
        MCG_CUDA(A.ratio.upload(ratio));
        MCG_CUDA(A.time_cell.upload(tc));
        MCG_CUDA(A.time_weight.upload(tw));
        M.ratio = A.ratio.ptr;
        M.time_cell = A.time_cell.ptr;
        M.time_weight = A.time_weight.ptr;
    }
    std::vector<int4> prog;
    std::vector<BridgeNode> bnodes;
    if (M.bridge) {
        std::vector<BridgeInstr> instrs;
        std::vector<Op> ops;
        uint32_t slots = 1;
        if (!compile_bridge(nodes, instrs)) return fail(MCG_ERR_BRIDGE, "invalid bridge grid");
        if (!bridge_program(nodes, instrs, ops, slots))
            return fail(MCG_ERR_UNSUPPORTED, "bridge needs more than 32 live values");
        int32_t zero_slot = 0;
        if (!step_program(ops, steps, prog, bnodes, zero_slot))
            return fail(MCG_ERR_BRIDGE, "internal: path program steps out of order");
        for (const BridgeNode& b : bnodes)
            if (b.out < 0 || b.out >= static_cast<int32_t>(slots) || b.left < 0 || b.left >= static_cast<int32_t>(slots) ||
                b.right < 0 || b.right >= static_cast<int32_t>(slots) || b.rank < 0 || b.rank >= static_cast<int32_t>(steps))
                return fail(MCG_ERR_BRIDGE, "internal: bridge node index out of range");
        MCG_CUDA(A.step_prog.upload(prog));
        MCG_CUDA(A.bridge_nodes.upload(bnodes));
        M.step_prog = A.step_prog.ptr;
        M.bridge_nodes = A.bridge_nodes.ptr;
        M.zero_slot = zero_slot;
        M.slot_count = slots;
    }
    {
        // The dimensions of a unit's normals in the order the kernel consumes
        // them: per step, each bridge node's rank for every factor, or the
        // step for every factor; dimension factor x steps + rank, or rank x
        // assets + factor when rank-major (path.rs:24-75).
        std::vector<uint32_t> zd;
        auto dim = [&](uint32_t f, uint32_t r) { return M.rank_major ? r * n + f : f * steps + r; };
        for (uint32_t st = 0; st < steps; ++st) {
            if (M.bridge) {
                for (int32_t j = 0; j < prog[st].y; ++j)
                    for (uint32_t q = 0; q < n; ++q)
                        zd.push_back(dim(q, static_cast<uint32_t>(bnodes[static_cast<size_t>(prog[st].x) + j].rank)));
            } else {
                for (uint32_t q = 0; q < n; ++q) zd.push_back(dim(q, st));
            }
        }
        for (uint32_t v : zd)
            if (v >= M.dimension) return fail(MCG_ERR_BRIDGE, "internal: normal dimension out of range");
        MCG_CUDA(A.z_dims.upload(zd));
        M.z_dims = A.z_dims.ptr;
        M.z_count = static_cast<uint32_t>(zd.size());
    }
    if (rqmc) {
        if (M.dimension > MCG_MAX_SOBOL_DIMENSION)
            return fail(MCG_ERR_SOBOL_DIMENSION, "effective Sobol dimension exceeds 21201");
        if (!d->sobol_directions || d->sobol_dimension_count < M.dimension)
            return fail(MCG_ERR_SOBOL_DIMENSION, "sobol_directions cover fewer dimensions than the plan needs");
        std::vector<uint32_t> dirs(d->sobol_directions, d->sobol_directions + static_cast<size_t>(M.dimension) * 32u);
        MCG_CUDA(A.directions.upload(dirs));
        const uint32_t rows = scrambles * M.dimension;
        MCG_CUDA(A.scr_dirs.alloc(static_cast<size_t>(rows) * 32u));
        MCG_CUDA(A.scr_shift.alloc(rows));
        MCG_CUDA(A.scr_low.alloc(static_cast<size_t>(rows) * 32u));
        scramble_table_kernel<<<(rows + 127) / 128, 128, 0, stream>>>(A.directions.ptr, M.dimension, scrambles, 0u,
                                                                     M.seed, A.scr_dirs.ptr, A.scr_shift.ptr);
        MCG_CUDA(cudaGetLastError());
        scramble_low_kernel<<<(rows * 32u + 127) / 128, 128, 0, stream>>>(A.scr_dirs.ptr, rows, A.scr_low.ptr);
        MCG_CUDA(cudaGetLastError());
        M.scr_dirs = A.scr_dirs.ptr;
        M.scr_shift = A.scr_shift.ptr;
        M.scr_low = A.scr_low.ptr;
    }
    M.product = d->product;
    M.side = d->side;
    M.strike = d->strike;
    M.notional = d->notional;
    M.smoothing = d->smoothing_half_width;
    M.df = std::exp(rc.log_discount(d->payment_time));
    if (multi_asset_smem(M) > 200 * 1024) return fail(MCG_ERR_UNSUPPORTED, "bridge slots exceed shared memory");
    const uint32_t tiles = static_cast<uint32_t>((units + kThreads - 1) / kThreads);
    MCG_CUDA(A.partials.alloc(static_cast<size_t>(tiles) * scrambles));
    MCG_CUDA(A.records.alloc(scrambles));
    MCG_CUDA(A.error.alloc(1));
    const ErrorWord init{~0ull, 0, 0, 0, 0};
    MCG_CUDA(cudaMemcpyAsync(A.error.ptr, &init, sizeof(init), cudaMemcpyHostToDevice, stream));
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, stream);
    cudaError_t e = launch_multi_asset(M, scrambles, A.partials.ptr, A.error.ptr, stream);
    if (e == cudaSuccess) {
        reduce_tiles_kernel<<<dim3(1, scrambles), 256, 0, stream>>>(A.partials.ptr, tiles, 1, A.records.ptr);
        e = cudaGetLastError();
    }
    cudaEventRecord(t1, stream);
    std::vector<StatRecord> rec(scrambles);
    ErrorWord ew{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(rec.data(), A.records.ptr, scrambles * sizeof(StatRecord),
                                              cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ew, A.error.ptr, sizeof(ew), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    float ms = 0.0f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
    r->kernel_launches = 2 + (rqmc ? 2 : 0);
    r->device_ms = ms;
    r->time_steps = steps;
    r->dimension = M.dimension;
    if (ew.key != ~0ull) {
        r->error.code = static_cast<int32_t>(ew.key & 0xff);
        r->error.sampling_unit = ew.key >> 8;
        return fail(static_cast<mcg_status>(r->error.code),
                    "sampling unit " + std::to_string(r->error.sampling_unit) + " failed");
    }
    HostStat h;
    if (!rqmc) {
        h = {rec[0].sum, rec[0].corr, static_cast<uint64_t>(rec[0].count), rec[0].mean, rec[0].m2};
    } else {
        std::vector<double> reps(scrambles);
        for (uint32_t sc = 0; sc < scrambles; ++sc) reps[sc] = (rec[sc].sum + rec[sc].corr) / static_cast<double>(units);
        h = two_pass(reps);
    }
    const uint64_t independent = rqmc ? scrambles : units;
    r->price_statistics = {h.sum, h.corr, h.count, h.mean, h.m2};
    r->price = make_estimate(h, independent, 1.0);
    r->sampling_variance = h.count > 1 ? h.m2 / static_cast<double>(h.count - 1) : 0.0;
    r->independent_sampling_units = independent;
    r->evaluated_paths = units * scrambles * (M.antithetic ? 2 : 1);
    return MCG_OK;
}

// ---- bump-and-revalue on common random numbers

// Compiled sides and device arrays of one bump evaluation, released on every exit.
struct BumpArrays {
    std::vector<mcg_plan*> plans;
    DeviceArray<DevicePlan> dplans;
    DeviceArray<uint32_t> masks;
    DeviceArray<StatRecord> partials, records, pair_partials, pair_records;
    DeviceArray<double> unit_prices;
    DeviceArray<BumpPair> pairs;
    DeviceArray<ErrorWord> errors;
    ~BumpArrays() {
        for (mcg_plan* p : plans) delete p;
        dplans.release();
        masks.release();
        for (auto* a : {&partials, &records, &pair_partials, &pair_records}) a->release();
        unit_prices.release();
        pairs.release();
        errors.release();
    }
};

// One scenario: the input a request moves and the half-width
// (Scenario, crates/pricing/src/engine/risk/bump.rs:35-44).
struct BumpScenario {
    int target;  // 0 spot, 1 volatility
    double amount;
};

// paired(), bump.rs:556-566: the mean of the ordered per-unit differences and
// the standard error of that mean.
mcg_status bump_paired(const HostStat& h, double& value, double& se) {
    if (h.count < 2) return fail(MCG_ERR_INVALID_ARGUMENT, "a paired standard error needs at least two sampling units");
    const double n = static_cast<double>(h.count);
    value = h.total() / n;
    se = std::sqrt(h.m2 / (n - 1.0) / n);
    return MCG_OK;
}

mcg_status bump_evaluate(const mcg_plan_desc* d, const mcg_bump_request* req, uint32_t count, cudaStream_t stream,
                         mcg_bump_estimate* est, mcg_bump_report* rep) {
    if (!d || !req || !est) return fail(MCG_ERR_INVALID_ARGUMENT, "null descriptor, requests or estimates");
    if (rep) std::memset(rep, 0, sizeof(*rep));
    if (count == 0 || count > 64) return fail(MCG_ERR_INVALID_ARGUMENT, "request_count must be 1..64");
    if (d->product_count != 1 || d->request_delta || d->request_gamma || d->request_vega ||
        d->request_local_vega_nodes)
        return fail(MCG_ERR_UNSUPPORTED, "a bump plan's base is one product, price only");
    if (d->discrete_dividends.count)
        return fail(MCG_ERR_UNSUPPORTED, "a bump plan's base has no discrete dividends");
    if (d->precision != MCG_PRECISION_F64) return fail(MCG_ERR_UNSUPPORTED, "a bump plan runs in FP64");
    // The distinct scenarios in first-use order (PricingSource::scenarios,
    // bump.rs:446-462): Delta and Gamma of one size share a pair.
    std::vector<BumpScenario> sc;
    std::vector<uint32_t> sc_of(count);
    bool gamma = false;
    for (uint32_t i = 0; i < count; ++i) {
        const mcg_bump_request& q = req[i];
        if (q.measure < MCG_BUMP_SPOT_DELTA || q.measure > MCG_BUMP_VOLATILITY_VEGA)
            return fail(MCG_ERR_INVALID_ARGUMENT, "request " + std::to_string(i) + ": unknown measure");
        if (!(q.size > 0.0) || !std::isfinite(q.size))
            return fail(MCG_ERR_INVALID_ARGUMENT, "request " + std::to_string(i) + ": bump_size must be positive");
        const int target = q.measure == MCG_BUMP_VOLATILITY_VEGA ? 1 : 0;
        if (target == 1 && d->model != MCG_MODEL_BLACK_SCHOLES)
            return fail(MCG_ERR_INVALID_ARGUMENT,
                        "a volatility bump needs a constant-volatility (Black-Scholes) model");
        const double level = target == 0 ? d->spot : d->volatility;
        const double amount = q.relative ? q.size * level : q.size;  // BumpSize::amount, api/measure.rs:429-436
        uint32_t j = 0;
        while (j < sc.size() && !(sc[j].target == target && sc[j].amount == amount)) ++j;
        if (j == sc.size()) sc.push_back({target, amount});
        sc_of[i] = j;
        gamma |= q.measure == MCG_BUMP_SPOT_GAMMA;
    }
    // Sides: scenario j up at 2j, down at 2j + 1; the base plan last (Gamma).
    const uint32_t ns = static_cast<uint32_t>(sc.size());
    const uint32_t sides = 2 * ns + (gamma ? 1u : 0u);
    const uint32_t base_side = 2 * ns;
    BumpArrays A;
    std::vector<DevicePlan> dp(sides);
    std::vector<uint32_t> masks(sides);
    for (uint32_t k = 0; k < sides; ++k) {
        mcg_plan_desc s = *d;
        if (k < base_side) {
            const BumpScenario& c = sc[k / 2];
            const double sign = (k % 2 == 0) ? 1.0 : -1.0;
            if (c.target == 0) {
                s.spot = d->spot + sign * c.amount;
                if (!(s.spot > 0.0) || !std::isfinite(s.spot))
                    return fail(MCG_ERR_INVALID_ARGUMENT, "bumped_spot must stay positive");
            } else {
                s.volatility = d->volatility + sign * c.amount;
                if (!(s.volatility > 0.0) || !std::isfinite(s.volatility))
                    return fail(MCG_ERR_INVALID_ARGUMENT, "the bumped volatility must stay positive");
            }
        }
        auto* plan = new (std::nothrow) mcg_plan();
        if (!plan) return fail(MCG_ERR_ALLOCATION, "plan allocation");
        A.plans.push_back(plan);
        const mcg_status st = build(&s, *plan, false);
        if (st != MCG_OK) return fail(st, "side " + std::to_string(k) + ": " + g_last_error);
        dp[k] = plan->dp;
        masks[k] = plan->mask;
    }
    const mcg_plan& first = *A.plans[0];
    const DevicePlan& P0 = first.dp;
    const bool lv = P0.model == MCG_MODEL_LOCAL_VOLATILITY;
    const bool rqmc = P0.engine == MCG_ENGINE_RQMC;
    const uint64_t units = P0.units;
    const uint32_t scrambles = P0.scramble_count;
    const uint32_t tiles = first.tiles;
    ScenarioLaunch L{};
    L.sides = sides;
    L.scrambles = scrambles;
    L.tiles = tiles;
    L.path = lv ? kBookLocalVol : (first.single_terminal ? kBookBsTerminal : kBookBsPath);
    L.evolutions = P0.antithetic ? 2 : 1;
    L.units = units;
    L.max_nodes = lv ? P0.nx : 0u;
    L.max_slots = lv ? std::max(P0.slot_count, 1u) : 0u;
    const size_t smem = scenario_smem_bytes(L.max_nodes, L.max_slots);
    if (smem > 200 * 1024) return fail(MCG_ERR_UNSUPPORTED, "bump plan grid too large for shared memory");
    if (!rqmc && static_cast<double>(sides) * static_cast<double>(units) * 8.0 > 8.0e9)
        return fail(MCG_ERR_UNSUPPORTED, "bump plan unit prices exceed 8 GB (sides x sampling units)");
    MCG_CUDA(A.dplans.upload(dp));
    MCG_CUDA(A.masks.upload(masks));
    MCG_CUDA(A.partials.alloc(static_cast<size_t>(sides) * scrambles * tiles * kComponents));
    MCG_CUDA(A.records.alloc(static_cast<size_t>(sides) * scrambles * kComponents));
    MCG_CUDA(A.errors.alloc(sides));
    std::vector<BumpPair> pairs(count);
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t j = sc_of[i];
        pairs[i] = BumpPair{2 * j, 2 * j + 1, base_side, req[i].measure == MCG_BUMP_SPOT_GAMMA ? 1 : 0,
                            sc[j].amount};
    }
    if (!rqmc) {
        MCG_CUDA(A.unit_prices.alloc(static_cast<size_t>(sides) * units));
        MCG_CUDA(A.pairs.upload(pairs));
        MCG_CUDA(A.pair_partials.alloc(static_cast<size_t>(count) * tiles));
        MCG_CUDA(A.pair_records.alloc(count));
    }
    L.plans = A.dplans.ptr;
    L.masks = A.masks.ptr;
    L.partials = A.partials.ptr;
    L.unit_prices = rqmc ? nullptr : A.unit_prices.ptr;
    L.errors = A.errors.ptr;
    cudaEvent_t t0, t1;
    MCG_CUDA(cudaEventCreate(&t0));
    MCG_CUDA(cudaEventCreate(&t1));
    MCG_CUDA(cudaMemsetAsync(A.errors.ptr, 0xff, sides * sizeof(ErrorWord), stream));
    MCG_CUDA(cudaEventRecord(t0, stream));
    uint32_t launches = 0;
    cudaError_t e = launch_scenarios(L, smem, stream);
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("scenario kernel: ") + cudaGetErrorString(e));
    ++launches;
    reduce_tiles_kernel<<<dim3(1, sides * scrambles), 256, 0, stream>>>(A.partials.ptr, tiles, kComponents,
                                                                       A.records.ptr);
    MCG_CUDA(cudaGetLastError());
    ++launches;
    if (!rqmc) {
        e = launch_bump_pairs(A.unit_prices.ptr, units, A.pairs.ptr, count, A.pair_partials.ptr, stream);
        if (e != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("pair kernel: ") + cudaGetErrorString(e));
        reduce_tiles_kernel<<<dim3(1, count), 256, 0, stream>>>(A.pair_partials.ptr, tiles, 1, A.pair_records.ptr);
        MCG_CUDA(cudaGetLastError());
        launches += 2;
    }
    MCG_CUDA(cudaEventRecord(t1, stream));
    std::vector<StatRecord> rec(static_cast<size_t>(sides) * scrambles * kComponents), prec(rqmc ? 0 : count);
    std::vector<ErrorWord> ew(sides);
    MCG_CUDA(cudaMemcpyAsync(rec.data(), A.records.ptr, rec.size() * sizeof(StatRecord), cudaMemcpyDeviceToHost,
                             stream));
    if (!rqmc)
        MCG_CUDA(cudaMemcpyAsync(prec.data(), A.pair_records.ptr, prec.size() * sizeof(StatRecord),
                                 cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaMemcpyAsync(ew.data(), A.errors.ptr, sides * sizeof(ErrorWord), cudaMemcpyDeviceToHost, stream));
    MCG_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    for (uint32_t k = 0; k < sides; ++k)
        if (ew[k].key != ~0ull) {
            if (rep) {
                rep->error.code = static_cast<int32_t>(ew[k].key & 0xff);
                rep->error.step = k;
                rep->error.sampling_unit = ew[k].key >> 8;
            }
            return fail(static_cast<mcg_status>(ew[k].key & 0xff),
                        "side " + std::to_string(k) + ": sampling unit " + std::to_string(ew[k].key >> 8) + " failed");
        }
    // Each side's price (its own plan's estimate) and, for RQMC, its scramble means.
    std::vector<mcg_estimate> price(sides);
    std::vector<std::vector<double>> reps(sides);
    for (uint32_t k = 0; k < sides; ++k) {
        HostStat h;
        if (!rqmc) {
            const StatRecord& x = rec[static_cast<size_t>(k) * kComponents];
            h = {x.sum, x.corr, static_cast<uint64_t>(x.count), x.mean, x.m2};
            price[k] = make_estimate(h, units, 1.0);
        } else {
            reps[k].resize(scrambles);
            for (uint32_t s = 0; s < scrambles; ++s) {
                const StatRecord& x = rec[(static_cast<size_t>(k) * scrambles + s) * kComponents];
                reps[k][s] = (x.sum + x.corr) / static_cast<double>(units);
            }
            h = two_pass(reps[k]);
            price[k] = make_estimate(h, scrambles, 1.0);
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        const BumpPair& pr = pairs[i];
        HostStat h;
        if (!rqmc) {
            const StatRecord& x = prec[i];
            h = {x.sum, x.corr, static_cast<uint64_t>(x.count), x.mean, x.m2};
        } else {
            std::vector<double> diff(scrambles);
            for (uint32_t s = 0; s < scrambles; ++s) {
                const double up = reps[pr.up][s], down = reps[pr.down][s];
                diff[s] = pr.second ? ((up - reps[pr.base][s]) + (down - reps[pr.base][s])) / (pr.h * pr.h)
                                    : (up - down) / (2.0 * pr.h);
            }
            h = two_pass(diff);
        }
        double value = 0.0, se = 0.0;
        const mcg_status st = bump_paired(h, value, se);
        if (st != MCG_OK) return st;
        if (!std::isfinite(value) || !std::isfinite(se))
            return fail(MCG_ERR_INVALID_ARGUMENT, "the bump is too small or too large for a finite difference");
        est[i] = mcg_bump_estimate{req[i].measure, sc_of[i], pr.h, value, se, h.count, price[pr.up].value,
                                   price[pr.down].value};
    }
    if (rep) {
        rep->scenarios = ns;
        rep->sides = sides;
        rep->evaluations = 2ull * ns + (gamma ? 1u : 0u);
        if (gamma) rep->base_price = price[base_side];
        const uint64_t steps = lv ? P0.steps : (first.single_terminal ? 1u : P0.observation_count);
        rep->path_steps = static_cast<uint64_t>(sides) * units * scrambles * steps * (P0.antithetic ? 2u : 1u);
        rep->kernel_launches = launches;
        rep->device_ms = ms;
    }
    return MCG_OK;
}

}  // namespace

extern "C" {

uint32_t mcg_abi_version(void) { return MCG_ABI_VERSION; }

const char* mcg_last_error(void) { return g_last_error.c_str(); }

mcg_status mcg_plan_create(const mcg_plan_desc* desc, mcg_plan** out_plan) {
    if (!out_plan) return fail(MCG_ERR_INVALID_ARGUMENT, "null out_plan");
    *out_plan = nullptr;
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
        return fail(MCG_ERR_CUDA, "no CUDA device is visible");
    auto* plan = new (std::nothrow) mcg_plan();
    if (!plan) return fail(MCG_ERR_ALLOCATION, "plan allocation");
    const mcg_status st = build(desc, *plan);
    if (st != MCG_OK) {
        delete plan;
        return st;
    }
    *out_plan = plan;
    return MCG_OK;
}

mcg_status mcg_plan_evaluate(mcg_plan* plan, void* stream, mcg_result* result) {
    return evaluate(plan, static_cast<cudaStream_t>(stream), result);
}

void mcg_plan_destroy(mcg_plan* plan) { delete plan; }

mcg_status mcg_lsm_price(const mcg_plan_desc* plan, const mcg_lsm_desc* lsm, void* stream,
                         mcg_lsm_result* result) {
    return lsm_price(plan, lsm, static_cast<cudaStream_t>(stream), result);
}

mcg_status mcg_lsm_dual(const mcg_plan_desc* plan, const mcg_lsm_desc* lsm, const mcg_dual_desc* dual,
                        void* stream, mcg_dual_result* result) {
    return lsm_dual(plan, lsm, dual, static_cast<cudaStream_t>(stream), result);
}

mcg_status mcg_book_create(const mcg_plan_desc* trades, uint32_t trade_count, const mcg_book_options* options,
                           mcg_book** out_book) {
    return book_create(trades, trade_count, options, out_book);
}

mcg_status mcg_book_evaluate(mcg_book* book, void* stream, mcg_estimate* prices, mcg_book_report* report) {
    return book_evaluate(book, static_cast<cudaStream_t>(stream), prices, report);
}

void mcg_book_destroy(mcg_book* book) { delete book; }

mcg_status mcg_mlp_forward(const float* params, const float* x, uint32_t count, float* out) {
    if (!params || !x || !out || count == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "mcg_mlp_forward arguments");
    DeviceArray<float> p, dx, dout;
    cudaError_t e = p.upload(std::vector<float>(params, params + kMlpParams));
    if (e == cudaSuccess) e = dx.upload(std::vector<float>(x, x + 2 * static_cast<size_t>(count)));
    if (e == cudaSuccess) e = dout.alloc(count);
    if (e == cudaSuccess) e = launch_mlp_forward(p.ptr, dx.ptr, count, dout.ptr, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(out, dout.ptr, count * sizeof(float), cudaMemcpyDeviceToHost);
    p.release();
    dx.release();
    dout.release();
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("mcg_mlp_forward: ") + cudaGetErrorString(e));
    return MCG_OK;
}

mcg_status mcg_mlp_gradient(const float* params, const float* x, const float* y, const uint8_t* mask,
                            uint32_t count, float* grad, float* loss) {
    if (!params || !x || !y || !mask || !grad || !loss || count == 0)
        return fail(MCG_ERR_INVALID_ARGUMENT, "mcg_mlp_gradient arguments");
    DeviceArray<float> p, dx, dy, partials, sums;
    DeviceArray<uint8_t> dm;
    const unsigned ctas = mlp_gradient_ctas(count);
    cudaError_t e = p.upload(std::vector<float>(params, params + kMlpParams));
    if (e == cudaSuccess) e = dx.upload(std::vector<float>(x, x + 2 * static_cast<size_t>(count)));
    if (e == cudaSuccess) e = dy.upload(std::vector<float>(y, y + count));
    if (e == cudaSuccess) e = dm.upload(std::vector<uint8_t>(mask, mask + count));
    if (e == cudaSuccess) e = partials.alloc(static_cast<size_t>(ctas) * kMlpPartial);
    if (e == cudaSuccess) e = sums.alloc(kMlpPartial);
    if (e == cudaSuccess) {
        MlpRows rows{};
        rows.count = count;
        rows.x = dx.ptr;
        rows.y = dy.ptr;
        rows.mask = dm.ptr;
        e = launch_mlp_gradient(p.ptr, rows, partials.ptr, ctas, nullptr);
    }
    if (e == cudaSuccess) e = launch_mlp_sum(partials.ptr, ctas, sums.ptr, nullptr);
    std::vector<float> host(kMlpPartial);
    if (e == cudaSuccess) e = cudaMemcpy(host.data(), sums.ptr, kMlpPartial * sizeof(float), cudaMemcpyDeviceToHost);
    p.release();
    dx.release();
    dy.release();
    partials.release();
    sums.release();
    dm.release();
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("mcg_mlp_gradient: ") + cudaGetErrorString(e));
    std::memcpy(grad, host.data(), kMlpParams * sizeof(float));
    *loss = host[kMlpParams];
    return MCG_OK;
}

mcg_status mcg_price(const mcg_plan_desc* desc, void* stream, mcg_result* result) {
    mcg_plan* plan = nullptr;
    mcg_status st = mcg_plan_create(desc, &plan);
    if (st != MCG_OK) return st;
    st = mcg_plan_evaluate(plan, stream, result);
    mcg_plan_destroy(plan);
    return st;
}

mcg_status mcg_plan_shape(const mcg_plan* plan, uint32_t* time_steps, uint32_t* effective_dimension,
                          uint32_t* grid_value_count) {
    if (!plan) return fail(MCG_ERR_INVALID_ARGUMENT, "null plan");
    if (time_steps) *time_steps = plan->dp.steps;
    if (effective_dimension) *effective_dimension = plan->dp.dimension;
    if (grid_value_count) *grid_value_count = plan->grid_values;
    return MCG_OK;
}

mcg_status mcg_philox_normals(uint64_t master_seed, uint64_t first_unit, uint64_t count, uint32_t dimensions,
                              uint32_t domain, double* out_host) {
    if (!out_host || count == 0 || dimensions == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "empty request");
    double* dev = nullptr;
    MCG_CUDA(cudaMalloc(&dev, count * dimensions * sizeof(double)));
    philox_normals_kernel<<<static_cast<unsigned>((count + 127) / 128), 128>>>(master_seed, first_unit, count,
                                                                              dimensions, domain, dev);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out_host, dev, count * dimensions * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dev);
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
    return MCG_OK;
}

mcg_status mcg_rqmc_words(const uint32_t* directions, uint32_t dimensions, uint64_t master_seed, uint32_t scramble,
                          uint64_t first_point, uint64_t count, uint32_t* out_host) {
    if (!directions || !out_host || count == 0 || dimensions == 0)
        return fail(MCG_ERR_INVALID_ARGUMENT, "empty request");
    if (first_point + count > (1ull << 32))
        return fail(MCG_ERR_INVALID_ARGUMENT, "Sobol point index beyond 2^32");
    uint32_t *dirs = nullptr, *table = nullptr, *shifts = nullptr, *out = nullptr, *low = nullptr;
    const uint32_t scrambles = scramble + 1;
    // Aligned requests go through the path kernels' warp-cooperative form.
    const bool warp = (first_point & 31u) == 0 && (count & 31u) == 0;
    MCG_CUDA(cudaMalloc(&dirs, static_cast<size_t>(dimensions) * 32 * 4));
    MCG_CUDA(cudaMalloc(&table, static_cast<size_t>(scrambles) * dimensions * 32 * 4));
    MCG_CUDA(cudaMalloc(&shifts, static_cast<size_t>(scrambles) * dimensions * 4));
    MCG_CUDA(cudaMalloc(&out, count * dimensions * 4));
    if (warp) MCG_CUDA(cudaMalloc(&low, static_cast<size_t>(scrambles) * dimensions * 32 * 4));
    cudaError_t e = cudaMemcpy(dirs, directions, static_cast<size_t>(dimensions) * 32 * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const uint32_t total = scrambles * dimensions;
        scramble_table_kernel<<<(total + 127) / 128, 128>>>(dirs, dimensions, scrambles, 0u, master_seed, table,
                                                           shifts);
        if (warp) {
            scramble_low_kernel<<<(total * 32u + 127) / 128, 128>>>(table, total, low);
            rqmc_words_warp_kernel<<<static_cast<unsigned>((count + 127) / 128), 128>>>(
                table, shifts, low, dimensions, scramble, first_point, count, out);
        } else {
            rqmc_words_kernel<<<static_cast<unsigned>((count + 127) / 128), 128>>>(table, shifts, dimensions,
                                                                                  scramble, first_point, count, out);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out_host, out, count * dimensions * 4, cudaMemcpyDeviceToHost);
    cudaFree(dirs);
    cudaFree(table);
    cudaFree(shifts);
    cudaFree(out);
    if (low) cudaFree(low);
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
    return MCG_OK;
}

mcg_status mcg_multi_asset_price(const mcg_multi_asset_desc* desc, void* stream, mcg_multi_asset_result* result) {
    return multi_asset_price(desc, static_cast<cudaStream_t>(stream), result);
}

mcg_status mcg_bump_evaluate(const mcg_plan_desc* base, const mcg_bump_request* requests, uint32_t request_count,
                             void* stream, mcg_bump_estimate* estimates, mcg_bump_report* report) {
    return bump_evaluate(base, requests, request_count, static_cast<cudaStream_t>(stream), estimates, report);
}

}  // extern "C"

namespace {

// SurfaceValidationTolerance::local_vol_vegakt_v1 (crates/pricing/src/market/ssvi.rs:30-58).
double tol_effective(double l, double r) { return std::max(1.0e-14, 1.0e-12 * std::max({1.0, std::fabs(l), std::fabs(r)})); }
bool permits_non_strict(double l, double r) { return l - r <= tol_effective(l, r); }
bool permits_strict(double l, double r) { return r - l > tol_effective(l, r); }

// PCHIP knot derivatives (ThetaPchip, crates/pricing/src/market/pchip.rs:178-237).
std::vector<double> pchip_knot_derivatives(const double* t, const double* v, uint32_t n) {
    std::vector<double> h(n - 1), sl(n - 1), dv(n, 0.0);
    for (uint32_t i = 0; i + 1 < n; ++i) {
        h[i] = t[i + 1] - t[i];
        sl[i] = (v[i + 1] - v[i]) / h[i];
    }
    auto sg = [](double x) { return std::signbit(x) ? -1.0 : 1.0; };
    auto endpoint = [&](double aw, double nw, double as, double ns) {
        double dd = ((2.0 * aw + nw) * as - aw * ns) / (aw + nw);
        if (sg(dd) != sg(as)) dd = 0.0;
        else if (sg(as) != sg(ns) && std::fabs(dd) > 3.0 * std::fabs(as)) dd = 3.0 * as;
        return dd;
    };
    if (n == 2) {
        dv[0] = dv[1] = sl[0];
        return dv;
    }
    dv[0] = endpoint(h[0], h[1], sl[0], sl[1]);
    for (uint32_t i = 1; i + 1 < n; ++i) {
        const double l = sl[i - 1], r = sl[i];
        if (l == 0.0 || r == 0.0 || sg(l) != sg(r)) {
            dv[i] = 0.0;
        } else {
            const double w1 = 2.0 * h[i] + h[i - 1];
            const double w2 = h[i] + 2.0 * h[i - 1];
            dv[i] = (w1 + w2) / (w1 / l + w2 / r);
        }
    }
    dv[n - 1] = endpoint(h[n - 2], h[n - 3], sl[n - 2], sl[n - 3]);
    return dv;
}

// Host phi(theta) for the SSVI admissibility checks (PhiSpec::evaluate, ssvi.rs:121-176).
void host_phi(const mcg_surface_desc& d, double theta, double& phi, double& dphi) {
    if (d.kind == MCG_SURFACE_SSVI_POWER_LAW) {
        phi = d.eta / (std::pow(theta, d.gamma) * std::pow(1.0 + theta, 1.0 - d.gamma));
        dphi = -phi * (d.gamma / theta + (1.0 - d.gamma) / (1.0 + theta));
        return;
    }
    const double z = d.lambda * theta;
    if (std::fabs(z) <= 1.0e-4) {
        phi = 0.5 + z * (-1.0 / 6.0 +
                         z * (1.0 / 24.0 + z * (-1.0 / 120.0 + z * (1.0 / 720.0 + z * (-1.0 / 5040.0 + z / 40320.0)))));
        dphi = d.lambda *
               (-1.0 / 6.0 + z * (1.0 / 12.0 + z * (-1.0 / 40.0 + z * (1.0 / 180.0 + z * (-1.0 / 1008.0 + z / 6720.0)))));
        return;
    }
    const double e = std::exp(-z);
    phi = (z - 1.0 + e) / (z * z);
    dphi = d.lambda * (2.0 - z - (z + 2.0) * e) / (z * z * z);
}

bool all_finite(const double* x, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i])) return false;
    return true;
}

// The surface constructors' checks: ThetaPchip::new (pchip.rs:27-90),
// StandardSsvi::new with PhiSpec::validate and validate_butterfly_bounds
// (ssvi.rs:77-118,347-388,501-525), EssviSlice::new / EssviSurface::new /
// validate_slice (essvi.rs:14-172,262-297).
std::string validate_surface(const mcg_surface_desc& d) {
    if (!std::isfinite(d.terminal_theta_slope) || d.terminal_theta_slope < 0.0) return "terminal_theta_slope";
    if (d.kind == MCG_SURFACE_ESSVI) {
        const uint32_t n = d.slice_count;
        if (n < 2 || !d.slice_times || !d.slice_thetas || !d.slice_psis || !d.slice_rho_psis)
            return "eSSVI needs at least two slices";
        for (uint32_t i = 0; i < n; ++i) {
            const double t = d.slice_times[i], th = d.slice_thetas[i], ps = d.slice_psis[i], rp = d.slice_rho_psis[i];
            if (!std::isfinite(t) || !std::isfinite(th) || !std::isfinite(ps) || !std::isfinite(rp))
                return "eSSVI slice " + std::to_string(i) + " is not finite";
            if (t <= 0.0 || th <= 0.0 || ps <= 0.0) return "eSSVI slice " + std::to_string(i) + " time/theta/psi";
            const double rho = rp / ps;
            if (!std::isfinite(rho) || std::fabs(rho) >= 1.0) return "eSSVI slice " + std::to_string(i) + " rho";
            const double wing = ps * (1.0 + std::fabs(rho));
            if (!std::isfinite(wing) || !permits_strict(wing, 4.0))
                return "eSSVI slice " + std::to_string(i) + " strict_wing_slope";
            const double curvature = ps * ps * (1.0 + std::fabs(rho));
            const double limit = 4.0 * th;
            if (!std::isfinite(curvature) || !std::isfinite(limit) || !permits_non_strict(curvature, limit))
                return "eSSVI slice " + std::to_string(i) + " curvature_bound";
        }
        for (uint32_t i = 0; i + 1 < n; ++i) {
            if (d.slice_times[i + 1] <= d.slice_times[i]) return "eSSVI slices unsorted";
            if (d.slice_thetas[i + 1] < d.slice_thetas[i]) return "eSSVI theta_non_decreasing";
            if (d.slice_psis[i + 1] < d.slice_psis[i]) return "eSSVI psi_non_decreasing";
            const double change = std::fabs(d.slice_rho_psis[i + 1] - d.slice_rho_psis[i]);
            if (!permits_non_strict(change, d.slice_psis[i + 1] - d.slice_psis[i])) return "eSSVI rho_psi_change_bound";
        }
        return "";
    }
    if (d.kind != MCG_SURFACE_SSVI_POWER_LAW && d.kind != MCG_SURFACE_SSVI_HESTON_LIKE) return "surface kind";
    const uint32_t n = d.theta_count;
    if (n < 2 || !d.theta_times || !d.theta_values) return "theta curve needs at least two knots";
    for (uint32_t i = 0; i < n; ++i) {
        if (!std::isfinite(d.theta_times[i]) || d.theta_times[i] <= 0.0) return "theta knot time";
        if (!std::isfinite(d.theta_values[i]) || d.theta_values[i] <= 0.0) return "theta value";
        if (i && d.theta_times[i] <= d.theta_times[i - 1]) return "theta knots unsorted";
        if (i && d.theta_values[i] < d.theta_values[i - 1]) return "theta decreasing";
    }
    if (!std::isfinite(d.rho) || std::fabs(d.rho) >= 1.0) return "rho";
    if (d.kind == MCG_SURFACE_SSVI_POWER_LAW) {
        if (!std::isfinite(d.eta) || d.eta <= 0.0) return "eta";
        if (!std::isfinite(d.gamma) || !(d.gamma > 0.0 && d.gamma < 1.0)) return "gamma";
        if (!permits_non_strict(d.gamma, 0.5)) return "power_law_gamma_at_most_one_half";
        const double wing = d.eta * (1.0 + std::fabs(d.rho));
        if (!std::isfinite(wing) || !permits_non_strict(wing, 2.0)) return "power_law_eta_wing_bound";
    } else {
        if (!std::isfinite(d.lambda) || d.lambda <= 0.0) return "lambda";
        if (!permits_non_strict((1.0 + std::fabs(d.rho)) / 4.0, d.lambda)) return "heston_like_lambda_lower_bound";
    }
    for (uint32_t i = 0; i < n; ++i) {
        const double theta = d.theta_values[i];
        double phi, dphi;
        host_phi(d, theta, phi, dphi);
        if (!std::isfinite(phi) || phi <= 0.0 || !std::isfinite(dphi)) return "phi";
        const double cf = 1.0 + std::fabs(d.rho);
        const double wing = theta * phi * cf;
        if (!std::isfinite(wing) || !permits_strict(wing, 4.0)) return "strict_wing_slope";
        const double curvature = theta * phi * phi * cf;
        if (!std::isfinite(curvature) || !permits_non_strict(curvature, 4.0)) return "curvature_bound";
        if (dphi >= 0.0) return "phi_strictly_decreasing";
        const double skew = phi + theta * dphi;
        if (skew < -tol_effective(skew, 0.0)) return "theta_phi_non_decreasing";
    }
    return "";
}

// A device array released when it leaves scope.
template <class T>
struct ScopedArray : DeviceArray<T> {
    ~ScopedArray() { this->release(); }
};

// Device copies of a validated surface.
struct DeviceSurface {
    Surface s{};
    DeviceArray<double> t, v, d, st, sth, sps, srp;
    ~DeviceSurface() {
        t.release();
        v.release();
        d.release();
        st.release();
        sth.release();
        sps.release();
        srp.release();
    }
};

mcg_status load_surface(const mcg_surface_desc* desc, DeviceSurface& out) {
    if (!desc) return fail(MCG_ERR_INVALID_ARGUMENT, "null surface");
    const std::string why = validate_surface(*desc);
    if (!why.empty()) return fail(MCG_ERR_MARKET, "surface: " + why);
    Surface& s = out.s;
    s.kind = desc->kind;
    s.slope = desc->terminal_theta_slope;
    s.rho = desc->rho;
    s.eta = desc->eta;
    s.gamma = desc->gamma;
    s.lambda = desc->lambda;
    if (desc->kind == MCG_SURFACE_ESSVI) {
        const uint32_t n = desc->slice_count;
        MCG_CUDA(out.st.upload(std::vector<double>(desc->slice_times, desc->slice_times + n)));
        MCG_CUDA(out.sth.upload(std::vector<double>(desc->slice_thetas, desc->slice_thetas + n)));
        MCG_CUDA(out.sps.upload(std::vector<double>(desc->slice_psis, desc->slice_psis + n)));
        MCG_CUDA(out.srp.upload(std::vector<double>(desc->slice_rho_psis, desc->slice_rho_psis + n)));
        s.st = out.st.ptr;
        s.stheta = out.sth.ptr;
        s.spsi = out.sps.ptr;
        s.srho_psi = out.srp.ptr;
        s.slices = n;
    } else {
        const uint32_t n = desc->theta_count;
        MCG_CUDA(out.t.upload(std::vector<double>(desc->theta_times, desc->theta_times + n)));
        MCG_CUDA(out.v.upload(std::vector<double>(desc->theta_values, desc->theta_values + n)));
        MCG_CUDA(out.d.upload(pchip_knot_derivatives(desc->theta_times, desc->theta_values, n)));
        s.t = out.t.ptr;
        s.v = out.v.ptr;
        s.d = out.d.ptr;
        s.n = n;
    }
    return MCG_OK;
}

mcg_status surface_grid(const mcg_surface_desc* desc, const double* time_nodes, uint32_t time_count,
                        const double* log_moneyness_nodes, uint32_t log_moneyness_count, double floor, double cap,
                        double* values, uint32_t* repairs) {
    if (!time_nodes || time_count < 2 || !log_moneyness_nodes || log_moneyness_count < 2 || !values)
        return fail(MCG_ERR_INVALID_ARGUMENT, "grid inputs");
    if (!all_finite(time_nodes, time_count) || !all_finite(log_moneyness_nodes, log_moneyness_count))
        return fail(MCG_ERR_MARKET, "grid nodes must be finite");
    for (uint32_t i = 0; i < time_count; ++i)
        if (time_nodes[i] < 0.0 || (i && !(time_nodes[i] > time_nodes[i - 1])))
            return fail(MCG_ERR_MARKET, "grid time nodes must be non-negative and increasing");
    for (uint32_t j = 1; j < log_moneyness_count; ++j)
        if (!(log_moneyness_nodes[j] > log_moneyness_nodes[j - 1]))
            return fail(MCG_ERR_MARKET, "log-moneyness nodes must be increasing");
    if (!(floor > 0.0) || !(cap > floor) || !std::isfinite(cap)) return fail(MCG_ERR_MARKET, "floor/cap");
    DeviceSurface S;
    mcg_status st = load_surface(desc, S);
    if (st != MCG_OK) return st;
    const size_t nv = static_cast<size_t>(time_count) * log_moneyness_count;
    ScopedArray<double> tn, xn, out;
    ScopedArray<uint32_t> counters;
    MCG_CUDA(tn.upload(std::vector<double>(time_nodes, time_nodes + time_count)));
    MCG_CUDA(xn.upload(std::vector<double>(log_moneyness_nodes, log_moneyness_nodes + log_moneyness_count)));
    MCG_CUDA(out.alloc(nv));
    MCG_CUDA(counters.upload(std::vector<uint32_t>(2, 0u)));
    cudaError_t e = launch_surface_grid(S.s, tn.ptr, time_count, xn.ptr, log_moneyness_count, floor, cap, out.ptr,
                                        counters.ptr, 0);
    uint32_t host_counters[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(values, out.ptr, nv * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(host_counters, counters.ptr, 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
    if (repairs) *repairs = host_counters[0];
    if (host_counters[1]) return fail(MCG_ERR_MARKET, "surface has a non-positive variance or density");
    return MCG_OK;
}

}  // namespace

extern "C" {

mcg_status mcg_ssvi_local_variance_grid(const double* theta_times, const double* theta_values, uint32_t theta_count,
                                        double terminal_slope, double rho, double eta, double gamma,
                                        const double* time_nodes, uint32_t time_count,
                                        const double* log_moneyness_nodes, uint32_t log_moneyness_count,
                                        double floor, double cap, double* values, uint32_t* repairs) {
    mcg_surface_desc d{};
    d.kind = MCG_SURFACE_SSVI_POWER_LAW;
    d.theta_times = theta_times;
    d.theta_values = theta_values;
    d.theta_count = theta_count;
    d.terminal_theta_slope = terminal_slope;
    d.rho = rho;
    d.eta = eta;
    d.gamma = gamma;
    return surface_grid(&d, time_nodes, time_count, log_moneyness_nodes, log_moneyness_count, floor, cap, values,
                        repairs);
}

mcg_status mcg_surface_local_variance_grid(const mcg_surface_desc* surface, const double* time_nodes,
                                           uint32_t time_count, const double* log_moneyness_nodes,
                                           uint32_t log_moneyness_count, double floor, double cap, double* values,
                                           uint32_t* repairs) {
    return surface_grid(surface, time_nodes, time_count, log_moneyness_nodes, log_moneyness_count, floor, cap,
                        values, repairs);
}

mcg_status mcg_surface_total_variance(const mcg_surface_desc* surface, const double* times,
                                      const double* log_moneyness, uint32_t count, double* out) {
    if (!times || !log_moneyness || !out || count == 0) return fail(MCG_ERR_INVALID_ARGUMENT, "surface points");
    for (uint32_t i = 0; i < count; ++i)
        if (!std::isfinite(times[i]) || times[i] <= 0.0 || !std::isfinite(log_moneyness[i]))
            return fail(MCG_ERR_INVALID_ARGUMENT, "surface query point " + std::to_string(i));
    DeviceSurface S;
    mcg_status st = load_surface(surface, S);
    if (st != MCG_OK) return st;
    ScopedArray<double> t, k, o;
    ScopedArray<uint32_t> failures;
    MCG_CUDA(t.upload(std::vector<double>(times, times + count)));
    MCG_CUDA(k.upload(std::vector<double>(log_moneyness, log_moneyness + count)));
    MCG_CUDA(o.alloc(4 * static_cast<size_t>(count)));
    MCG_CUDA(failures.upload(std::vector<uint32_t>(1, 0u)));
    cudaError_t e = launch_surface_eval(S.s, t.ptr, k.ptr, count, o.ptr, failures.ptr, 0);
    uint32_t bad = 0;
    if (e == cudaSuccess) e = cudaMemcpy(out, o.ptr, 4 * static_cast<size_t>(count) * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&bad, failures.ptr, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
    if (bad) return fail(MCG_ERR_MARKET, "surface has a non-finite or non-positive total variance");
    return MCG_OK;
}

mcg_status mcg_measure_fp64_peak(void* stream, double* tflops) {
    if (!tflops) return fail(MCG_ERR_INVALID_ARGUMENT, "null output");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 0;
    MCG_CUDA(cudaGetDevice(&device));
    MCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    double* sink = nullptr;
    MCG_CUDA(cudaMalloc(&sink, 1024 * sizeof(double)));
    const int iterations = 4096, threads = 256, blocks = sms * 8;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fp64_peak_kernel<<<blocks, threads, 0, st>>>(sink, 16);  // warm-up
    cudaEventRecord(a, st);
    fp64_peak_kernel<<<blocks, threads, 0, st>>>(sink, iterations);
    cudaEventRecord(b, st);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return fail(MCG_ERR_CUDA, cudaGetErrorString(e));
    const double flops = 2.0 * 8.0 * 16.0 * iterations * static_cast<double>(threads) * blocks;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return MCG_OK;
}

}  // extern "C"

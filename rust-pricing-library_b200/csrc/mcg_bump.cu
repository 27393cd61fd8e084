// mcg_bump.cu -- bump-and-revalue scenario sides priced in one launch.
//
// The reference prices each side of a scenario as its own task on the base
// task's seeds and pairs the sides' recorded sampling units
// (CompiledScenarios::evaluate, crates/pricing/src/engine/risk/bump.rs:626-690;
// units_from_recorded, :490-523).  Here every side is a compiled plan staged
// per CTA from a device array, and one grid of (tile, scramble, side) CTAs runs
// the single-plan tile functions (mcg_bs_tile.cuh, mcg_lv_tile.cuh) on all of
// them: each side's tile records are those of evaluating its plan alone, and
// pseudo-MC sides also leave each unit's discounted price, which
// bump_pair_kernel differences unit by unit into CTA statistics records.
//
// Compiled with -fmad=false like the path kernels it shares code with.
#include "mcg_bs_tile.cuh"
#include "mcg_bump.cuh"
#include "mcg_lv_tile.cuh"

namespace mcg {
namespace {

__host__ __device__ constexpr size_t align16(size_t n) { return (n + 15) & ~size_t(15); }

template <int PATH, int E>
__global__ void __launch_bounds__(kThreads) scenario_kernel(const ScenarioLaunch L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DevicePlan& P = *reinterpret_cast<DevicePlan*>(smem_raw);
    double2* s_b = reinterpret_cast<double2*>(smem_raw + align16(sizeof(DevicePlan)));  // cell bounds
    double* s_w = reinterpret_cast<double*>(s_b + L.max_nodes);
    Stat* s_red = reinterpret_cast<Stat*>(s_w + static_cast<size_t>(L.max_slots) * kThreads);
    const uint32_t tile = blockIdx.x, scramble = blockIdx.y, side = blockIdx.z;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(L.plans + side);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&P);
    for (uint32_t i = threadIdx.x; i < sizeof(DevicePlan) / 4; i += kThreads) dst[i] = src[i];
    __syncthreads();
    const uint64_t point = static_cast<uint64_t>(tile) * kThreads + threadIdx.x;
    const bool valid = point < P.units;
    StatRecord* out =
        L.partials + ((static_cast<size_t>(side) * L.scrambles + scramble) * L.tiles + tile) * kComponents;
    double* unit_price = L.unit_prices ? L.unit_prices + static_cast<size_t>(side) * L.units : nullptr;
    const uint32_t mask = L.masks[side];
    ErrorWord* err = L.errors + side;
    if constexpr (PATH == kBookLocalVol) {
        const int nx = static_cast<int>(P.nx);
        for (int i = threadIdx.x; i + 1 < nx; i += kThreads) s_b[i] = make_double2(P.grid_x[i], P.grid_x[i + 1]);
        __syncthreads();
        const GridView g{nullptr, nullptr, nullptr, nx, s_b, P.grid_cells, P.grid_x[0], P.grid_x[nx - 1]};
        lv_tile<E, 1>(P, g, s_w, s_red, scramble, point, valid, out, mask, err, 0, false, nullptr, nullptr, false,
                      nullptr, unit_price);
    } else if constexpr (PATH == kBookBsTerminal) {
        bs_terminal_tile<false>(P, s_red, scramble, point, valid, out, mask, unit_price);
    } else {
        if (P.antithetic)
            bs_path_tile<1, 2>(P, s_red, scramble, point, valid, out, mask, err, 0, unit_price);
        else
            bs_path_tile<1, 1>(P, s_red, scramble, point, valid, out, mask, err, 0, unit_price);
    }
}

// Paired differences of pseudo-MC unit prices, bump.rs:648-671: one CTA per
// (tile, pair), its statistics record at partials[pair * tiles + tile].
__global__ void __launch_bounds__(kThreads) bump_pair_kernel(const double* __restrict__ prices, uint64_t units,
                                                             const BumpPair* __restrict__ pairs,
                                                             StatRecord* partials) {
    __shared__ Stat s_red[4];
    const BumpPair pr = pairs[blockIdx.y];
    const uint64_t u = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = u < units;
    double d = 0.0;
    if (valid) {
        const double up = prices[static_cast<size_t>(pr.up) * units + u];
        const double down = prices[static_cast<size_t>(pr.down) * units + u];
        if (pr.second) {
            const double b = prices[static_cast<size_t>(pr.base) * units + u];
            d = ((up - b) + (down - b)) / (pr.h * pr.h);
        } else {
            d = (up - down) / (2.0 * pr.h);
        }
    }
    const double vals[1] = {d};
    cta_reduce_write<1>(vals, valid, 1u, partials + static_cast<size_t>(blockIdx.y) * gridDim.x + blockIdx.x, s_red);
}

}  // namespace

size_t scenario_smem_bytes(uint32_t max_nodes, uint32_t max_slots) {
    return align16(sizeof(DevicePlan)) + static_cast<size_t>(max_nodes) * sizeof(double2) +
           static_cast<size_t>(max_slots) * kThreads * sizeof(double) + 4 * kComponents * sizeof(Stat);
}

cudaError_t launch_scenarios(const ScenarioLaunch& L, size_t smem, cudaStream_t stream) {
    const dim3 grid(L.tiles, L.scrambles, L.sides);
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<grid, kThreads, smem, stream>>>(L);
        return cudaGetLastError();
    };
    if (L.path == kBookLocalVol) {
        if (L.evolutions == 2) return go(scenario_kernel<kBookLocalVol, 2>);
        return go(scenario_kernel<kBookLocalVol, 1>);
    }
    if (L.path == kBookBsTerminal) return go(scenario_kernel<kBookBsTerminal, 1>);
    return go(scenario_kernel<kBookBsPath, 1>);
}

cudaError_t launch_bump_pairs(const double* unit_prices, uint64_t units, const BumpPair* pairs, uint32_t pair_count,
                              StatRecord* partials, cudaStream_t stream) {
    const dim3 grid(static_cast<unsigned>((units + kThreads - 1) / kThreads), pair_count);
    bump_pair_kernel<<<grid, kThreads, 0, stream>>>(unit_prices, units, pairs, partials);
    return cudaGetLastError();
}

}  // namespace mcg

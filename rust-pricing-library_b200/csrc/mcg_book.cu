// mcg_book.cu -- a book of trades priced in one persistent launch.
//
// No counterpart in the reference, which prices one plan per call
// (SimulationPlan::execute, crates/pricing/src/engine/risk/valuation.rs:19-33).
// Every trade is a compiled single-product plan (its own model, surface,
// maturity, step count and product); the kernel runs the very per-tile path
// evaluation of the single-plan kernels (mcg_bs_tile.cuh, mcg_lv_tile.cuh),
// so each trade's statistics are bit for bit those of evaluating its plan
// alone.
//
// Scheduling: a fixed grid of CTAs (a multiple of the SM count, chosen with
// the tiles per work item by the host's autotuner) pulls work items from a
// queue ordered heaviest first (longest-processing-time first: step count x
// tiles), one atomicAdd per item and no waiting.  An item stages its trade's
// plan (and the cell bounds of its local-variance grid) into shared memory and
// evaluates its tiles;
// tile records land at the trade's tile positions, so the reduction that
// follows is the single-plan one.
//
// Compiled with -fmad=false like the path kernels it shares code with.
#include "mcg_book.cuh"
#include "mcg_bs_tile.cuh"
#include "mcg_lv_tile.cuh"

namespace mcg {
namespace {

__host__ __device__ constexpr size_t align16(size_t n) { return (n + 15) & ~size_t(15); }

__global__ void __launch_bounds__(kThreads) book_kernel(const BookLaunch L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t s_item;
    DevicePlan& P = *reinterpret_cast<DevicePlan*>(smem_raw);
    double2* s_b = reinterpret_cast<double2*>(smem_raw + align16(sizeof(DevicePlan)));  // cell bounds
    double* s_w = reinterpret_cast<double*>(s_b + L.max_nodes);
    Stat* s_red = reinterpret_cast<Stat*>(s_w + static_cast<size_t>(L.max_slots) * kThreads);
    for (;;) {
        __syncthreads();  // the previous item is done with the shared plan and grid
        if (threadIdx.x == 0) s_item = atomicAdd(L.next, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= L.item_count) return;
        const BookItem item = L.items[it];
        const uint32_t* src = reinterpret_cast<const uint32_t*>(L.plans + item.trade);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&P);
        for (uint32_t i = threadIdx.x; i < sizeof(DevicePlan) / 4; i += kThreads) dst[i] = src[i];
        __syncthreads();
        const int nx = static_cast<int>(P.nx);
        if (item.path == kBookLocalVol) {
            for (int i = threadIdx.x; i + 1 < nx; i += kThreads) s_b[i] = make_double2(P.grid_x[i], P.grid_x[i + 1]);
            __syncthreads();
        }
        // The grid's cell records are read through L1, the cell bounds from shared memory.
        const GridView g{nullptr, nullptr, nullptr, nx, s_b, P.grid_cells,
                         item.path == kBookLocalVol ? P.grid_x[0] : 0.0,
                         item.path == kBookLocalVol ? P.grid_x[nx - 1] : 0.0};
        const uint32_t mask = L.masks[item.trade];
        ErrorWord* err = L.errors + item.trade;
        for (uint32_t t = 0; t < item.tiles; ++t) {
            const uint32_t tile = item.first_tile + t;
            const uint64_t point = static_cast<uint64_t>(tile) * kThreads + threadIdx.x;
            const bool valid = point < P.units;
            StatRecord* out = L.partials + (static_cast<size_t>(item.trade) * L.tiles_per_trade + tile) * kComponents;
            if (item.path == kBookLocalVol)
                lv_tile<1, 1>(P, g, s_w, s_red, 0, point, valid, out, mask, err, 0);
            else if (item.path == kBookBsTerminal)
                bs_terminal_tile<false>(P, s_red, 0, point, valid, out, mask);
            else
                bs_path_tile<1>(P, s_red, 0, point, valid, out, mask, err, 0);
        }
    }
}

}  // namespace

size_t book_smem_bytes(uint32_t max_values, uint32_t max_nodes, uint32_t max_slots) {
    (void)max_values;  // the grid values are read through L1
    return align16(sizeof(DevicePlan)) + static_cast<size_t>(max_nodes) * sizeof(double2) +
           static_cast<size_t>(max_slots) * kThreads * sizeof(double) + 4 * kComponents * sizeof(Stat);
}

cudaError_t book_prepare(size_t smem) {
    return cudaFuncSetAttribute(book_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
}

cudaError_t book_occupancy(size_t smem, int* ctas_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, book_kernel, kThreads, smem);
}

cudaError_t launch_book(const BookLaunch& L, unsigned ctas, size_t smem, cudaStream_t stream) {
    book_kernel<<<ctas, kThreads, smem, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace mcg

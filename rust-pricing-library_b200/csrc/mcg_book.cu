// mcg_book.cu -- a book of trades priced by one persistent launch per family.
//
// No counterpart in the reference, which prices one plan per call
// (SimulationPlan::execute, crates/pricing/src/engine/risk/valuation.rs:19-33).
// Every trade is a compiled single-product plan (its own model, surface,
// maturity, step count and product); the kernels run the very per-tile path
// evaluation of the single-plan kernels (mcg_bs_tile.cuh, mcg_lv_tile.cuh), in
// the same specialisation the single-plan launch picks for that trade (batched
// normals included), so each trade's statistics are bit for bit those of
// evaluating its plan alone.
//
// Families: the trades are split by path kind, and each family has its own
// persistent kernel, specialised and register-budgeted for it -- local
// volatility with discrete products runs two paths per thread with batched
// normals (5 CTAs of 128 per SM), local volatility with a continuous barrier
// one path per thread with the bridge state, Black-Scholes single-terminal and
// multi-observation paths their own tile functions.  A family kernel keeps a
// fixed grid of CTAs (its occupancy x the SM count) that pulls work items from
// the family's queue, ordered heaviest first (longest-processing-time first:
// step count x tiles), one atomicAdd per item and no waiting.  An item stages
// its trade's plan (and the cell bounds of its local-variance grid) into shared
// memory and evaluates its tiles; tile records land at the trade's tile
// positions, so the reduction that follows is the single-plan one.
//
// Compiled with -fmad=false like the path kernels it shares code with.
#include "mcg_book.cuh"
#include "mcg_bs_tile.cuh"
#include "mcg_lv_tile.cuh"

namespace mcg {
namespace {

__host__ __device__ constexpr size_t align16(size_t n) { return (n + 15) & ~size_t(15); }

__host__ __device__ constexpr int family_paths(uint32_t f) { return f == kFamilyLvDiscrete ? 2 : 1; }
__host__ __device__ constexpr bool family_lv(uint32_t f) { return f == kFamilyLvDiscrete || f == kFamilyLvBarrier; }

// Dynamic shared memory of a family kernel, one layout for the kernel and the
// host's size: the staged plan, then (local volatility only) the cell bounds,
// the bridge slots, the batched normals and their tail lists, then the CTA
// reduction scratch.  Byte offsets.
struct BookSmem {
    size_t bounds, slots, normals, lists, reduce, total;
};

__host__ __device__ inline BookSmem book_smem(uint32_t family, uint32_t max_nodes, uint32_t max_slots) {
    BookSmem m{};
    const size_t q = static_cast<size_t>(family_paths(family));
    const size_t zb = static_cast<size_t>(family_paths(family) == 2 ? z_batch<2>() : z_batch<1>());
    size_t at = align16(sizeof(DevicePlan));
    if (family_lv(family)) {
        m.bounds = at;
        at += static_cast<size_t>(max_nodes) * sizeof(double2);
        m.slots = at;
        at += q * max_slots * kThreads * sizeof(double);
    }
    if (family_lv(family) || family == kFamilyBsPath) {
        m.normals = at;
        at += zb * q * kThreads * sizeof(double);
        m.lists = at;
        at += align16((kThreads / 32) * 32 * zb * q * sizeof(uint16_t));
    }
    m.reduce = at;
    at += 4 * kComponents * sizeof(Stat);
    m.total = at;
    return m;
}

// 5 CTAs per SM for the path families (the Black--Scholes path family took
// 673 ms of the 4096-trade book at 4 CTAs and 128 registers, 613 ms at 5).
template <int F>
__global__ void __launch_bounds__(kThreads, family_lv(F) ? 5 : (F == kFamilyBsPath ? 5 : 1))
    book_kernel(const BookLaunch L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t s_item;
    constexpr int Q = family_paths(F);
    const BookSmem m = book_smem(F, L.max_nodes, L.max_slots);
    DevicePlan& P = *reinterpret_cast<DevicePlan*>(smem_raw);
    double2* s_b = reinterpret_cast<double2*>(smem_raw + m.bounds);      // cell bounds
    double* s_w = reinterpret_cast<double*>(smem_raw + m.slots);         // bridge slots
    double* s_z = reinterpret_cast<double*>(smem_raw + m.normals);       // batched normals
    uint16_t* s_zlist = reinterpret_cast<uint16_t*>(smem_raw + m.lists);  // tail lists
    Stat* s_red = reinterpret_cast<Stat*>(smem_raw + m.reduce);
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
        StatRecord* base = L.partials + static_cast<size_t>(item.trade) * L.tiles_per_trade * kComponents;
        const uint32_t mask = L.masks[item.trade];
        ErrorWord* err = L.errors + item.trade;
        if constexpr (family_lv(F)) {
            const int nx = static_cast<int>(P.nx);
            for (int i = threadIdx.x; i + 1 < nx; i += kThreads) s_b[i] = make_double2(P.grid_x[i], P.grid_x[i + 1]);
            __syncthreads();
            // The grid's cell records are read through L1, the cell bounds from shared memory.
            const GridView g{nullptr, nullptr, nullptr, nx, s_b, P.grid_cells, P.grid_x[0], P.grid_x[nx - 1]};
            for (uint32_t t = 0; t < item.tiles; t += Q) {
                const uint32_t tile = item.first_tile + t;
                const uint64_t point = static_cast<uint64_t>(tile) * kThreads + threadIdx.x;
                if constexpr (Q == 2) {
                    // tiles `tile` and `tile + 1`, as the single-plan two-path kernel pairs them
                    StatRecord* second =
                        tile + 1 < L.tiles_per_trade ? base + static_cast<size_t>(tile + 1) * kComponents : nullptr;
                    lv_tile<1, 1, 0, 0, 2>(P, g, s_w, s_red, 0, point, point < P.units,
                                           base + static_cast<size_t>(tile) * kComponents, mask, err, 0, true, s_z,
                                           s_zlist, point + kThreads < P.units, second);
                } else {
                    lv_tile<1, 1, 0, 1, 1>(P, g, s_w, s_red, 0, point, point < P.units,
                                           base + static_cast<size_t>(tile) * kComponents, mask, err, 0, true, s_z,
                                           s_zlist);
                }
            }
        } else {
            for (uint32_t t = 0; t < item.tiles; ++t) {
                const uint32_t tile = item.first_tile + t;
                const uint64_t point = static_cast<uint64_t>(tile) * kThreads + threadIdx.x;
                StatRecord* out = base + static_cast<size_t>(tile) * kComponents;
                if constexpr (F == kFamilyBsTerminal)
                    bs_terminal_tile<false>(P, s_red, 0, point, point < P.units, out, mask);
                else if (P.antithetic)
                    bs_path_tile<1, 2>(P, s_red, 0, point, point < P.units, out, mask, err, 0, nullptr, s_z, s_zlist);
                else
                    bs_path_tile<1, 1>(P, s_red, 0, point, point < P.units, out, mask, err, 0, nullptr, s_z, s_zlist);
            }
        }
    }
}

template <class Fn>
cudaError_t with_kernel(uint32_t family, Fn fn) {
    switch (family) {
        case kFamilyLvDiscrete: return fn(book_kernel<kFamilyLvDiscrete>);
        case kFamilyLvBarrier: return fn(book_kernel<kFamilyLvBarrier>);
        case kFamilyBsTerminal: return fn(book_kernel<kFamilyBsTerminal>);
        default: return fn(book_kernel<kFamilyBsPath>);
    }
}

}  // namespace

size_t book_smem_bytes(uint32_t family, uint32_t max_nodes, uint32_t max_slots) {
    return book_smem(family, max_nodes, max_slots).total;
}

cudaError_t book_prepare(uint32_t family, size_t smem) {
    return with_kernel(family, [&](auto kernel) {
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    });
}

cudaError_t book_occupancy(uint32_t family, size_t smem, int* ctas_per_sm) {
    return with_kernel(family, [&](auto kernel) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, kernel, kThreads, smem);
    });
}

cudaError_t launch_book(uint32_t family, const BookLaunch& L, unsigned ctas, size_t smem, cudaStream_t stream) {
    return with_kernel(family, [&](auto kernel) {
        kernel<<<ctas, kThreads, smem, stream>>>(L);
        return cudaGetLastError();
    });
}

}  // namespace mcg

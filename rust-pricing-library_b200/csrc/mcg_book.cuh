// mcg_book.cuh -- the batched book: work items and launch interface shared by
// the persistent kernels (mcg_book.cu) and the host orchestration (mcg_host.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mcg_plan.h"

namespace mcg {

struct ErrorWord;

// Path evaluation of one trade (also the scenario kernels' path kind).
enum BookPath : uint32_t { kBookLocalVol = 0, kBookBsTerminal = 1, kBookBsPath = 2 };

// Families of trades, each priced by its own persistent kernel specialised on
// it: local volatility with discrete products (two paths per thread, batched
// normals), local volatility with a continuous barrier (one path per thread,
// batched normals, the bridge state), Black-Scholes single-terminal and
// Black-Scholes multi-observation paths.
enum BookFamily : uint32_t {
    kFamilyLvDiscrete = 0,
    kFamilyLvBarrier = 1,
    kFamilyBsTerminal = 2,
    kFamilyBsPath = 3,
    kBookFamilies = 4
};

// One unit of work: `tiles` consecutive 128-unit tiles of one trade (an even
// number, from an even first tile, in the two-path family).
struct BookItem {
    uint32_t trade;
    uint32_t first_tile;
    uint32_t tiles;
    uint32_t path;  // BookPath
};

struct BookLaunch {
    const DevicePlan* plans;   // [trades]
    const uint32_t* masks;     // [trades] statistics components each trade reduces
    const BookItem* items;     // [items] of this family, heaviest first
    uint32_t item_count;
    unsigned int* next;        // this family's work-queue cursor, zero before the launch
    StatRecord* partials;      // [trades][tiles][kComponents]
    uint32_t tiles_per_trade;
    ErrorWord* errors;         // [trades]
    uint32_t max_nodes, max_slots;  // shared-memory extents over the family's trades
};

size_t book_smem_bytes(uint32_t family, uint32_t max_nodes, uint32_t max_slots);
cudaError_t book_prepare(uint32_t family, size_t smem);
cudaError_t book_occupancy(uint32_t family, size_t smem, int* ctas_per_sm);
cudaError_t launch_book(uint32_t family, const BookLaunch& L, unsigned ctas, size_t smem, cudaStream_t stream);

}  // namespace mcg

// mcg_book.cuh -- the batched book: work items and launch interface shared by
// the persistent kernel (mcg_book.cu) and the host orchestration (mcg_host.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mcg_plan.h"

namespace mcg {

struct ErrorWord;

// Path evaluation of one trade.
enum BookPath : uint32_t { kBookLocalVol = 0, kBookBsTerminal = 1, kBookBsPath = 2 };

// One unit of work: `tiles` consecutive 128-unit tiles of one trade.
struct BookItem {
    uint32_t trade;
    uint32_t first_tile;
    uint32_t tiles;
    uint32_t path;  // BookPath
};

struct BookLaunch {
    const DevicePlan* plans;   // [trades]
    const uint32_t* masks;     // [trades] statistics components each trade reduces
    const BookItem* items;     // [items], heaviest first
    uint32_t item_count;
    unsigned int* next;        // work-queue cursor, zero before the launch
    StatRecord* partials;      // [trades][tiles][kComponents]
    uint32_t tiles_per_trade;
    ErrorWord* errors;         // [trades]
    uint32_t max_values, max_nodes, max_slots;  // shared-memory extents over the book
};

size_t book_smem_bytes(uint32_t max_values, uint32_t max_nodes, uint32_t max_slots);
cudaError_t book_prepare(size_t smem);
cudaError_t book_occupancy(size_t smem, int* ctas_per_sm);
cudaError_t launch_book(const BookLaunch& L, unsigned ctas, size_t smem, cudaStream_t stream);

}  // namespace mcg

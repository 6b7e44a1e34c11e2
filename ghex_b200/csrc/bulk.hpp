// Bulk column kernel (bulk.cu): unstructured index-list columns whose levels are contiguous and
// 16-byte aligned (list descriptors in 16-byte units) moved by the asynchronous copy engine: a CTA
// of one warp loads its tile's columns into shared memory with cp.async.bulk (completion counted on
// an mbarrier) and stores them to their destination columns with cp.async.bulk. No element passes
// through registers, and the small CTAs keep many tiles' bytes in flight per SM.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ghexb
{
constexpr int k_bulk_columns = 64;     // columns per tile at most (the index block's size)
constexpr int k_bulk_stage = 16384;    // bytes of columns per tile at most (the CTA's shared stage)
constexpr int k_bulk_block_ints = 2 * k_bulk_columns;

// A tile: ncols columns of col_bytes (a multiple of 16, at most k_bulk_stage) each; column c moves
// from src + sidx[c] * s_is to dst + didx[c] * d_is, its indices in the tile's index block
// (k_bulk_block_ints ints: the source indices, then the destination indices).
struct alignas(16) btile
{
    const char* src;
    char* dst;
    int64_t s_is, d_is; // bytes per index step
    uint32_t ncols, col_bytes;
    uint32_t pad[2];
};
static_assert(sizeof(btile) == 48, "btile is three 16-byte words");

// One CTA of 32 threads per tile. `status` (nullptr: none) gets bit 0 when a wait for a tile's
// loads gave up (its columns are then not stored).
cudaError_t launch_bulk(const btile* tiles, const int32_t* blocks, int ntiles, unsigned* status, cudaStream_t stream);
} // namespace ghexb

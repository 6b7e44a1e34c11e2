// Bulk column kernel (bulk.cu): unstructured index-list columns whose levels are contiguous and
// 16-byte aligned (list descriptors in 16-byte units) moved by the asynchronous copy engine: a CTA
// of one warp loads its tile's columns into shared memory with cp.async.bulk (completion counted on
// an mbarrier) and stores them to their destination columns with cp.async.bulk. No element passes
// through registers, and the small CTAs keep many tiles' bytes in flight per SM.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ghexb
{
constexpr int k_bulk_columns = 64;     // columns per tile at most (the index block's size)
constexpr int k_bulk_stage = 16384;    // bytes of columns per tile at most (the CTA's shared stage)
constexpr int k_bulk_block_ints = 2 * k_bulk_columns;

// A tile: ncols columns of col_bytes (a multiple of 16, at most k_bulk_stage) each; column c moves
// from src + sidx[c] * s_is to dst + didx[c] * d_is, its indices in the tile's index block
// (k_bulk_block_ints ints: the source indices, then the destination indices). With smap and dmap
// >= 0 the columns move four at a time: the source and destination fields are 2-D tensor maps
// (a row per index, the column's levels in a row, boxes one row high) read with tile::gather4
// and written with tile::scatter4 at the columns' indices; a group of fewer than four columns
// repeats its last column, which moves the same bytes to the same place again.
struct alignas(16) btile
{
    const char* src;
    char* dst;
    int64_t s_is, d_is; // bytes per index step
    uint32_t ncols, col_bytes;
    int32_t smap, dmap; // tensor maps of the source and destination fields, or -1
};
static_assert(sizeof(btile) == 48, "btile is three 16-byte words");

// One CTA of 32 threads per tile; `maps` holds the tiles' tensor maps (nullptr when no tile has
// any). `status` (nullptr: none) gets bit 0 when a wait for a tile's loads gave up (its columns
// are then not stored).
cudaError_t launch_bulk(const btile* tiles, const int32_t* blocks, const CUtensorMap* maps, int ntiles, unsigned* status,
    cudaStream_t stream);

// Adjoint of unstructured columns in bulk form: a tile of nown owner columns, each with nimg image
// columns, all of col_bytes (a multiple of 16, at most k_bgather_zero) with their levels
// contiguous. The CTA loads every column into shared memory, adds each owner's images into it in
// order (acc = own; acc = acc + image_i), and stores the owner columns back and zeros into the
// image columns, all by the copy engine. Its index block holds the columns' addresses, per owner
// the owner's then its images' (k_bgather_entries at most). `status` gets bit 2 when a wait for a
// tile's loads gave up (nothing of the tile is then stored).
constexpr int k_bgather_entries = 96;
constexpr int k_bgather_zero = 2048;
struct alignas(16) bgtile
{
    uint32_t nown, nimg, col_bytes, levels;
    uint32_t esize;
    uint32_t pad[3];
};
static_assert(sizeof(bgtile) == 32, "bgtile is two 16-byte words");
cudaError_t launch_bulk_gather(const bgtile* tiles, const uint64_t* blocks, int ntiles, unsigned* status,
    cudaStream_t stream);
} // namespace ghexb

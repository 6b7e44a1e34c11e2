// Host launchers of the forward exchange and box adjoint kernels (exchange.cu).
#pragma once

#include <cuda_runtime.h>

#include "descriptors.hpp"

namespace ghexb
{
constexpr int k_max_block = 512;
// Threads per CTA of the gather kernel.
constexpr int k_gather_block = 256;

// Elements a thread moves in a forward tile of `unit`-byte elements when the kernel runs with
// K elements per thread (16-byte units take half: their registers are twice as wide).
__host__ __device__ constexpr int forward_per_thread(int k, int unit)
{
    return unit == 16 ? (k > 1 ? k / 2 : 1) : k;
}

// Elements per thread of a gather tile whose cell has `nimg` images: about sixteen loads in
// flight per thread (the owner and its images of every element).
__host__ __device__ constexpr int gather_per_thread(int nimg)
{
    return nimg <= 1 ? 8 : nimg <= 3 ? 4 : 2;
}

// Element classes: each runs its own specialised loop in the kernels.
enum forward_class : int32_t
{
    k_box8 = 0,
    k_box8_neg,
    k_box4,
    k_box4_neg,
    k_box2,
    k_box1,
    k_list16,
    k_list8,
    k_list4,
    k_list2,
    k_list1,
    k_pair8,
    k_pair4,
    k_forward_classes
};
__host__ __device__ constexpr int forward_class_of(int kind, int unit, bool neg)
{
    return kind == 2 ? (unit == 8 ? k_pair8 : k_pair4)
         : kind == 0 ? (unit == 8 ? (neg ? k_box8_neg : k_box8)
                           : unit == 4 ? (neg ? k_box4_neg : k_box4)
                           : unit == 2 ? k_box2
                                       : k_box1)
                     : (unit == 16 ? k_list16 : unit == 8 ? k_list8 : unit == 4 ? k_list4 : unit == 2 ? k_list2 : k_list1);
}
// gather classes: (element size, images)
__host__ __device__ constexpr int gather_class(int esize, int nimg)
{
    return (esize == 8 ? 0 : k_max_images) + (nimg - 1);
}
// classes of unstructured owner groups follow those of box cells
__host__ __device__ constexpr int list_gather_class(int esize, int nimg)
{
    return 2 * k_max_images + gather_class(esize, nimg);
}
constexpr int k_gather_classes = 4 * k_max_images;

// Forward exchange of tiles[0, ntiles), one CTA per tile: a tile holds at most
// forward_per_thread(k, unit) * block elements; k is 4, 8 or 16.
// Index block of a list tile: the source indices of its (at most k_block_columns) columns, then
// their destination indices.
constexpr int k_block_columns = 32;
constexpr int k_block_ints = 2 * k_block_columns;

// `lists` (list_bytes long): the index lists the list tiles read, brought into L2 by the first
// CTAs of the launch; nullptr when there are none. `blocks`: k_block_ints ints per tile, the
// index blocks of the flagged list tiles (xtile pad[0] = 1), or nullptr (the tiles then read
// their indices through sidx / didx).
cudaError_t launch_exchange(const xtile* tiles, int ntiles, int k, int block, cudaStream_t stream,
    const void* lists = nullptr, size_t list_bytes = 0, const int32_t* blocks = nullptr);
// Adjoint in gather form of tiles[0, ntiles), one CTA per tile: a tile holds at most
// gather_per_thread(nimg) * k_gather_block elements. launch_gather takes box cells,
// launch_list_gather unstructured owner groups with `cols`, their column table.
cudaError_t launch_gather(const gtile* tiles, int ntiles, cudaStream_t stream);
// `blocks` (nullptr: none): k_gblock_entries column-table entries per tile, the tile's slice of
// `cols`, loaded by its CTA beside the record; used by the tiles whose record flags it (pad[0]).
constexpr int k_gblock_entries = 96;
cudaError_t launch_list_gather(const gtile* tiles, int ntiles, const uint64_t* cols, const uint64_t* blocks,
    cudaStream_t stream);
} // namespace ghexb

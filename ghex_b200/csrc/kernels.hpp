// Host launchers of the ghex_b200 device kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "descriptors.hpp"

namespace ghexb
{
// Forward exchange over tiles[0, ntiles): box and list descriptors, any element type.
cudaError_t launch_exchange(const box_desc* boxes, const list_desc* lists, const tile* tiles,
    int ntiles, int grid, int block, cudaStream_t stream);

// Adjoint over tiles[0, ntiles) whose owner elements are pairwise distinct:
// owner += halo (owner -= halo for negated components); halo = 0. Float and double only.
cudaError_t launch_adjoint(const box_desc* boxes, const list_desc* lists, const tile* tiles,
    int ntiles, int grid, int block, cudaStream_t stream);

// Reads n16 16-byte words of `buf` so that the L2 holds clean lines of an unrelated buffer;
// `sink` receives a value only when the data sum to a sentinel that a zero-filled buffer never
// produces, which keeps the loads alive.
cudaError_t launch_l2_flush(const uint4* buf, size_t n16, unsigned* sink, int grid, cudaStream_t stream);

constexpr int k_max_block = 512;
} // namespace ghexb

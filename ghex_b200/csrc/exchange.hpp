// Host launchers of the forward exchange and box adjoint kernels (exchange.cu).
#pragma once

#include <cuda_runtime.h>

#include "descriptors.hpp"

namespace ghexb
{
constexpr int k_max_block = 512;
// Elements per thread of a gather tile whose cell has `nimg` images: about sixteen loads in
// flight per thread (the owner and its images of every element).
constexpr int gather_per_thread(int nimg)
{
    return nimg <= 1 ? 8 : nimg <= 3 ? 4 : 2;
}

// Elements a thread moves in a forward tile of `unit`-byte elements when the kernel runs with
// K elements per thread (16-byte units take half: their registers are twice as wide).
constexpr int forward_per_thread(int k, int unit)
{
    return unit == 16 ? (k > 1 ? k / 2 : 1) : k;
}

// One CTA per tile: tiles[blockIdx.x] holds at most forward_per_thread(k, unit) * block elements.
// k is 4, 8 or 16.
cudaError_t launch_exchange(const xtile* tiles, int ntiles, int k, int block, cudaStream_t stream);
// Threads per CTA of the gather kernel.
constexpr int k_gather_block = 256;
// One CTA per tile: tiles[blockIdx.x] holds at most gather_per_thread(nimg) * k_gather_block elements.
cudaError_t launch_gather(const gtile* tiles, int ntiles, cudaStream_t stream);
} // namespace ghexb

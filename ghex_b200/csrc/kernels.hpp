// Host launchers of the phased adjoint kernels and the L2 flush (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "descriptors.hpp"

namespace ghexb
{
// Adjoint over tiles[0, ntiles) whose owner elements are pairwise distinct:
// owner += halo (owner -= halo for negated components); halo = 0. Float and double only.
// CTAs claim tiles through counters[0..1] (zero before the launch, zero again after it);
// launches sharing counters must be ordered on one stream. block <= 512.
cudaError_t launch_box_adjoint(const box_desc* boxes, const tile* tiles, int ntiles, unsigned* counters, int grid,
    int block, cudaStream_t stream);
cudaError_t launch_list_adjoint(const list_desc* lists, const tile* tiles, int ntiles, unsigned* counters, int grid,
    int block, cudaStream_t stream);

// Reads n16 16-byte words of `buf` so that the L2 holds clean lines of an unrelated buffer;
// `sink` receives a value only when the data sum to a sentinel that a zero-filled buffer never
// produces, which keeps the loads alive.
cudaError_t launch_l2_flush(const uint4* buf, size_t n16, unsigned* sink, int grid, cudaStream_t stream);

// Calibration copy of `rows` rows of n elements of es (4 or 8) bytes at the given element strides;
// mode 0 copies, 1 only reads the source rows, 2 only writes the destination rows.
cudaError_t launch_row_copy(const void* src, void* dst, uint32_t rows, uint32_t n, int64_t src_stride,
    int64_t dst_stride, int es, int mode, cudaStream_t stream);
} // namespace ghexb

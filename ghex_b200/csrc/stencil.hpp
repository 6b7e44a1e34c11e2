// The 7-point update of the differentiable-exchange workload (stencil.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ghexb
{
constexpr int k_stencil_batch = 32; // domains per launch

struct stencil_domain
{
    const void* in;
    void* out;
    int32_t ex, ey, ez;      // extents including the halo
    int32_t halo;            // width of the halo on every side
    int64_t sx, sy, sz;      // element strides
};

// Launches the forward update (adjoint == false) or its transpose over n domains of one dtype.
cudaError_t launch_stencil7(bool f64, const stencil_domain* doms, int n, double alpha, bool adjoint, cudaStream_t stream);
} // namespace ghexb

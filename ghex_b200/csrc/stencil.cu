// The 7-point update of the differentiable-exchange workload and its adjoint.
//
// GHEX has no stencil: this is the compute step of the program whose gradient the exchange's
// adjoint is checked in (exchange, then x <- x + alpha * L(x) on the interior, repeated). It is a
// plain memory-bound sweep; its arithmetic is spelled out with round-to-nearest intrinsics in a
// fixed order (no contraction into fused multiply-adds), so that an elementwise CPU restatement
// reproduces it bit for bit:
//
//   forward, interior p:   s  = ((((x[p-ex] + x[p+ex]) + x[p-ey]) + x[p+ey]) + x[p-ez]) + x[p+ez]
//                          y[p] = x[p] + alpha * (s - 6 * x[p])
//   forward, halo p:       y[p] = 0
//   adjoint, every p:      G(q) = gy[q] on the interior, 0 elsewhere (and outside the array)
//                          t  = ((((G(p-ex) + G(p+ex)) + G(p-ey)) + G(p+ey)) + G(p-ez)) + G(p+ez)
//                          gx[p] = G(p) + alpha * (t - 6 * G(p))
#include <cuda_runtime.h>

#include <cstdint>

#include "stencil.hpp"

namespace ghexb
{
namespace
{
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <typename T> __device__ __forceinline__ T sub_rn(T a, T b);
template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

struct domain_args
{
    stencil_domain d[k_stencil_batch];
};

// One thread per element; blockIdx.y selects the domain. x is the fastest index of the thread
// numbering so that neighbouring threads touch neighbouring elements when sx == 1.
template <typename T, bool ADJOINT>
__global__ void __launch_bounds__(256) stencil7_kernel(const __grid_constant__ domain_args args, T alpha)
{
    const stencil_domain& d = args.d[blockIdx.y];
    const int64_t n = (int64_t)d.ex * d.ey * d.ez;
    const T* __restrict__ in = static_cast<const T*>(d.in);
    T* __restrict__ out = static_cast<T*>(d.out);
    const int h = d.halo;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e % d.ex);
        const int64_t r = e / d.ex;
        const int j = (int)(r % d.ey);
        const int k = (int)(r / d.ey);
        const int64_t p = i * d.sx + j * d.sy + k * d.sz;
        const bool interior = i >= h && i < d.ex - h && j >= h && j < d.ey - h && k >= h && k < d.ez - h;
        if constexpr (!ADJOINT)
        {
            T y = T(0);
            if (interior)
            {
                const T x = in[p];
                T s = add_rn(in[p - d.sx], in[p + d.sx]);
                s = add_rn(s, in[p - d.sy]);
                s = add_rn(s, in[p + d.sy]);
                s = add_rn(s, in[p - d.sz]);
                s = add_rn(s, in[p + d.sz]);
                y = add_rn(x, mul_rn(alpha, sub_rn(s, mul_rn(T(6), x))));
            }
            out[p] = y;
        }
        else
        {
            // G(q): the gradient on interior elements, zero on the halo and outside the array
            auto G = [&](int ii, int jj, int kk) -> T {
                const bool in_ = ii >= h && ii < d.ex - h && jj >= h && jj < d.ey - h && kk >= h && kk < d.ez - h;
                return in_ ? in[ii * d.sx + jj * d.sy + kk * d.sz] : T(0);
            };
            const T g = interior ? in[p] : T(0);
            T t = add_rn(G(i - 1, j, k), G(i + 1, j, k));
            t = add_rn(t, G(i, j - 1, k));
            t = add_rn(t, G(i, j + 1, k));
            t = add_rn(t, G(i, j, k - 1));
            t = add_rn(t, G(i, j, k + 1));
            out[p] = add_rn(g, mul_rn(alpha, sub_rn(t, mul_rn(T(6), g))));
        }
    }
}

template <typename T>
cudaError_t launch_t(const stencil_domain* doms, int n, double alpha, bool adjoint, cudaStream_t stream)
{
    for (int b = 0; b < n; b += k_stencil_batch)
    {
        domain_args args{};
        const int m = n - b < k_stencil_batch ? n - b : k_stencil_batch;
        int64_t most = 0;
        for (int i = 0; i < m; ++i)
        {
            args.d[i] = doms[b + i];
            const int64_t e = (int64_t)doms[b + i].ex * doms[b + i].ey * doms[b + i].ez;
            most = e > most ? e : most;
        }
        const int block = 256;
        int64_t gx = (most + block - 1) / block;
        if (gx > 4 * 148 * 8) gx = 4 * 148 * 8; // grid-stride beyond a few waves
        if (gx < 1) gx = 1;
        const dim3 grid((unsigned)gx, (unsigned)m);
        if (adjoint)
            stencil7_kernel<T, true><<<grid, block, 0, stream>>>(args, (T)alpha);
        else
            stencil7_kernel<T, false><<<grid, block, 0, stream>>>(args, (T)alpha);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
} // namespace

cudaError_t launch_stencil7(bool f64, const stencil_domain* doms, int n, double alpha, bool adjoint, cudaStream_t stream)
{
    return f64 ? launch_t<double>(doms, n, alpha, adjoint, stream) : launch_t<float>(doms, n, alpha, adjoint, stream);
}
} // namespace ghexb

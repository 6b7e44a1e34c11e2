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

#include <algorithm>
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

// A block of 32 x 8 threads covers a 32 x 8 patch of (i, j) columns of one domain (blockIdx.z)
// and a slab of k_slab planes; each thread takes one column through the slab. The column's own
// values of planes k0 - 1 .. k0 + k_slab are loaded once into registers (each serves three
// planes), the four in-plane neighbours of every plane come from the caches, where the
// neighbouring threads of the block load them as their own columns. All loads of the slab are
// issued before the first result, so a thread keeps up to 5 * k_slab + 2 loads in flight.
constexpr int k_tile_x = 32, k_tile_y = 8, k_slab = 4;

template <typename T, bool ADJOINT>
__global__ void __launch_bounds__(k_tile_x * k_tile_y) stencil7_kernel(const __grid_constant__ domain_args args, T alpha,
    unsigned nslabs, unsigned nblocks_y)
{
    const stencil_domain& d = args.d[blockIdx.z];
    const int i = blockIdx.x * k_tile_x + threadIdx.x;
    const int h = d.halo, ex = d.ex, ey = d.ey, ez = d.ez;
    const int64_t sx = d.sx, sy = d.sy, sz = d.sz;
    const auto within = [](int v, int lo, int hi) { return v >= lo && v < hi; };
    for (unsigned b = blockIdx.y; b < nblocks_y; b += gridDim.y)
    {
        const unsigned ytile = b / nslabs;
        const int j = (int)(ytile * k_tile_y + threadIdx.y);
        const int k0 = (int)(b - ytile * nslabs) * k_slab;
        if (i >= ex || j >= ey || k0 >= ez) continue;
        const int64_t base = i * sx + j * sy;
        const T* __restrict__ c = static_cast<const T*>(d.in) + base;
        T* __restrict__ o = static_cast<T*>(d.out) + base;
        const bool iin = within(i, h, ex - h), jin = within(j, h, ey - h), col = iin && jin;
        T v[k_slab + 2];     // the column at planes k0 - 1 + q
        T nb[k_slab][4];     // -x, +x, -y, +y neighbours at plane k0 + q
        if constexpr (!ADJOINT)
        {
            // interior planes [h, ez - h) read planes h - 1 .. ez - h of interior columns, all in the array
#pragma unroll
            for (int q = 0; q < k_slab + 2; ++q)
            {
                const int k = k0 - 1 + q;
                v[q] = col && k >= h - 1 && k <= ez - h ? c[k * sz] : T(0);
            }
#pragma unroll
            for (int q = 0; q < k_slab; ++q)
            {
                const int k = k0 + q;
                const bool on = col && within(k, h, ez - h);
                const T* p = c + k * sz;
                nb[q][0] = on ? p[-sx] : T(0);
                nb[q][1] = on ? p[sx] : T(0);
                nb[q][2] = on ? p[-sy] : T(0);
                nb[q][3] = on ? p[sy] : T(0);
            }
#pragma unroll
            for (int q = 0; q < k_slab; ++q)
            {
                const int k = k0 + q;
                T y = T(0);
                if (col && within(k, h, ez - h))
                {
                    const T x = v[q + 1];
                    T s = add_rn(nb[q][0], nb[q][1]);
                    s = add_rn(s, nb[q][2]);
                    s = add_rn(s, nb[q][3]);
                    s = add_rn(s, v[q]);
                    s = add_rn(s, v[q + 2]);
                    y = add_rn(x, mul_rn(alpha, sub_rn(s, mul_rn(T(6), x))));
                }
                if (k < ez) o[k * sz] = y;
            }
        }
        else
        {
            // G(q) = gy[q] on interior elements, 0 elsewhere: a neighbour column is read only where
            // it is interior, so every read is in the array
            const bool mxm = within(i - 1, h, ex - h) && jin, mxp = within(i + 1, h, ex - h) && jin;
            const bool mym = iin && within(j - 1, h, ey - h), myp = iin && within(j + 1, h, ey - h);
#pragma unroll
            for (int q = 0; q < k_slab + 2; ++q)
            {
                const int k = k0 - 1 + q;
                v[q] = col && within(k, h, ez - h) ? c[k * sz] : T(0);
            }
#pragma unroll
            for (int q = 0; q < k_slab; ++q)
            {
                const int k = k0 + q;
                const bool kin = within(k, h, ez - h);
                const T* p = c + k * sz;
                nb[q][0] = mxm && kin ? p[-sx] : T(0);
                nb[q][1] = mxp && kin ? p[sx] : T(0);
                nb[q][2] = mym && kin ? p[-sy] : T(0);
                nb[q][3] = myp && kin ? p[sy] : T(0);
            }
#pragma unroll
            for (int q = 0; q < k_slab; ++q)
            {
                const int k = k0 + q;
                const T g = v[q + 1];
                T t = add_rn(nb[q][0], nb[q][1]);
                t = add_rn(t, nb[q][2]);
                t = add_rn(t, nb[q][3]);
                t = add_rn(t, v[q]);
                t = add_rn(t, v[q + 2]);
                if (k < ez) o[k * sz] = add_rn(g, mul_rn(alpha, sub_rn(t, mul_rn(T(6), g))));
            }
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
        int mx = 0, my = 0, mz = 0;
        for (int i = 0; i < m; ++i)
        {
            args.d[i] = doms[b + i];
            mx = std::max(mx, doms[b + i].ex), my = std::max(my, doms[b + i].ey), mz = std::max(mz, doms[b + i].ez);
        }
        if (mx <= 0 || my <= 0 || mz <= 0) continue;
        const unsigned xtiles = (unsigned)((mx + k_tile_x - 1) / k_tile_x);
        const unsigned nslabs = (unsigned)((mz + k_slab - 1) / k_slab);
        const uint64_t ny = (uint64_t)((my + k_tile_y - 1) / k_tile_y) * nslabs;
        if (ny > 0xffffffffull) return cudaErrorInvalidValue;
        const dim3 grid(xtiles, (unsigned)std::min<uint64_t>(ny, 65535), (unsigned)m);
        const dim3 block(k_tile_x, k_tile_y);
        if (adjoint)
            stencil7_kernel<T, true><<<grid, block, 0, stream>>>(args, (T)alpha, nslabs, (unsigned)ny);
        else
            stencil7_kernel<T, false><<<grid, block, 0, stream>>>(args, (T)alpha, nslabs, (unsigned)ny);
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

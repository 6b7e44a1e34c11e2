// Device kernels of ghex_b200 (sm_100a).
//
// The exchange is pure data movement, so the kernels are built for HBM bandwidth, not for
// the tensor cores:
//  * one persistent launch walks a tile table (tiles are contiguous ranges of one descriptor's
//    flattened index space); tiles of box and list descriptors, of any element size, mix freely;
//  * consecutive threads take consecutive elements along the destination's contiguous
//    dimension, so halo writes are coalesced; every thread keeps ILP independent loads in flight
//    before its stores, which is what keeps enough bytes in flight per SM on HBM3e;
//  * index math is 32-bit with multiply-high divisions by the (invariant) box extents;
//  * unstructured columns move as 16-byte units when every column is 16-byte aligned.
// A halo element moves from the source interior to the destination halo with exactly one read
// and one write: no intermediate message buffer exists.
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace ghexb
{
namespace
{
// loads in flight per thread: 8 for elements up to 8 bytes, 4 for 16-byte units
template<typename T>
struct ilp
{
    static constexpr int value = 4;
};

template<typename T>
__device__ __forceinline__ T xor_bits(T v, uint64_t m)
{
    return v ^ (T)m;
}
template<>
__device__ __forceinline__ uint4 xor_bits<uint4>(uint4 v, uint64_t)
{
    return v;
}

// ---- forward: strided box ---------------------------------------------------------------
template<typename T>
__device__ __noinline__ void box_tile(const box_desc* __restrict__ bd, uint32_t start, uint32_t count)
{
    const T* __restrict__ src = reinterpret_cast<const T*>(bd->src);
    T* __restrict__ dst = reinterpret_cast<T*>(bd->dst);
    const int32_t n0 = bd->n0, n1 = bd->n1, n2 = bd->n2;
    const int32_t s0 = bd->s0, s1 = bd->s1, s2 = bd->s2, s3 = bd->s3;
    const int32_t d0 = bd->d0, d1 = bd->d1, d2 = bd->d2, d3 = bd->d3;
    const fast_div f0 = bd->div0, f1 = bd->div1, f2 = bd->div2;
    const uint64_t xm = bd->xor_mask;
    const uint32_t step = blockDim.x;
    constexpr int k_ilp = ilp<T>::value;
    for (uint32_t base = threadIdx.x; base < count; base += step * k_ilp)
    {
        T v[k_ilp];
        int32_t doff[k_ilp];
#pragma unroll
        for (int k = 0; k < k_ilp; ++k)
        {
            const uint32_t i = base + k * step;
            if (i < count)
            {
                const uint32_t f = start + i;
                const uint32_t q0 = f0.div(f);
                const int32_t i0 = (int32_t)(f - q0 * (uint32_t)n0);
                const uint32_t q1 = f1.div(q0);
                const int32_t i1 = (int32_t)(q0 - q1 * (uint32_t)n1);
                const uint32_t q2 = f2.div(q1);
                const int32_t i2 = (int32_t)(q1 - q2 * (uint32_t)n2);
                const int32_t i3 = (int32_t)q2;
                const int32_t so = i0 * s0 + i1 * s1 + i2 * s2 + i3 * s3;
                doff[k] = i0 * d0 + i1 * d1 + i2 * d2 + i3 * d3;
                v[k] = src[so];
            }
        }
#pragma unroll
        for (int k = 0; k < k_ilp; ++k)
        {
            const uint32_t i = base + k * step;
            if (i < count) dst[doff[k]] = xor_bits(v[k], xm);
        }
    }
}

// ---- forward: index-list columns --------------------------------------------------------
template<typename T>
__device__ __noinline__ void list_tile(const list_desc* __restrict__ ld, uint32_t start, uint32_t count)
{
    const T* __restrict__ src = reinterpret_cast<const T*>(ld->src);
    T* __restrict__ dst = reinterpret_cast<T*>(ld->dst);
    const int32_t* __restrict__ sidx = ld->sidx;
    const int32_t* __restrict__ didx = ld->didx;
    const int32_t L = ld->levels, cnt = ld->count;
    const int32_t s_is = ld->s_is, s_ls = ld->s_ls, d_is = ld->d_is, d_ls = ld->d_ls;
    const bool lf = ld->level_fastest != 0;
    const fast_div fq = ld->divq;
    const uint32_t step = blockDim.x;
    constexpr int k_ilp = ilp<T>::value;
    for (uint32_t base = threadIdx.x; base < count; base += step * k_ilp)
    {
        T v[k_ilp];
        int32_t doff[k_ilp];
#pragma unroll
        for (int k = 0; k < k_ilp; ++k)
        {
            const uint32_t i = base + k * step;
            if (i < count)
            {
                const uint32_t f = start + i;
                const uint32_t q = fq.div(f);
                int32_t col, lev;
                if (lf) col = (int32_t)q, lev = (int32_t)(f - q * (uint32_t)L);
                else
                    lev = (int32_t)q, col = (int32_t)(f - q * (uint32_t)cnt);
                const int32_t so = sidx[col] * s_is + lev * s_ls;
                doff[k] = didx[col] * d_is + lev * d_ls;
                v[k] = src[so];
            }
        }
#pragma unroll
        for (int k = 0; k < k_ilp; ++k)
        {
            const uint32_t i = base + k * step;
            if (i < count) dst[doff[k]] = v[k];
        }
    }
}

__global__ void __launch_bounds__(k_max_block, 2) exchange_kernel(const box_desc* __restrict__ boxes,
    const list_desc* __restrict__ lists, const tile* __restrict__ tiles, int ntiles)
{
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        const tile tl = tiles[t];
        if (tl.kind == 0)
        {
            const box_desc* bd = boxes + tl.desc;
            switch (bd->esize)
            {
                case 8: box_tile<unsigned long long>(bd, tl.start, tl.count); break;
                case 4: box_tile<uint32_t>(bd, tl.start, tl.count); break;
                case 2: box_tile<uint16_t>(bd, tl.start, tl.count); break;
                default: box_tile<uint8_t>(bd, tl.start, tl.count); break;
            }
        }
        else
        {
            const list_desc* ld = lists + tl.desc;
            switch (ld->unit)
            {
                case 16: list_tile<uint4>(ld, tl.start, tl.count); break;
                case 8: list_tile<unsigned long long>(ld, tl.start, tl.count); break;
                case 4: list_tile<uint32_t>(ld, tl.start, tl.count); break;
                case 2: list_tile<uint16_t>(ld, tl.start, tl.count); break;
                default: list_tile<uint8_t>(ld, tl.start, tl.count); break;
            }
        }
    }
}

// ---- adjoint ------------------------------------------------------------------------------
// Within one launch no two elements share an owner, so the read-add-write of the owner needs no
// atomics and the order of additions per owner is the order of the launches.
template<typename F>
__device__ __noinline__ void box_adjoint_tile(const box_desc* __restrict__ bd, uint32_t start, uint32_t count)
{
    F* __restrict__ owner = reinterpret_cast<F*>(const_cast<char*>(bd->src));
    F* __restrict__ halo = reinterpret_cast<F*>(bd->dst);
    const int32_t n0 = bd->n0, n1 = bd->n1, n2 = bd->n2;
    const int32_t s0 = bd->s0, s1 = bd->s1, s2 = bd->s2, s3 = bd->s3;
    const int32_t d0 = bd->d0, d1 = bd->d1, d2 = bd->d2, d3 = bd->d3;
    const fast_div f0 = bd->div0, f1 = bd->div1, f2 = bd->div2;
    const bool neg = bd->xor_mask != 0;
    const uint32_t step = blockDim.x;
    constexpr int k_ilp = 4;
    for (uint32_t base = threadIdx.x; base < count; base += step * k_ilp)
    {
        F h[k_ilp], o[k_ilp];
        int32_t so[k_ilp], doff[k_ilp];
#pragma unroll
        for (int k = 0; k < k_ilp; ++k)
        {
            const uint32_t i = base + k * step;
            if (i < count)
            {
                const uint32_t f = start + i;
                const uint32_t q0 = f0.div(f);
                const int32_t i0 = (int32_t)(f - q0 * (uint32_t)n0);
                const uint32_t q1 = f1.div(q0);
                const int32_t i1 = (int32_t)(q0 - q1 * (uint32_t)n1);
                const uint32_t q2 = f2.div(q1);
                const int32_t i2 = (int32_t)(q1 - q2 * (uint32_t)n2);
                const int32_t i3 = (int32_t)q2;
                so[k] = i0 * s0 + i1 * s1 + i2 * s2 + i3 * s3;
                doff[k] = i0 * d0 + i1 * d1 + i2 * d2 + i3 * d3;
                h[k] = halo[doff[k]];
                o[k] = owner[so[k]];
            }
        }
#pragma unroll
        for (int k = 0; k < k_ilp; ++k)
        {
            const uint32_t i = base + k * step;
            if (i < count)
            {
                owner[so[k]] = neg ? (o[k] - h[k]) : (o[k] + h[k]);
                halo[doff[k]] = F(0);
            }
        }
    }
}

template<typename F>
__device__ __noinline__ void list_adjoint_tile(const list_desc* __restrict__ ld, uint32_t start, uint32_t count)
{
    F* __restrict__ owner = reinterpret_cast<F*>(const_cast<char*>(ld->src));
    F* __restrict__ halo = reinterpret_cast<F*>(ld->dst);
    const int32_t* __restrict__ sidx = ld->sidx;
    const int32_t* __restrict__ didx = ld->didx;
    const int32_t L = ld->levels, cnt = ld->count;
    const int32_t s_is = ld->s_is, s_ls = ld->s_ls, d_is = ld->d_is, d_ls = ld->d_ls;
    const bool lf = ld->level_fastest != 0;
    const fast_div fq = ld->divq;
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x)
    {
        const uint32_t f = start + i;
        const uint32_t q = fq.div(f);
        int32_t col, lev;
        if (lf) col = (int32_t)q, lev = (int32_t)(f - q * (uint32_t)L);
        else
            lev = (int32_t)q, col = (int32_t)(f - q * (uint32_t)cnt);
        const int32_t so = sidx[col] * s_is + lev * s_ls;
        const int32_t doff = didx[col] * d_is + lev * d_ls;
        const F h = halo[doff];
        owner[so] = owner[so] + h;
        halo[doff] = F(0);
    }
}

__global__ void __launch_bounds__(k_max_block, 2) adjoint_kernel(const box_desc* __restrict__ boxes,
    const list_desc* __restrict__ lists, const tile* __restrict__ tiles, int ntiles)
{
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        const tile tl = tiles[t];
        if (tl.kind == 0)
        {
            const box_desc* bd = boxes + tl.desc;
            if (bd->esize == 8) box_adjoint_tile<double>(bd, tl.start, tl.count);
            else
                box_adjoint_tile<float>(bd, tl.start, tl.count);
        }
        else
        {
            const list_desc* ld = lists + tl.desc;
            if (ld->unit == 8) list_adjoint_tile<double>(ld, tl.start, tl.count);
            else
                list_adjoint_tile<float>(ld, tl.start, tl.count);
        }
    }
}
__global__ void __launch_bounds__(256) l2_flush_kernel(const uint4* __restrict__ buf, size_t n16, unsigned* sink)
{
    unsigned acc = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
    {
        const uint4 v = buf[i];
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x9e3779b9u) *sink = acc;
}
} // namespace

cudaError_t launch_l2_flush(const uint4* buf, size_t n16, unsigned* sink, int grid, cudaStream_t stream)
{
    l2_flush_kernel<<<grid, 256, 0, stream>>>(buf, n16, sink);
    return cudaGetLastError();
}

cudaError_t launch_exchange(const box_desc* boxes, const list_desc* lists, const tile* tiles,
    int ntiles, int grid, int block, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    exchange_kernel<<<grid, block, 0, stream>>>(boxes, lists, tiles, ntiles);
    return cudaGetLastError();
}

cudaError_t launch_adjoint(const box_desc* boxes, const list_desc* lists, const tile* tiles,
    int ntiles, int grid, int block, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    adjoint_kernel<<<grid, block, 0, stream>>>(boxes, lists, tiles, ntiles);
    return cudaGetLastError();
}

} // namespace ghexb

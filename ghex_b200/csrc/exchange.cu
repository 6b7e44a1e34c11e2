// Forward exchange and box adjoint kernels (sm_100a).
//
// The exchange is pure data movement, latency-bound at halo sizes: a kernel's time is a few
// dependent memory round trips plus the bytes over HBM bandwidth. The kernels are built for few
// round trips and many bytes in flight:
//  * one CTA per tile, no tile loop: the grid is the tile table, CTAs never wait on each other
//    or on a scheduler, and the hardware block scheduler balances the waves;
//  * a tile record carries everything needed to address its elements (96 bytes forward, 256
//    bytes adjoint), read once by a few threads into shared memory: one round trip before the
//    data loads;
//  * every thread issues all of its K loads before its first store, so K elements per thread
//    are in flight; consecutive threads take consecutive elements, so rows along the
//    destination's contiguous dimension are coalesced;
//  * element coordinates come from two multiply-high divisions per element (fast_div), no
//    per-row bookkeeping, so short rows waste no lanes.
// A halo element moves from the source interior to the destination halo with one read and one
// write; no intermediate buffer exists.
#include <cuda_runtime.h>

#include "exchange.hpp"

namespace ghexb
{
namespace
{
__device__ __forceinline__ uint32_t fdiv(uint32_t n, uint32_t m, uint32_t l)
{
    return (__umulhi(n, m) + n) >> l;
}

template<typename T> struct sign_bit;
template<> struct sign_bit<uint32_t>
{
    static constexpr uint32_t v = 0x80000000u;
};
template<> struct sign_bit<unsigned long long>
{
    static constexpr unsigned long long v = 0x8000000000000000ull;
};

template<typename T> __device__ __forceinline__ T ld_stream(const T* p) { return __ldcg(p); }
template<> __device__ __forceinline__ uint16_t ld_stream(const uint16_t* p) { return __ldcg(reinterpret_cast<const unsigned short*>(p)); }
template<> __device__ __forceinline__ uint8_t ld_stream(const uint8_t* p) { return __ldcg(reinterpret_cast<const unsigned char*>(p)); }

// Loads the record of this CTA into shared memory (W 16-byte words).
template<int W, typename R>
__device__ __forceinline__ void load_record(R& sh, const R* __restrict__ g)
{
    if (threadIdx.x < W)
        reinterpret_cast<uint4*>(&sh)[threadIdx.x] = __ldg(reinterpret_cast<const uint4*>(g) + threadIdx.x);
    __syncthreads();
}

// ---- forward ---------------------------------------------------------------------------------
template<int K, typename T, bool NEG>
__device__ __forceinline__ void box_elements(const xtile& t)
{
    const T* __restrict__ src = reinterpret_cast<const T*>(t.src);
    T* __restrict__ dst = reinterpret_cast<T*>(t.dst);
    T v[K];
    int32_t doff[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        doff[k] = -1;
        if (e < t.count)
        {
            const uint32_t g = t.e0 + e;
            const uint32_t r = fdiv(g, t.m0, t.l0);
            const int32_t i0 = (int32_t)(g - r * t.n0);
            const uint32_t i2 = fdiv(r, t.m1, t.l1);
            const int32_t i1 = (int32_t)(r - i2 * t.n1);
            v[k] = ld_stream(src + (i0 * t.s0 + i1 * t.s1 + (int32_t)i2 * t.s2));
            doff[k] = i0 * t.d0 + i1 * t.d1 + (int32_t)i2 * t.d2;
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (k * blockDim.x + threadIdx.x < t.count)
        {
            if constexpr (NEG) dst[doff[k]] = v[k] ^ sign_bit<T>::v;
            else
                dst[doff[k]] = v[k];
        }
}

template<int K, typename T>
__device__ __forceinline__ void list_elements(const xtile& t)
{
    const T* __restrict__ src = reinterpret_cast<const T*>(t.src);
    T* __restrict__ dst = reinterpret_cast<T*>(t.dst);
    int32_t so[K], doff[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        so[k] = 0;
        doff[k] = 0;
        if (e < t.count)
        {
            const uint32_t g = t.e0 + e;
            const uint32_t col = fdiv(g, t.m0, t.l0);
            const int32_t lev = (int32_t)(g - col * t.n0);
            so[k] = __ldg(t.sidx + col) * t.s0 + lev * t.s1;
            doff[k] = __ldg(t.didx + col) * t.d0 + lev * t.d1;
        }
    }
    T v[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (k * blockDim.x + threadIdx.x < t.count) v[k] = ld_stream(src + so[k]);
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (k * blockDim.x + threadIdx.x < t.count) dst[doff[k]] = v[k];
}

template<int K>
__global__ void __launch_bounds__(k_max_block) exchange_kernel(const xtile* __restrict__ tiles)
{
    __shared__ xtile t;
    load_record<6>(t, tiles + blockIdx.x);
    if (t.kind == 0)
    {
        switch (t.unit)
        {
            case 8:
                if (t.neg) box_elements<K, unsigned long long, true>(t);
                else
                    box_elements<K, unsigned long long, false>(t);
                break;
            case 4:
                if (t.neg) box_elements<K, uint32_t, true>(t);
                else
                    box_elements<K, uint32_t, false>(t);
                break;
            case 2: box_elements<K, uint16_t, false>(t); break;
            default: box_elements<K, uint8_t, false>(t); break;
        }
    }
    else
    {
        switch (t.unit)
        {
            case 16: list_elements<(K > 1 ? K / 2 : 1), uint4>(t); break;
            case 8: list_elements<K, unsigned long long>(t); break;
            case 4: list_elements<K, uint32_t>(t); break;
            case 2: list_elements<K, uint16_t>(t); break;
            default: list_elements<K, uint8_t>(t); break;
        }
    }
}

// ---- box adjoint in gather form --------------------------------------------------------------
// NI images per owner element (the cell's image count, dispatched at run time); all loads of a
// thread's K owner elements and their images are issued before the first store.
template<int K, int NI, typename F>
__device__ __forceinline__ void gather_elements(const gtile& t)
{
    F* __restrict__ own = reinterpret_cast<F*>(t.own);
    F h[K][NI];
    F acc[K];
    int32_t ooff[K];
    int32_t hoff[K][NI];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        if (e < t.count)
        {
            const uint32_t g = t.e0 + e;
            const uint32_t r = fdiv(g, t.m0, t.l0);
            const int32_t i0 = (int32_t)(g - r * t.n0);
            const uint32_t q = fdiv(r, t.m1, t.l1);
            const int32_t i1 = (int32_t)(r - q * t.n1), i2 = (int32_t)q;
            ooff[k] = i0 * t.o0 + i1 * t.o1 + i2 * t.o2;
            acc[k] = __ldcg(own + ooff[k]);
#pragma unroll
            for (int i = 0; i < NI; ++i)
            {
                hoff[k][i] = i0 * t.img[i].t0 + i1 * t.img[i].t1 + i2 * t.img[i].t2;
                h[k][i] = __ldcg(reinterpret_cast<const F*>(t.img[i].ptr) + hoff[k][i]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (k * blockDim.x + threadIdx.x < t.count)
        {
            F a = acc[k];
#pragma unroll
            for (int i = 0; i < NI; ++i)
            {
                a = t.img[i].neg ? a - h[k][i] : a + h[k][i];
                reinterpret_cast<F*>(t.img[i].ptr)[hoff[k][i]] = F(0);
            }
            own[ooff[k]] = a;
        }
}

template<typename F>
__device__ __forceinline__ void gather_dispatch(const gtile& t)
{
    switch (t.nimg)
    {
        case 1: gather_elements<gather_per_thread(1), 1, F>(t); break;
        case 2: gather_elements<gather_per_thread(2), 2, F>(t); break;
        case 3: gather_elements<gather_per_thread(3), 3, F>(t); break;
        case 4: gather_elements<gather_per_thread(4), 4, F>(t); break;
        case 5: gather_elements<gather_per_thread(5), 5, F>(t); break;
        case 6: gather_elements<gather_per_thread(6), 6, F>(t); break;
        case 7: gather_elements<gather_per_thread(7), 7, F>(t); break;
        default: gather_elements<gather_per_thread(8), 8, F>(t); break;
    }
}

__global__ void __launch_bounds__(k_gather_block, 3) gather_kernel(const gtile* __restrict__ tiles)
{
    __shared__ gtile t;
    load_record<16>(t, tiles + blockIdx.x);
    if (t.esize == 8) gather_dispatch<double>(t);
    else
        gather_dispatch<float>(t);
}
} // namespace

cudaError_t launch_exchange(const xtile* tiles, int ntiles, int k, int block, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    switch (k)
    {
        case 4: exchange_kernel<4><<<ntiles, block, 0, stream>>>(tiles); break;
        case 8: exchange_kernel<8><<<ntiles, block, 0, stream>>>(tiles); break;
        case 16: exchange_kernel<16><<<ntiles, block, 0, stream>>>(tiles); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_gather(const gtile* tiles, int ntiles, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    gather_kernel<<<ntiles, k_gather_block, 0, stream>>>(tiles);
    return cudaGetLastError();
}
} // namespace ghexb

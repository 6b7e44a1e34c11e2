// Forward exchange and box adjoint kernels (sm_100a).
//
// The exchange is pure data movement, latency-bound at halo sizes: a kernel's time is a few
// dependent memory round trips plus the bytes over HBM bandwidth. The kernels are built for few
// round trips and many bytes in flight:
//  * one launch covers every tile, one CTA per tile; a CTA runs the code specialised for its
//    tile's element class (box, pair of x faces or list; element size; negation; for the
//    adjoint the number of images), and the hardware block scheduler balances CTAs across SMs:
//    no scheduler of ours, no atomics, CTAs never wait on each other;
//  * a tile record carries everything needed to address its elements (112 bytes forward, 256
//    bytes adjoint): one round trip before the data loads;
//  * every thread issues all of its K loads before its first store, so K elements per thread
//    are in flight; consecutive threads take consecutive elements, so rows along the
//    destination's contiguous dimension are coalesced;
//  * element coordinates come from two multiply-high divisions per element (fast_div), no
//    per-row bookkeeping, so short rows waste no lanes.
// A halo element moves from the source interior to the destination halo with one read and one
// write; no intermediate buffer exists.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

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
// Stores through st.global: the compiler then knows that they cannot alias the tile record in
// shared memory and keeps the record's fields in registers across them.
template<typename T> __device__ __forceinline__ void st_global(T* p, T v) { __stcg(p, v); }
template<> __device__ __forceinline__ void st_global(uint16_t* p, uint16_t v)
{
    __stcg(reinterpret_cast<unsigned short*>(p), (unsigned short)v);
}
template<> __device__ __forceinline__ void st_global(uint8_t* p, uint8_t v)
{
    __stcg(reinterpret_cast<unsigned char*>(p), (unsigned char)v);
}
template<> __device__ __forceinline__ uint16_t ld_stream(const uint16_t* p)
{
    return __ldcg(reinterpret_cast<const unsigned short*>(p));
}
template<> __device__ __forceinline__ uint8_t ld_stream(const uint8_t* p)
{
    return __ldcg(reinterpret_cast<const unsigned char*>(p));
}

// CTAs start roughly in block order, about a thousand at a time: the record of the CTA that
// starts a wave later is brought into L2 now, so that after the first wave a CTA's first round
// trip is an L2 hit rather than a DRAM access (the tables are read once per exchange, cold after
// other work has run).
constexpr unsigned k_record_prefetch = 1024;

// Loads this CTA's record (W 16-byte words) into shared memory.
template<int W, typename R>
__device__ __forceinline__ void load_record(R& t, const R* __restrict__ tiles)
{
    if (threadIdx.x == 32 && blockIdx.x + k_record_prefetch < gridDim.x)
    {
        const char* next = reinterpret_cast<const char*>(tiles + blockIdx.x + k_record_prefetch);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(next));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(next + sizeof(R) - 1));
    }
    if (threadIdx.x < W)
        reinterpret_cast<uint4*>(&t)[threadIdx.x] = __ldg(reinterpret_cast<const uint4*>(tiles + blockIdx.x) + threadIdx.x);
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
        doff[k] = 0;
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
            if constexpr (NEG) st_global(dst + doff[k], (T)(v[k] ^ sign_bit<T>::v));
            else
                st_global(dst + doff[k], v[k]);
        }
}

// blk: the tile's index block in shared memory (the indices of columns t.u0, t.u0 + 1, ...), or
// nullptr when the tile reads its indices from the lists
template<int K, typename T>
__device__ __forceinline__ void list_elements(const xtile& t, const int32_t* blk)
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
            if (blk)
            {
                const uint32_t c = col - (uint32_t)t.u0;
                so[k] = blk[c] * t.s0 + lev * t.s1;
                doff[k] = blk[k_block_columns + c] * t.d0 + lev * t.d1;
            }
            else
            {
                so[k] = __ldg(t.sidx + col) * t.s0 + lev * t.s1;
                doff[k] = __ldg(t.didx + col) * t.d0 + lev * t.d1;
            }
        }
    }
    T v[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (k * blockDim.x + threadIdx.x < t.count) v[k] = ld_stream(src + so[k]);
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (k * blockDim.x + threadIdx.x < t.count) st_global(dst + doff[k], v[k]);
}

// Pairs of x-face boxes: a segment of na + nb destination elements is contiguous, so the warp's
// stores to it coalesce into whole sectors.
template<int K, typename T>
__device__ __forceinline__ void pair_elements(const xtile& t)
{
    T* __restrict__ dst = reinterpret_cast<T*>(t.dst);
    T v[K];
    int32_t doff[K];
    bool ok[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        ok[k] = false;
        doff[k] = 0;
        if (e < t.count)
        {
            const uint32_t g = t.e0 + e;
            const uint32_t q = fdiv(g, t.m0, t.l0);
            const int32_t c = (int32_t)(g - q * t.n0);
            const uint32_t i2 = fdiv(q, t.m1, t.l1);
            const int32_t s = (int32_t)(q - i2 * t.n1);
            const bool a = c < (int32_t)t.na;
            if (a ? s >= 1 : s + 1 < (int32_t)t.n1)
            {
                const T* src = reinterpret_cast<const T*>(a ? t.src : t.src2);
                const int32_t so = a ? c * t.s0 + (s - 1) * t.s1 + (int32_t)i2 * t.s2
                                     : (c - (int32_t)t.na) * t.u0 + s * t.u1 + (int32_t)i2 * t.u2;
                v[k] = ld_stream(src + so);
                if (a ? t.neg : t.neg2) v[k] ^= sign_bit<T>::v;
                doff[k] = c + (s - 1) * t.d1 + (int32_t)i2 * t.d2;
                ok[k] = true;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (ok[k]) st_global(dst + doff[k], v[k]);
}

// The index lists of the list tiles: the first CTAs bring them into L2 at the start of the launch,
// 4 KB each (one 128-byte line per lane of their last warp), so that the CTAs of later waves find
// their indices in L2 when their records arrive.
__device__ __forceinline__ void prefetch_lists(const char* __restrict__ lists, uint32_t bytes)
{
    if (bytes == 0 || threadIdx.x < blockDim.x - 32) return;
    const uint64_t off = (uint64_t)blockIdx.x * 4096 + (threadIdx.x - (blockDim.x - 32)) * 128;
    if (off < bytes) asm volatile("prefetch.global.L2 [%0];" ::"l"(lists + off));
}

template<int K>
__global__ void __launch_bounds__(k_max_block, K >= 16 ? 1 : 2) exchange_kernel(const xtile* __restrict__ tiles,
    const char* __restrict__ lists, uint32_t list_bytes, const int32_t* __restrict__ blocks)
{
    __shared__ xtile t;
    __shared__ __align__(16) int32_t blk_s[k_block_ints];
    prefetch_lists(lists, list_bytes);
    // the tile's index block, in the same round trip as its record (threads 7..22: 16 words)
    if (blocks && threadIdx.x >= k_xtile_words && threadIdx.x < k_xtile_words + k_block_ints / 4)
        reinterpret_cast<int4*>(blk_s)[threadIdx.x - k_xtile_words] =
            __ldg(reinterpret_cast<const int4*>(blocks + (size_t)blockIdx.x * k_block_ints) + (threadIdx.x - k_xtile_words));
    load_record<k_xtile_words>(t, tiles);
    const int32_t* blk = blocks && t.pad[0] ? blk_s : nullptr;
    switch (t.cls)
    {
#define GHEXB_CASE(C, F)                                                                                               \
    case C: F(t); break;
        GHEXB_CASE(k_box8, (box_elements<K, unsigned long long, false>))
        GHEXB_CASE(k_box8_neg, (box_elements<K, unsigned long long, true>))
        GHEXB_CASE(k_box4, (box_elements<K, uint32_t, false>))
        GHEXB_CASE(k_box4_neg, (box_elements<K, uint32_t, true>))
        GHEXB_CASE(k_box2, (box_elements<K, uint16_t, false>))
        GHEXB_CASE(k_box1, (box_elements<K, uint8_t, false>))
        case k_list16: list_elements<forward_per_thread(K, 16), uint4>(t, blk); break;
        case k_list8: list_elements<K, unsigned long long>(t, blk); break;
        case k_list4: list_elements<K, uint32_t>(t, blk); break;
        case k_list2: list_elements<K, uint16_t>(t, blk); break;
        case k_list1: list_elements<K, uint8_t>(t, blk); break;
        GHEXB_CASE(k_pair8, (pair_elements<K, unsigned long long>))
        GHEXB_CASE(k_pair4, (pair_elements<K, uint32_t>))
#undef GHEXB_CASE
        default: break;
    }
}

// ---- box adjoint in gather form --------------------------------------------------------------
// NI images per owner element; all loads of a thread's K owner elements and their images are
// issued before the first store.
template<int K, int NI, typename F>
__device__ __forceinline__ void gather_elements(const gtile& t)
{
    F* __restrict__ own = reinterpret_cast<F*>(t.own);
    F h[K][NI];
    F acc[K];
    // an element's cell coordinates are derived again for the stores rather than its offsets held
    // in registers across the loads
    auto coords = [&](uint32_t e, int32_t& i0, int32_t& i1, int32_t& i2) {
        const uint32_t g = t.e0 + e;
        const uint32_t r = fdiv(g, t.m0, t.l0);
        i0 = (int32_t)(g - r * t.n0);
        const uint32_t q = fdiv(r, t.m1, t.l1);
        i1 = (int32_t)(r - q * t.n1), i2 = (int32_t)q;
    };
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        if (e < t.count)
        {
            int32_t i0, i1, i2;
            coords(e, i0, i1, i2);
            acc[k] = __ldcg(own + (i0 * t.o0 + i1 * t.o1 + i2 * t.o2));
#pragma unroll
            for (int i = 0; i < NI; ++i)
                h[k][i] = __ldcg(reinterpret_cast<const F*>(t.img[i].ptr) + (i0 * t.img[i].t0 + i1 * t.img[i].t1 + i2 * t.img[i].t2));
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        if (e < t.count)
        {
            int32_t i0, i1, i2;
            coords(e, i0, i1, i2);
            F a = acc[k];
#pragma unroll
            for (int i = 0; i < NI; ++i)
            {
                a = t.img[i].neg ? a - h[k][i] : a + h[k][i];
                st_global(reinterpret_cast<F*>(t.img[i].ptr) + (i0 * t.img[i].t0 + i1 * t.img[i].t1 + i2 * t.img[i].t2), F(0));
            }
            st_global(own + (i0 * t.o0 + i1 * t.o1 + i2 * t.o2), a);
        }
    }
}

// Unstructured owner columns: element e is level e mod n0 of owner e / n0 of the group; the
// owner's and its images' column addresses come from the column table.
template<int K, int NI, typename F>
__device__ __forceinline__ void list_gather_elements(const gtile& t, const uint64_t* __restrict__ cols,
    const uint64_t* blk)
{
    F h[K][NI];
    F acc[K];
    // the tile's columns from its block in shared memory, else from the column table; a column's
    // address is looked up again for the stores rather than held in registers across the loads
    const uint32_t j0 = blk ? fdiv(t.e0, t.m0, t.l0) : 0u;
    const uint64_t* base = blk ? blk - (size_t)j0 * (NI + 1) : cols + t.col0;
    auto column = [&](uint32_t e, int i) {
        const uint32_t g = t.e0 + e;
        const uint32_t j = fdiv(g, t.m0, t.l0);
        const int32_t lev = (int32_t)(g - j * t.n0);
        const uint64_t* p = base + (size_t)j * (NI + 1) + i;
        return reinterpret_cast<F*>(blk ? *p : __ldg(p)) + lev * (i == 0 ? t.o0 : t.img[0].t0);
    };
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        if (e < t.count)
        {
            acc[k] = __ldcg(column(e, 0));
#pragma unroll
            for (int i = 0; i < NI; ++i) h[k][i] = __ldcg(column(e, 1 + i));
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint32_t e = k * blockDim.x + threadIdx.x;
        if (e < t.count)
        {
            F a = acc[k];
#pragma unroll
            for (int i = 0; i < NI; ++i)
            {
                a = a + h[k][i];
                st_global(column(e, 1 + i), F(0));
            }
            st_global(column(e, 0), a);
        }
    }
}

__global__ void __launch_bounds__(k_gather_block, 3) gather_kernel(const gtile* __restrict__ tiles)
{
    __shared__ gtile t;
    load_record<16>(t, tiles);
    switch (t.cls)
    {
#define GHEXB_CASE(NI)                                                                                                 \
    case gather_class(8, NI): gather_elements<gather_per_thread(NI), NI, double>(t); break;                          \
    case gather_class(4, NI): gather_elements<gather_per_thread(NI), NI, float>(t); break;
        GHEXB_CASE(1)
        GHEXB_CASE(2)
        GHEXB_CASE(3)
        GHEXB_CASE(4)
        GHEXB_CASE(5)
        GHEXB_CASE(6)
        GHEXB_CASE(7)
        GHEXB_CASE(8)
#undef GHEXB_CASE
        default: break;
    }
}

// The unstructured owner groups have a kernel of their own, so that the box kernel's code (and
// its instruction-cache footprint) stays that of the box classes.
static_assert(k_gblock_entries % 2 == 0 && 16 + k_gblock_entries / 2 <= k_gather_block, "column block load lanes");

__global__ void __launch_bounds__(k_gather_block, 4) list_gather_kernel(const gtile* __restrict__ tiles,
    const uint64_t* __restrict__ cols, const uint64_t* __restrict__ blocks)
{
    __shared__ gtile t;
    __shared__ __align__(16) uint64_t blk_s[k_gblock_entries];
    // threads 16.. load the tile's column block while threads 0..15 load the record
    if (blocks && threadIdx.x >= 16 && threadIdx.x < 16 + k_gblock_entries / 2)
        reinterpret_cast<uint4*>(blk_s)[threadIdx.x - 16] =
            __ldg(reinterpret_cast<const uint4*>(blocks + (size_t)blockIdx.x * k_gblock_entries) + (threadIdx.x - 16));
    load_record<16>(t, tiles);
    const uint64_t* blk = blocks && t.pad[0] ? blk_s : nullptr;
    switch (t.cls)
    {
#define GHEXB_CASE(NI)                                                                                                 \
    case list_gather_class(8, NI): list_gather_elements<gather_per_thread(NI), NI, double>(t, cols, blk); break;     \
    case list_gather_class(4, NI): list_gather_elements<gather_per_thread(NI), NI, float>(t, cols, blk); break;
        GHEXB_CASE(1)
        GHEXB_CASE(2)
        GHEXB_CASE(3)
        GHEXB_CASE(4)
        GHEXB_CASE(5)
        GHEXB_CASE(6)
        GHEXB_CASE(7)
        GHEXB_CASE(8)
#undef GHEXB_CASE
        default: break;
    }
}

} // namespace

cudaError_t launch_exchange(const xtile* tiles, int ntiles, int k, int block, cudaStream_t stream, const void* lists,
    size_t list_bytes, const int32_t* blocks)
{
    if (ntiles <= 0) return cudaSuccess;
    if (block < 32 || block > k_max_block || block % 32) return cudaErrorInvalidValue;
    const int grid = ntiles;
    const char* pl = static_cast<const char*>(lists);
    const uint32_t pb = lists ? (uint32_t)std::min<size_t>(list_bytes, 0xffffffffu) : 0u;
    switch (k)
    {
        case 4: exchange_kernel<4><<<grid, block, 0, stream>>>(tiles, pl, pb, blocks); break;
        case 8: exchange_kernel<8><<<grid, block, 0, stream>>>(tiles, pl, pb, blocks); break;
        case 16: exchange_kernel<16><<<grid, block, 0, stream>>>(tiles, pl, pb, blocks); break;
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

cudaError_t launch_list_gather(const gtile* tiles, int ntiles, const uint64_t* cols, const uint64_t* blocks,
    cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    list_gather_kernel<<<ntiles, k_gather_block, 0, stream>>>(tiles, cols, blocks);
    return cudaGetLastError();
}
} // namespace ghexb

// Phased adjoint kernels and the L2 flush of the autotuner (sm_100a).
//
// The phased adjoint is the fallback of the gather-form box adjoint (exchange.cu) for layouts the
// gather cells cannot describe, and the adjoint of unstructured index lists. Descriptors are
// grouped into phases in which no two elements share an owner, so within a launch the
// read-add-write of an owner needs no atomics and the order of additions per owner is the order
// of the launches. A launch walks a tile table persistently: CTAs claim tiles from a counter.
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace ghexb
{
namespace
{
constexpr int k_per_thread = 8; // elements a thread moves per chunk (row_map: p * j <= 8)

// ---- dynamic tile scheduler -----------------------------------------------------------------
// CTAs claim tiles from a global counter, one atomic per tile. The last CTA to finish returns
// both counters to zero, so every launch starts from zero; launches that share counters must
// therefore be ordered on one stream (a plan's launches are). Nothing ever waits on the counters.
struct sched
{
    unsigned* next; // next tile to claim
    unsigned* done; // CTAs finished
};

__device__ __forceinline__ void sched_finish(const sched& s)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        if (atomicAdd(s.done, 1u) == gridDim.x - 1)
        {
            atomicExch(s.next, 0u);
            atomicExch(s.done, 0u);
        }
    }
}

// One chunk of work: `count` consecutive rows of a descriptor starting at row `start`.
struct chunk
{
    int32_t desc;
    uint32_t start;
    uint32_t count;
};

template<typename D>
__device__ __forceinline__ uint32_t rows_per_chunk(const D* d)
{
    return (blockDim.x >> d->map.wlog) * d->map.p;
}

// Walks the tiles the CTA claims as chunks. Claims run one tile ahead: thread 0 holds the next
// claim in a register (its atomic was issued a whole tile earlier) and publishes it through
// shared memory when the current tile ends; the record of the following tile is loaded before it
// is needed. init() and next() must be called by all threads of the CTA together.
template<typename D>
struct chunk_walker
{
    const D* __restrict__ descs;
    const tile* __restrict__ tiles;
    int ntiles;
    sched s;
    unsigned* slot; // shared memory, two words
    tile cur, after;
    uint32_t off;
    bool valid, after_valid;
    unsigned pending; // thread 0: claimed, not yet published

    __device__ void init()
    {
        if (threadIdx.x == 0)
        {
            slot[0] = atomicAdd(s.next, 1u);
            slot[1] = atomicAdd(s.next, 1u);
            pending = atomicAdd(s.next, 1u);
        }
        __syncthreads();
        const unsigned t0 = slot[0], t1 = slot[1];
        valid = t0 < (unsigned)ntiles;
        after_valid = t1 < (unsigned)ntiles;
        if (valid) cur = tiles[t0];
        if (after_valid) after = tiles[t1];
        off = 0;
    }
    __device__ void advance()
    {
        cur = after;
        valid = after_valid;
        off = 0;
        __syncthreads(); // every thread has read the previous publication
        if (threadIdx.x == 0)
        {
            slot[0] = pending;
            pending = atomicAdd(s.next, 1u);
        }
        __syncthreads();
        const unsigned t = slot[0];
        after_valid = t < (unsigned)ntiles;
        if (after_valid) after = tiles[t];
    }
    __device__ bool next(chunk& c)
    {
        if (!valid) return false;
        const uint32_t cap = rows_per_chunk(descs + cur.desc);
        c.desc = cur.desc;
        c.start = cur.start + off;
        c.count = min(cap, cur.count - off);
        off += c.count;
        if (off >= cur.count) advance();
        return true;
    }
};

// ---- row iteration ----------------------------------------------------------------------------
// Calls f(k, row, i0) for the elements this thread owns in a chunk: k < 8 is the thread's slot,
// row < count the chunk-relative row, i0 < n the position in the row. Rows are interleaved across
// warps so that neighbouring warps take neighbouring rows.
// Only the slots k in [KLO, KHI) are visited.
template<int KLO = 0, int KHI = k_per_thread, typename F>
__device__ __forceinline__ void for_chunk_elements(const row_map m, uint32_t count, int n, F&& f)
{
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t R = 32u >> m.wlog;
    const uint32_t lr = lane >> m.wlog, lc = lane & ((1u << m.wlog) - 1u);
    const int J = m.j, K = m.p * m.j;
    int p = KLO / J, j = KLO - (KLO / J) * J;
#pragma unroll
    for (int k = KLO; k < KHI; ++k)
    {
        if (k >= K) break;
        const uint32_t row = ((uint32_t)p * nw + warp) * R + lr;
        const int i0 = (int)(lc + ((uint32_t)j << m.wlog));
        if (row < count && i0 < n) f(k, row, i0);
        if (++j == J) j = 0, ++p;
    }
}

// Register-path persistent loop (small element classes, adjoint).
template<typename D, typename Body>
__device__ __forceinline__ void register_loop(const D* __restrict__ descs, const tile* __restrict__ tiles,
    int ntiles, const sched& sc, Body&& body)
{
    __shared__ unsigned claim[2];
    chunk_walker<D> w{descs, tiles, ntiles, sc, claim, {}, {}, 0u, false, false, 0u};
    w.init();
    chunk c{0, 0, 0};
    while (w.next(c)) body(descs + c.desc, c);
    sched_finish(sc);
}

// ---- adjoint ----------------------------------------------------------------------------------
// Within one launch no two elements share an owner, so the read-add-write of the owner needs no
// atomics and the order of additions per owner is the order of the launches.
template<typename F>
__device__ __forceinline__ void box_adjoint_rows(const box_desc* __restrict__ bd, const chunk& c)
{
    F* __restrict__ owner = reinterpret_cast<F*>(const_cast<char*>(bd->src));
    F* __restrict__ halo = reinterpret_cast<F*>(bd->dst);
    const int32_t s0 = bd->s0, s1 = bd->s1, s2 = bd->s2, d0 = bd->d0, d1 = bd->d1, d2 = bd->d2;
    const uint32_t n1 = (uint32_t)bd->n1;
    const fast_div f1 = bd->div1;
    const bool neg = bd->xor_mask != 0;
    for_chunk_elements(bd->map, c.count, bd->n0, [&](int, uint32_t row, int i0) {
        const uint32_t r = c.start + row;
        const uint32_t q = f1.div(r);
        const int32_t i1 = (int32_t)(r - q * n1), i2 = (int32_t)q;
        const int32_t so = i0 * s0 + i1 * s1 + i2 * s2;
        const int32_t doff = i0 * d0 + i1 * d1 + i2 * d2;
        const F h = halo[doff];
        const F o = owner[so];
        owner[so] = neg ? (o - h) : (o + h);
        halo[doff] = F(0);
    });
}

template<typename F>
__device__ __forceinline__ void list_adjoint_rows(const list_desc* __restrict__ ld, const chunk& c)
{
    F* __restrict__ owner = reinterpret_cast<F*>(const_cast<char*>(ld->src));
    F* __restrict__ halo = reinterpret_cast<F*>(ld->dst);
    const int32_t* __restrict__ sidx = ld->sidx;
    const int32_t* __restrict__ didx = ld->didx;
    const int32_t s_is = ld->s_is, s_ls = ld->s_ls, d_is = ld->d_is, d_ls = ld->d_ls;
    for_chunk_elements(ld->map, c.count, ld->levels, [&](int, uint32_t row, int lev) {
        const int32_t so = sidx[c.start + row] * s_is + lev * s_ls;
        const int32_t doff = didx[c.start + row] * d_is + lev * d_ls;
        const F hv = halo[doff];
        owner[so] = owner[so] + hv;
        halo[doff] = F(0);
    });
}

__global__ void __launch_bounds__(512, 2) box_adjoint_kernel(
    const box_desc* __restrict__ boxes, const tile* __restrict__ tiles, int ntiles, sched sc)
{
    register_loop(boxes, tiles, ntiles, sc, [](const box_desc* bd, const chunk& c) {
        if (bd->esize == 8) box_adjoint_rows<double>(bd, c);
        else
            box_adjoint_rows<float>(bd, c);
    });
}

__global__ void __launch_bounds__(512, 2) list_adjoint_kernel(
    const list_desc* __restrict__ lists, const tile* __restrict__ tiles, int ntiles, sched sc)
{
    register_loop(lists, tiles, ntiles, sc, [](const list_desc* ld, const chunk& c) {
        if (ld->unit == 8) list_adjoint_rows<double>(ld, c);
        else
            list_adjoint_rows<float>(ld, c);
    });
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

// Calibration copy of short rows: dst[r*dst_stride + i] = src[r*src_stride + i] for r < rows, i < n;
// consecutive threads take consecutive elements, each thread 8 elements (all loads before any
// store), as the exchange kernel moves the rows of a box, without its tile records.
// MODE 0 copies, 1 only reads (a value reaches dst only in the impossible case that the rows sum
// to a sentinel), 2 only writes (each element its own index).
template<typename T, int MODE>
__global__ void __launch_bounds__(256) row_copy_kernel(const T* __restrict__ src, T* __restrict__ dst, uint32_t rows,
    uint32_t n, int64_t src_stride, int64_t dst_stride)
{
    constexpr int K = 8;
    const uint64_t total = (uint64_t)rows * n;
    T v[K];
    int64_t o[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const uint64_t e = ((uint64_t)blockIdx.x * K + k) * blockDim.x + threadIdx.x;
        o[k] = -1;
        v[k] = (T)e;
        if (e < total)
        {
            const uint64_t r = e / n, i = e - r * n;
            if (MODE != 2) v[k] = __ldcg(src + r * src_stride + i);
            o[k] = (int64_t)(r * dst_stride + i);
        }
    }
    if (MODE == 1)
    {
        T acc = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) acc ^= o[k] >= 0 ? v[k] : T(0);
        if (acc == (T)0x5bd1e995u && o[0] >= 0) dst[o[0]] = acc;
        return;
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (o[k] >= 0) __stcg(dst + o[k], v[k]);
}

template<typename T>
cudaError_t row_copy(const void* src, void* dst, uint32_t rows, uint32_t n, int64_t ss, int64_t ds, int mode,
    unsigned grid, cudaStream_t stream)
{
    const T* s = static_cast<const T*>(src);
    T* d = static_cast<T*>(dst);
    switch (mode)
    {
        case 0: row_copy_kernel<T, 0><<<grid, 256, 0, stream>>>(s, d, rows, n, ss, ds); break;
        case 1: row_copy_kernel<T, 1><<<grid, 256, 0, stream>>>(s, d, rows, n, ss, ds); break;
        case 2: row_copy_kernel<T, 2><<<grid, 256, 0, stream>>>(s, d, rows, n, ss, ds); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_row_copy(const void* src, void* dst, uint32_t rows, uint32_t n, int64_t src_stride,
    int64_t dst_stride, int es, int mode, cudaStream_t stream)
{
    const uint64_t total = (uint64_t)rows * n;
    if (total == 0) return cudaSuccess;
    const unsigned grid = (unsigned)((total + 8 * 256 - 1) / (8 * 256));
    if (es == 8) return row_copy<unsigned long long>(src, dst, rows, n, src_stride, dst_stride, mode, grid, stream);
    if (es == 4) return row_copy<unsigned>(src, dst, rows, n, src_stride, dst_stride, mode, grid, stream);
    return cudaErrorInvalidValue;
}

cudaError_t launch_l2_flush(const uint4* buf, size_t n16, unsigned* sink, int grid, cudaStream_t stream)
{
    l2_flush_kernel<<<grid, 256, 0, stream>>>(buf, n16, sink);
    return cudaGetLastError();
}

cudaError_t launch_box_adjoint(const box_desc* boxes, const tile* tiles, int ntiles, unsigned* counters, int grid,
    int block, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    box_adjoint_kernel<<<grid, block, 0, stream>>>(boxes, tiles, ntiles, sched{counters, counters + 1});
    return cudaGetLastError();
}

cudaError_t launch_list_adjoint(const list_desc* lists, const tile* tiles, int ntiles, unsigned* counters, int grid,
    int block, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    list_adjoint_kernel<<<grid, block, 0, stream>>>(lists, tiles, ntiles, sched{counters, counters + 1});
    return cudaGetLastError();
}

} // namespace ghexb

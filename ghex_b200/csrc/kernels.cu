// Device kernels of ghex_b200 (sm_100a).
//
// The exchange is pure data movement, so the kernels are built for HBM bandwidth and for few
// instructions per byte, not for the tensor cores:
//  * work is organised in rows: a row is one contiguous run along the destination's fastest
//    dimension (a box row) or one column of an index list. W = 2^wlog lanes share a row, so a warp
//    covers 32 / W short rows (an x-face halo row of 3 cells takes 4 lanes) or one long row;
//    there is one division per row and none per element;
//  * one persistent launch walks a tile table (a tile is a range of rows of one descriptor);
//    CTAs claim tiles dynamically, one tile ahead, so short-row tiles (the most DRAM sectors per
//    byte) and long-row tiles balance across SMs;
//  * the 4- and 8-byte element classes stage their loads through shared memory with cp.async:
//    a load in flight costs a shared-memory slot, not a register, and three pipeline stages keep
//    two chunks of loads in flight while the oldest chunk is stored;
//  * unstructured columns move as 16-byte units when every column is 16-byte aligned.
// A halo element moves from the source interior to the destination halo with exactly one read
// and one write: no intermediate message buffer exists.
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace ghexb
{
namespace
{
constexpr int k_per_thread = 8; // elements a thread moves per chunk (row_map: p * j <= 8)
constexpr int k_stages = 3;

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

// ---- cp.async -------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async(uint32_t smem, const void* g, int bytes)
{
    if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem), "l"(g) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem), "l"(g) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// waits until at most k_stages - 1 groups are pending: the oldest chunk has landed
__device__ __forceinline__ void cp_async_wait_ahead()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(k_stages - 1) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

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

// ---- forward: boxes ---------------------------------------------------------------------------
// Issue and drain are instantiated per J (elements per lane per row); a thread takes P = 8 / J
// rows per chunk, so both loops unroll completely: per row one division and one address, per
// element one cp.async (or one shared load and one store) at a constant offset.
struct lane_pos
{
    uint32_t row0;   // first chunk-relative row of this thread
    uint32_t rstep;  // rows between this thread's consecutive rows
    int lc;          // position of this lane inside its row
    int w;           // lanes per row
};

__device__ __forceinline__ lane_pos lane_position(const row_map m)
{
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t R = 32u >> m.wlog;
    return lane_pos{warp * R + (lane >> m.wlog), nw * R, (int)(lane & ((1u << m.wlog) - 1u)), 1 << m.wlog};
}

template<int J, int SLOT>
__device__ __forceinline__ void box_issue_j(const box_desc* __restrict__ bd, const chunk& c, uint32_t stage)
{
    constexpr int P = k_per_thread / J;
    const lane_pos lp = lane_position(bd->map);
    const int es = (int)bd->esize, n0 = bd->n0;
    const int32_t s0 = bd->s0, s1 = bd->s1, s2 = bd->s2;
    const uint32_t n1 = (uint32_t)bd->n1;
    const fast_div f1 = bd->div1;
    const int64_t jstep = (int64_t)lp.w * s0 * es;
    const char* src = bd->src + (int64_t)lp.lc * s0 * es;
    const uint32_t sl = stage + threadIdx.x * SLOT, kstep = blockDim.x * SLOT;
    uint32_t row = lp.row0;
#pragma unroll
    for (int p = 0; p < P; ++p, row += lp.rstep)
    {
        if (row < c.count)
        {
            const uint32_t r = c.start + row;
            const uint32_t q = f1.div(r);
            const char* rp = src + (int64_t)((int32_t)(r - q * n1) * s1 + (int32_t)q * s2) * es;
#pragma unroll
            for (int j = 0; j < J; ++j)
                if (lp.lc + j * lp.w < n0) cp_async(sl + (p * J + j) * kstep, rp + j * jstep, es);
        }
    }
}

template<int J, int SLOT>
__device__ __forceinline__ void box_drain_j(const box_desc* __restrict__ bd, const chunk& c, const char* stage)
{
    constexpr int P = k_per_thread / J;
    const lane_pos lp = lane_position(bd->map);
    const int n0 = bd->n0;
    const int32_t d0 = bd->d0, d1 = bd->d1, d2 = bd->d2;
    const uint32_t n1 = (uint32_t)bd->n1;
    const fast_div f1 = bd->div1;
    const uint64_t xm = bd->xor_mask;
    const bool wide = bd->esize == 8;
    const char* sl = stage + threadIdx.x * SLOT;
    const uint32_t kstep = blockDim.x * SLOT;
    uint32_t row = lp.row0;
    if (wide)
    {
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(bd->dst) + lp.lc * d0;
        const int32_t jstep = lp.w * d0;
#pragma unroll
        for (int p = 0; p < P; ++p, row += lp.rstep)
            if (row < c.count)
            {
                const uint32_t r = c.start + row;
                const uint32_t q = f1.div(r);
                unsigned long long* rp = dst + ((int32_t)(r - q * n1) * d1 + (int32_t)q * d2);
#pragma unroll
                for (int j = 0; j < J; ++j)
                    if (lp.lc + j * lp.w < n0)
                        rp[j * jstep] = *reinterpret_cast<const unsigned long long*>(sl + (p * J + j) * kstep) ^ xm;
            }
    }
    else
    {
        uint32_t* dst = reinterpret_cast<uint32_t*>(bd->dst) + lp.lc * d0;
        const int32_t jstep = lp.w * d0;
        const uint32_t xm32 = (uint32_t)xm;
#pragma unroll
        for (int p = 0; p < P; ++p, row += lp.rstep)
            if (row < c.count)
            {
                const uint32_t r = c.start + row;
                const uint32_t q = f1.div(r);
                uint32_t* rp = dst + ((int32_t)(r - q * n1) * d1 + (int32_t)q * d2);
#pragma unroll
                for (int j = 0; j < J; ++j)
                    if (lp.lc + j * lp.w < n0)
                        rp[j * jstep] = *reinterpret_cast<const uint32_t*>(sl + (p * J + j) * kstep) ^ xm32;
            }
    }
}

// dispatch on J (uniform across the CTA: one descriptor per chunk)
#define GHEXB_DISPATCH_J(jval, CALL)                                                                                   \
    switch (jval)                                                                                                      \
    {                                                                                                                  \
        case 1: CALL(1); break;                                                                                        \
        case 2: CALL(2); break;                                                                                        \
        case 3: CALL(3); break;                                                                                        \
        case 4: CALL(4); break;                                                                                        \
        case 5: CALL(5); break;                                                                                        \
        case 6: CALL(6); break;                                                                                        \
        case 7: CALL(7); break;                                                                                        \
        default: CALL(8); break;                                                                                       \
    }

template<int SLOT>
__device__ __forceinline__ void box_issue(const box_desc* __restrict__ bd, const chunk& c, uint32_t stage)
{
#define GHEXB_CALL(J) box_issue_j<J, SLOT>(bd, c, stage)
    GHEXB_DISPATCH_J(bd->map.j, GHEXB_CALL)
#undef GHEXB_CALL
}

template<int SLOT>
__device__ __forceinline__ void box_drain(const box_desc* __restrict__ bd, const chunk& c, const char* stage)
{
#define GHEXB_CALL(J) box_drain_j<J, SLOT>(bd, c, stage)
    GHEXB_DISPATCH_J(bd->map.j, GHEXB_CALL)
#undef GHEXB_CALL
}

// Register path for 1- and 2-byte elements (no cp.async for those sizes).
template<typename T>
__device__ __forceinline__ void box_rows_reg(const box_desc* __restrict__ bd, const chunk& c)
{
    const T* __restrict__ src = reinterpret_cast<const T*>(bd->src);
    T* __restrict__ dst = reinterpret_cast<T*>(bd->dst);
    const int32_t s0 = bd->s0, s1 = bd->s1, s2 = bd->s2, d0 = bd->d0, d1 = bd->d1, d2 = bd->d2;
    const uint32_t n1 = (uint32_t)bd->n1;
    const fast_div f1 = bd->div1;
    const uint32_t xm = (uint32_t)bd->xor_mask;
    T v[k_per_thread];
    int32_t doff[k_per_thread];
    bool ok[k_per_thread];
#pragma unroll
    for (int k = 0; k < k_per_thread; ++k) ok[k] = false;
    for_chunk_elements(bd->map, c.count, bd->n0, [&](int k, uint32_t row, int i0) {
        const uint32_t r = c.start + row;
        const uint32_t q = f1.div(r);
        const int32_t i1 = (int32_t)(r - q * n1), i2 = (int32_t)q;
        v[k] = src[i0 * s0 + i1 * s1 + i2 * s2];
        doff[k] = i0 * d0 + i1 * d1 + i2 * d2;
        ok[k] = true;
    });
#pragma unroll
    for (int k = 0; k < k_per_thread; ++k)
        if (ok[k]) dst[doff[k]] = (T)(v[k] ^ xm);
}

// ---- forward: index lists ---------------------------------------------------------------------
template<int J, int SLOT>
__device__ __forceinline__ void list_issue_j(const list_desc* __restrict__ ld, const chunk& c, uint32_t stage)
{
    constexpr int P = k_per_thread / J;
    const lane_pos lp = lane_position(ld->map);
    const int u = (int)ld->unit, L = ld->levels;
    const int32_t* __restrict__ sidx = ld->sidx;
    const int32_t s_is = ld->s_is, s_ls = ld->s_ls;
    const int64_t jstep = (int64_t)lp.w * s_ls * u;
    const char* src = ld->src + (int64_t)lp.lc * s_ls * u;
    const uint32_t sl = stage + threadIdx.x * SLOT, kstep = blockDim.x * SLOT;
    uint32_t row = lp.row0;
#pragma unroll
    for (int p = 0; p < P; ++p, row += lp.rstep)
        if (row < c.count)
        {
            const char* rp = src + (int64_t)__ldg(sidx + c.start + row) * s_is * u;
#pragma unroll
            for (int j = 0; j < J; ++j)
                if (lp.lc + j * lp.w < L) cp_async(sl + (p * J + j) * kstep, rp + j * jstep, u);
        }
}

template<int J, int SLOT>
__device__ __forceinline__ void list_drain_j(const list_desc* __restrict__ ld, const chunk& c, const char* stage)
{
    constexpr int P = k_per_thread / J;
    const lane_pos lp = lane_position(ld->map);
    const int L = ld->levels;
    const int32_t* __restrict__ didx = ld->didx;
    const int32_t d_is = ld->d_is, d_ls = ld->d_ls;
    const char* sl = stage + threadIdx.x * SLOT;
    const uint32_t kstep = blockDim.x * SLOT;
    uint32_t row = lp.row0;
    if (ld->unit == 16)
    {
        uint4* dst = reinterpret_cast<uint4*>(ld->dst) + lp.lc * d_ls;
        const int32_t jstep = lp.w * d_ls;
#pragma unroll
        for (int p = 0; p < P; ++p, row += lp.rstep)
            if (row < c.count)
            {
                uint4* rp = dst + __ldg(didx + c.start + row) * d_is;
#pragma unroll
                for (int j = 0; j < J; ++j)
                    if (lp.lc + j * lp.w < L) rp[j * jstep] = *reinterpret_cast<const uint4*>(sl + (p * J + j) * kstep);
            }
    }
    else
    {
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(ld->dst) + lp.lc * d_ls;
        const int32_t jstep = lp.w * d_ls;
#pragma unroll
        for (int p = 0; p < P; ++p, row += lp.rstep)
            if (row < c.count)
            {
                unsigned long long* rp = dst + __ldg(didx + c.start + row) * d_is;
#pragma unroll
                for (int j = 0; j < J; ++j)
                    if (lp.lc + j * lp.w < L)
                        rp[j * jstep] = *reinterpret_cast<const unsigned long long*>(sl + (p * J + j) * kstep);
            }
    }
}

template<int SLOT>
__device__ __forceinline__ void list_issue(const list_desc* __restrict__ ld, const chunk& c, uint32_t stage)
{
#define GHEXB_CALL(J) list_issue_j<J, SLOT>(ld, c, stage)
    GHEXB_DISPATCH_J(ld->map.j, GHEXB_CALL)
#undef GHEXB_CALL
}

template<int SLOT>
__device__ __forceinline__ void list_drain(const list_desc* __restrict__ ld, const chunk& c, const char* stage)
{
#define GHEXB_CALL(J) list_drain_j<J, SLOT>(ld, c, stage)
    GHEXB_DISPATCH_J(ld->map.j, GHEXB_CALL)
#undef GHEXB_CALL
}

template<typename T>
__device__ __forceinline__ void list_rows_reg(const list_desc* __restrict__ ld, const chunk& c)
{
    const T* __restrict__ src = reinterpret_cast<const T*>(ld->src);
    T* __restrict__ dst = reinterpret_cast<T*>(ld->dst);
    const int32_t* __restrict__ sidx = ld->sidx;
    const int32_t* __restrict__ didx = ld->didx;
    const int32_t s_is = ld->s_is, s_ls = ld->s_ls, d_is = ld->d_is, d_ls = ld->d_ls;
    T v[k_per_thread];
    int32_t doff[k_per_thread];
    bool ok[k_per_thread];
#pragma unroll
    for (int k = 0; k < k_per_thread; ++k) ok[k] = false;
    for_chunk_elements(ld->map, c.count, ld->levels, [&](int k, uint32_t row, int lev) {
        v[k] = src[__ldg(sidx + c.start + row) * s_is + lev * s_ls];
        doff[k] = __ldg(didx + c.start + row) * d_is + lev * d_ls;
        ok[k] = true;
    });
#pragma unroll
    for (int k = 0; k < k_per_thread; ++k)
        if (ok[k]) dst[doff[k]] = v[k];
}

// ---- staged persistent pipeline ----------------------------------------------------------------
// Three chunks in flight: chunk n + 2 is issued while chunk n drains. Exactly two groups (possibly
// empty) are committed before the loop and one per iteration, so chunk n is the n-th committed
// group and wait_group 2 at iteration n means it has landed. Element (thread t, slot k) of a
// stage lives at byte (k * blockDim + t) * SLOT, so every shared-memory byte belongs to one
// thread and no barrier is needed between stages.
template<int SLOT, typename D, typename Issue, typename Drain>
__device__ __forceinline__ void staged_pipeline(const D* __restrict__ descs, const tile* __restrict__ tiles,
    int ntiles, const sched& sc, Issue&& issue, Drain&& drain)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ unsigned claim[2];
    static_assert(k_stages == 3, "the pipeline below rotates three chunks");
    const uint32_t stage_bytes = k_per_thread * blockDim.x * SLOT;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    chunk_walker<D> w{descs, tiles, ntiles, sc, claim, {}, {}, 0u, false, false, 0u};
    w.init();
    chunk c0{0, 0, 0}, c1{0, 0, 0}, c2{0, 0, 0};
    bool h0 = w.next(c0);
    if (h0) issue(descs + c0.desc, c0, sbase);
    cp_async_commit();
    bool h1 = h0 && w.next(c1);
    if (h1) issue(descs + c1.desc, c1, sbase + stage_bytes);
    cp_async_commit();
    for (uint32_t n = 0; h0; ++n)
    {
        const bool h2 = h1 && w.next(c2);
        if (h2) issue(descs + c2.desc, c2, sbase + ((n + 2) % 3) * stage_bytes);
        cp_async_commit();
        cp_async_wait_ahead();
        drain(descs + c0.desc, c0, smem + (n % 3) * stage_bytes);
        c0 = c1, h0 = h1;
        c1 = c2, h1 = h2;
    }
    cp_async_wait_all();
    sched_finish(sc);
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

// Box descriptors in one persistent launch; LARGE selects the 8/4-byte class (staged), else 2/1.
template<bool LARGE>
__global__ void __launch_bounds__(k_max_block, 2) box_exchange_kernel(
    const box_desc* __restrict__ boxes, const tile* __restrict__ tiles, int ntiles, sched sc)
{
    if constexpr (LARGE)
    {
        staged_pipeline<8>(boxes, tiles, ntiles, sc,
            [](const box_desc* bd, const chunk& c, uint32_t st) { box_issue<8>(bd, c, st); },
            [](const box_desc* bd, const chunk& c, const char* st) { box_drain<8>(bd, c, st); });
    }
    else
    {
        register_loop(boxes, tiles, ntiles, sc, [](const box_desc* bd, const chunk& c) {
            if (bd->esize == 2) box_rows_reg<uint16_t>(bd, c);
            else
                box_rows_reg<uint8_t>(bd, c);
        });
    }
}

// List descriptors in one persistent launch; LARGE selects 16/8-byte units (staged), else 4/2/1.
template<bool LARGE>
__global__ void __launch_bounds__(k_max_block, 2) list_exchange_kernel(
    const list_desc* __restrict__ lists, const tile* __restrict__ tiles, int ntiles, sched sc)
{
    if constexpr (LARGE)
    {
        staged_pipeline<16>(lists, tiles, ntiles, sc,
            [](const list_desc* ld, const chunk& c, uint32_t st) { list_issue<16>(ld, c, st); },
            [](const list_desc* ld, const chunk& c, const char* st) { list_drain<16>(ld, c, st); });
    }
    else
    {
        register_loop(lists, tiles, ntiles, sc, [](const list_desc* ld, const chunk& c) {
            if (ld->unit == 4) list_rows_reg<uint32_t>(ld, c);
            else if (ld->unit == 2)
                list_rows_reg<uint16_t>(ld, c);
            else
                list_rows_reg<uint8_t>(ld, c);
        });
    }
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

__global__ void __launch_bounds__(k_max_block, 2) box_adjoint_kernel(
    const box_desc* __restrict__ boxes, const tile* __restrict__ tiles, int ntiles, sched sc)
{
    register_loop(boxes, tiles, ntiles, sc, [](const box_desc* bd, const chunk& c) {
        if (bd->esize == 8) box_adjoint_rows<double>(bd, c);
        else
            box_adjoint_rows<float>(bd, c);
    });
}

__global__ void __launch_bounds__(k_max_block, 2) list_adjoint_kernel(
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

// Allows the staged kernels the shared memory of their stages at the largest block size.
cudaError_t raise_smem_limits()
{
    static const cudaError_t e = [] {
        cudaError_t r = cudaFuncSetAttribute(box_exchange_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
            k_stages * k_per_thread * k_max_block * 8);
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(list_exchange_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                k_stages * k_per_thread * k_max_block * 16);
        return r;
    }();
    return e;
}
} // namespace

cudaError_t launch_l2_flush(const uint4* buf, size_t n16, unsigned* sink, int grid, cudaStream_t stream)
{
    l2_flush_kernel<<<grid, 256, 0, stream>>>(buf, n16, sink);
    return cudaGetLastError();
}

cudaError_t launch_box_exchange(const box_desc* boxes, const tile* tiles, int ntiles, bool large, unsigned* counters,
    int grid, int block, cudaStream_t stream)
{
    if (const cudaError_t e = raise_smem_limits(); e != cudaSuccess) return e;
    if (ntiles <= 0) return cudaSuccess;
    const sched sc{counters, counters + 1};
    if (large)
        box_exchange_kernel<true><<<grid, block, (size_t)k_stages * k_per_thread * block * 8, stream>>>(
            boxes, tiles, ntiles, sc);
    else
        box_exchange_kernel<false><<<grid, block, 0, stream>>>(boxes, tiles, ntiles, sc);
    return cudaGetLastError();
}

cudaError_t launch_list_exchange(const list_desc* lists, const tile* tiles, int ntiles, bool large, unsigned* counters,
    int grid, int block, cudaStream_t stream)
{
    if (const cudaError_t e = raise_smem_limits(); e != cudaSuccess) return e;
    if (ntiles <= 0) return cudaSuccess;
    const sched sc{counters, counters + 1};
    if (large)
        list_exchange_kernel<true><<<grid, block, (size_t)k_stages * k_per_thread * block * 16, stream>>>(
            lists, tiles, ntiles, sc);
    else
        list_exchange_kernel<false><<<grid, block, 0, stream>>>(lists, tiles, ntiles, sc);
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

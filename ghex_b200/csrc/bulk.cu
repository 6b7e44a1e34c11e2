// Bulk column kernel (bulk.hpp): one warp per tile; lane 0 arms the tile's mbarrier with the
// tile's bytes, every lane issues the bulk loads of its columns (lane, lane + 32) into the shared
// stage, all wait for the barrier (bounded in time), then every lane issues the bulk stores of its
// columns and waits until the copy engine has read them out of shared memory.
#include "async_copy.hpp"
#include "bulk.hpp"

namespace ghexb
{
namespace
{
__device__ __forceinline__ void gather4(void* dst, const CUtensorMap* map, const int32_t* rows, uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                 ::"r"(smem_u32(dst)), "l"(map), "r"(0), "r"(rows[0]), "r"(rows[1]), "r"(rows[2]), "r"(rows[3]),
                 "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void scatter4(const CUtensorMap* map, const int32_t* rows, const void* src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile::scatter4.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];"
                 ::"l"(map), "r"(0), "r"(rows[0]), "r"(rows[1]), "r"(rows[2]), "r"(rows[3]), "r"(smem_u32(src))
                 : "memory");
}

__global__ void __launch_bounds__(32) bulk_kernel(const btile* __restrict__ tiles, const int32_t* __restrict__ blocks,
    const CUtensorMap* __restrict__ maps, unsigned* status)
{
    __shared__ __align__(128) unsigned char stage[k_bulk_stage];
    __shared__ __align__(16) btile t;
    __shared__ __align__(16) int32_t blk[k_bulk_block_ints];
    __shared__ __align__(8) uint64_t bar;
    const unsigned lane = threadIdx.x;
    // the record (three 16-byte words) and the index block (32 words), one round trip
    if (lane < 3) reinterpret_cast<uint4*>(&t)[lane] = __ldg(reinterpret_cast<const uint4*>(tiles + blockIdx.x) + lane);
    reinterpret_cast<int4*>(blk)[lane] = __ldg(reinterpret_cast<const int4*>(blocks + (size_t)blockIdx.x * k_bulk_block_ints) + lane);
    if (lane == 0)
    {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    __syncwarp();
    const uint32_t n = t.ncols, cb = t.col_bytes;
    const bool four = t.smap >= 0;
    const uint32_t groups = (n + 3) / 4; // four columns at a time: lanes 0 .. groups - 1
    int32_t rows[4];
    if (lane == 0) mbar_expect_tx(&bar, four ? groups * 4 * cb : n * cb);
    __syncwarp();
    if (four)
    {
        if (lane < groups)
        {
            for (int q = 0; q < 4; ++q) rows[q] = blk[min(4 * lane + (uint32_t)q, n - 1)];
            gather4(stage + lane * 4 * cb, maps + t.smap, rows, &bar);
        }
    }
    else
        for (uint32_t c = lane; c < n; c += 32) bulk_load(stage + c * cb, t.src + (int64_t)blk[c] * t.s_is, cb, &bar);
    if (!mbar_wait(&bar, 0))
    {
        // the loads did not complete in time: the tile's columns are not stored; the CTA waits
        // (again bounded) for its loads, which write into its shared memory, before it ends
        if (lane == 0 && status) atomicOr(status, 1u);
        (void)mbar_wait(&bar, 0);
        return;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (four)
    {
        if (lane < groups)
        {
            for (int q = 0; q < 4; ++q) rows[q] = blk[k_bulk_columns + min(4 * lane + (uint32_t)q, n - 1)];
            scatter4(maps + t.dmap, rows, stage + lane * 4 * cb);
        }
    }
    else
        for (uint32_t c = lane; c < n; c += 32) bulk_store(t.dst + (int64_t)blk[k_bulk_columns + c] * t.d_is, stage + c * cb, cb);
    bulk_commit();
    bulk_wait_read();
}

// acc = own; acc = acc + image_i in order, for every level of every owner column of the stage
template<typename F>
__device__ __forceinline__ void gather_stage(unsigned char* stage, const bgtile& t, unsigned lane)
{
    const uint32_t per = t.nimg + 1, total = t.nown * t.levels;
    for (uint32_t e = lane; e < total; e += 32)
    {
        const uint32_t c = e / t.levels, lev = e - c * t.levels;
        F* own = reinterpret_cast<F*>(stage + (size_t)c * per * t.col_bytes) + lev;
        F a = *own;
        for (uint32_t i = 1; i <= t.nimg; ++i) a = a + reinterpret_cast<const F*>(stage + (size_t)(c * per + i) * t.col_bytes)[lev];
        *own = a;
    }
}

__global__ void __launch_bounds__(32) bulk_gather_kernel(const bgtile* __restrict__ tiles, const uint64_t* __restrict__ blocks,
    unsigned* status)
{
    __shared__ __align__(128) unsigned char stage[k_bulk_stage];
    __shared__ __align__(16) unsigned char zero[k_bgather_zero];
    __shared__ __align__(16) bgtile t;
    __shared__ __align__(16) uint64_t blk[k_bgather_entries];
    __shared__ __align__(8) uint64_t bar;
    const unsigned lane = threadIdx.x;
    // the record (two words) and the column addresses (48 words), one round trip
    const uint4* b = reinterpret_cast<const uint4*>(blocks + (size_t)blockIdx.x * k_bgather_entries);
    if (lane < 2) reinterpret_cast<uint4*>(&t)[lane] = __ldg(reinterpret_cast<const uint4*>(tiles + blockIdx.x) + lane);
    for (unsigned w = lane; w < k_bgather_entries / 2; w += 32) reinterpret_cast<uint4*>(blk)[w] = __ldg(b + w);
    for (unsigned w = lane; w < k_bgather_zero / 16; w += 32) reinterpret_cast<uint4*>(zero)[w] = make_uint4(0, 0, 0, 0);
    if (lane == 0)
    {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    __syncwarp();
    const uint32_t n = t.nown * (t.nimg + 1), cb = t.col_bytes;
    if (lane == 0) mbar_expect_tx(&bar, n * cb);
    __syncwarp();
    for (uint32_t c = lane; c < n; c += 32) bulk_load(stage + c * cb, reinterpret_cast<const void*>(blk[c]), cb, &bar);
    if (!mbar_wait(&bar, 0))
    {
        // the loads did not complete in time: nothing is stored; the CTA waits (again bounded) for
        // its loads, which write into its shared memory, before it ends
        if (lane == 0 && status) atomicOr(status, 4u);
        (void)mbar_wait(&bar, 0);
        return;
    }
    if (t.esize == 8) gather_stage<double>(stage, t, lane);
    else
        gather_stage<float>(stage, t, lane);
    // the sums and the zeros, written by the threads, are read by the copy engine
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    const uint32_t per = t.nimg + 1;
    for (uint32_t c = lane; c < n; c += 32)
        bulk_store(reinterpret_cast<void*>(blk[c]), c % per == 0 ? static_cast<const void*>(stage + c * cb) : zero, cb);
    bulk_commit();
    bulk_wait_read();
}
} // namespace

cudaError_t launch_bulk_gather(const bgtile* tiles, const uint64_t* blocks, int ntiles, unsigned* status,
    cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    bulk_gather_kernel<<<ntiles, 32, 0, stream>>>(tiles, blocks, status);
    return cudaGetLastError();
}

cudaError_t launch_bulk(const btile* tiles, const int32_t* blocks, const CUtensorMap* maps, int ntiles, unsigned* status,
    cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    bulk_kernel<<<ntiles, 32, 0, stream>>>(tiles, blocks, maps, status);
    return cudaGetLastError();
}
} // namespace ghexb

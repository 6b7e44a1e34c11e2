// Staged exchange kernel: tensor-map loads of halo source regions into shared memory, stores to
// the halos (sm_100a). See staged.hpp for the work items and the tensor-map classes.
//
// One persistent CTA runs items blockIdx.x, blockIdx.x + gridDim.x, ... in turn through a ring of
// `stages` shared-memory stages. Warp 0 is the producer: one thread copies the item record into
// the stage's slot, announces the load's bytes on the stage's `full` mbarrier and issues the
// cp.async.bulk.tensor load, up to `stages` loads ahead of the consumers. The other warps consume:
// they wait for `full`, write the stage's elements to the halo (consecutive threads to consecutive
// destination addresses) and arrive on the stage's `empty` mbarrier, which releases the stage to
// the producer. Every wait is bounded in time (about a second); a wait that gives up sets a bit in
// the status word, the producer still waits for the loads it issued (also bounded), and the CTA
// returns: the kernel always ends.
#include <cudaTypedefs.h>

#include <mutex>

#include "async_copy.hpp"
#include "staged.hpp"

namespace ghexb
{
namespace
{
constexpr int k_max_stages = 16;
constexpr int k_max_consumers = 8;

__device__ __forceinline__ uint32_t fdiv(uint32_t n, uint32_t m, uint32_t l) { return (__umulhi(n, m) + n) >> l; }

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                 ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
                 : "memory");
}

template<typename T> struct sign_of;
template<> struct sign_of<uint32_t> { static constexpr uint32_t v = 0x80000000u; };
template<> struct sign_of<unsigned long long> { static constexpr unsigned long long v = 0x8000000000000000ull; };

template<typename T, bool NEG>
__device__ __forceinline__ void write_stage(const sitem& it, const unsigned char* stage, uint32_t t, uint32_t nt)
{
    const T* __restrict__ buf = reinterpret_cast<const T*>(stage);
    T* __restrict__ dst = reinterpret_cast<T*>(it.dst);
    constexpr int U = 4; // elements per thread and pass: their shared loads issue before their stores
    for (uint32_t e0 = 0; e0 < it.count; e0 += U * nt)
    {
        T v[U];
        int32_t o[U];
#pragma unroll
        for (int k = 0; k < U; ++k)
        {
            const uint32_t e = e0 + k * nt + t;
            o[k] = INT32_MIN;
            if (e < it.count)
            {
                const uint32_t q = fdiv(e, it.mu, it.lu);
                const uint32_t u = e - q * it.nu;
                const uint32_t z = fdiv(q, it.mv, it.lv);
                const uint32_t w = q - z * it.nv;
                v[k] = buf[it.sbase + u * it.su + w * it.sv + z * it.sz];
                o[k] = (int32_t)u * it.du + (int32_t)w * it.dv + (int32_t)z * it.dz;
            }
        }
#pragma unroll
        for (int k = 0; k < U; ++k)
            if (o[k] != INT32_MIN)
            {
                if constexpr (NEG) __stcg(dst + o[k], (T)(v[k] ^ sign_of<T>::v));
                else
                    __stcg(dst + o[k], v[k]);
            }
    }
}

template<>
__device__ __forceinline__ void write_stage<uint16_t, false>(const sitem& it, const unsigned char* stage, uint32_t t,
    uint32_t nt)
{
    const uint16_t* buf = reinterpret_cast<const uint16_t*>(stage);
    unsigned short* dst = reinterpret_cast<unsigned short*>(it.dst);
    for (uint32_t e = t; e < it.count; e += nt)
    {
        const uint32_t q = fdiv(e, it.mu, it.lu), u = e - q * it.nu, z = fdiv(q, it.mv, it.lv), w = q - z * it.nv;
        __stcg(dst + ((int32_t)u * it.du + (int32_t)w * it.dv + (int32_t)z * it.dz),
            (unsigned short)buf[it.sbase + u * it.su + w * it.sv + z * it.sz]);
    }
}

template<>
__device__ __forceinline__ void write_stage<uint8_t, false>(const sitem& it, const unsigned char* stage, uint32_t t,
    uint32_t nt)
{
    unsigned char* dst = reinterpret_cast<unsigned char*>(it.dst);
    for (uint32_t e = t; e < it.count; e += nt)
    {
        const uint32_t q = fdiv(e, it.mu, it.lu), u = e - q * it.nu, z = fdiv(q, it.mv, it.lv), w = q - z * it.nv;
        __stcg(dst + ((int32_t)u * it.du + (int32_t)w * it.dv + (int32_t)z * it.dz),
            (unsigned char)stage[it.sbase + u * it.su + w * it.sv + z * it.sz]);
    }
}

__global__ void __launch_bounds__(32 * (1 + k_max_consumers)) staged_kernel(staged_launch a)
{
    extern __shared__ __align__(128) unsigned char dyn[];
    __shared__ uint64_t full[k_max_stages], empty[k_max_stages];
    __shared__ sitem slot[k_max_stages];
    // stages start on a 128-byte boundary (the launch adds 128 bytes for this)
    unsigned char* smem = dyn + ((128u - (smem_u32(dyn) & 127u)) & 127u);
    const uint32_t S = (uint32_t)a.stages;
    if (threadIdx.x == 0)
    {
        for (uint32_t s = 0; s < S; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], (uint32_t)a.consumers);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0)
    {
        if (lane != 0) return;
        uint32_t n = 0;
        bool ok = true;
        for (int i = blockIdx.x; i < a.nitems; i += gridDim.x, ++n)
        {
            const uint32_t s = n % S;
            if (n >= S && !mbar_wait(&empty[s], (n / S - 1) & 1))
            {
                ok = false;
                break;
            }
            const uint4* src = reinterpret_cast<const uint4*>(a.items + i);
            uint4* to = reinterpret_cast<uint4*>(&slot[s]);
#pragma unroll
            for (int w = 0; w < (int)(sizeof(sitem) / 16); ++w) to[w] = __ldg(src + w);
            mbar_expect_tx(&full[s], slot[s].bytes);
            tma_load_3d(smem + (size_t)s * a.stage_bytes, a.maps + slot[s].map, 0, slot[s].c1, slot[s].c2, &full[s]);
        }
        if (!ok) atomicOr(a.status, 1u);
        // the CTA must not end while a load it issued is still writing its shared memory
        for (uint32_t k = n > S ? n - S : 0; k < n; ++k)
            if (!mbar_wait(&full[k % S], (k / S) & 1)) atomicOr(a.status, 1u);
        return;
    }
    const uint32_t t = threadIdx.x - 32, nt = 32u * (uint32_t)a.consumers;
    uint32_t n = 0;
    for (int i = blockIdx.x; i < a.nitems; i += gridDim.x, ++n)
    {
        const uint32_t s = n % S;
        if (!mbar_wait(&full[s], (n / S) & 1))
        {
            atomicOr(a.status, 2u);
            return;
        }
        const sitem& it = slot[s];
        const unsigned char* stage = smem + (size_t)s * a.stage_bytes;
        switch (it.es * 2 + it.neg)
        {
            case 16: write_stage<unsigned long long, false>(it, stage, t, nt); break;
            case 17: write_stage<unsigned long long, true>(it, stage, t, nt); break;
            case 8: write_stage<uint32_t, false>(it, stage, t, nt); break;
            case 9: write_stage<uint32_t, true>(it, stage, t, nt); break;
            case 4: write_stage<uint16_t, false>(it, stage, t, nt); break;
            case 2: write_stage<uint8_t, false>(it, stage, t, nt); break;
            default: break;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
} // namespace

cudaError_t staged_prepare(int smem_bytes)
{
    return cudaFuncSetAttribute(staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
}

cudaError_t launch_staged(const staged_launch& a, cudaStream_t stream)
{
    if (a.nitems <= 0) return cudaSuccess;
    if (a.stages < 2 || a.stages > k_max_stages || a.consumers < 1 || a.consumers > k_max_consumers ||
        a.stage_bytes % 128 || a.grid < 1)
        return cudaErrorInvalidValue;
    staged_kernel<<<a.grid, 32 * (1 + a.consumers), (size_t)a.stages * a.stage_bytes + 128, stream>>>(a);
    return cudaGetLastError();
}

CUresult encode_tensor_map(CUtensorMap* map, CUtensorMapDataType type, cuuint32_t rank, void* base,
    const cuuint64_t* dims, const cuuint64_t* strides, const cuuint32_t* box, CUtensorMapL2promotion promo)
{
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return CUDA_ERROR_NOT_SUPPORTED;
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return g_encode(map, type, rank, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
        promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}
} // namespace ghexb

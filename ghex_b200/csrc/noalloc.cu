// ghexb_exchange_noalloc: the batched exchange without any device allocation.
//
// Some callers cannot allocate device memory at the point where they exchange halos: an
// application whose memory manager owns the device memory (a pool allocator that reserved HBM at
// start-up and treats any other cudaMalloc as a failure), or code that must not call
// cudaMalloc/cudaFree because those calls may synchronize the whole device. For them the work
// tables live in a fixed, file-scope device array instead of per-plan allocations.
//
// The array is k_noalloc_scratch_bytes large and exists once per device for as long as the
// library is loaded. Every call rebuilds the tables on the host (index lists, then forward tiles),
// copies them into the array on the caller's stream and launches the one batched exchange kernel
// on the same stream at the default tuning. A stream that is being captured is refused: the copy
// reads a host buffer that exists only during the call. All calls share the array, which keeps the
// contents of the last call: calls whose work overlaps on the GPU (on different streams, without
// ordering between them) race on it and must not be made.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>

#include "exchange.hpp"
#include "plan.hpp"

namespace
{
constexpr size_t k_noalloc_scratch_bytes = size_t(4) << 20; // 4 MiB per device

__device__ __align__(256) unsigned char g_noalloc_scratch[k_noalloc_scratch_bytes];

std::mutex g_scratch_mutex;
std::map<int, unsigned char*> g_scratch_address; // device -> device address of g_noalloc_scratch

// The device address of the scratch array on `device`, looked up once per device with that device
// current. In host code the array's name is only a host-side stand-in, never a device address.
// Every call checks that `device` is the current device: the copy and the launch go to the current
// device, and the tables and fields live on `device`.
unsigned char* scratch_address(int device)
{
    int current = -1;
    ghexb::check_cuda(cudaGetDevice(&current), "cudaGetDevice");
    if (current != device)
        throw ghexb::error(GHEXB_ERR_INVALID, "ghexb_exchange_noalloc: the context's device must be the current device");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    auto it = g_scratch_address.find(device);
    if (it != g_scratch_address.end()) return it->second;
    void* p = nullptr;
    ghexb::check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_address[device] = static_cast<unsigned char*>(p);
    return static_cast<unsigned char*>(p);
}

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

template<typename T>
size_t put(std::vector<unsigned char>& buf, size_t off, const std::vector<T>& v)
{
    if (!v.empty()) std::memcpy(buf.data() + off, v.data(), v.size() * sizeof(T));
    return align16(off + v.size() * sizeof(T));
}
} // namespace

extern "C" int ghexb_exchange_noalloc(ghexb_context ctx, const ghexb_field* fields, int n, void* stream)
{
    try
    {
        if (!ctx || !fields) throw ghexb::error(GHEXB_ERR_INVALID, "null argument");
        auto s = static_cast<cudaStream_t>(stream);
        // The tables are copied from a host buffer that lives only for this call: a captured copy
        // would read freed memory at every replay, so a capturing stream is refused.
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        ghexb::check_cuda(cudaStreamIsCapturing(s, &capture), "cudaStreamIsCapturing");
        if (capture != cudaStreamCaptureStatusNone)
            throw ghexb::error(GHEXB_ERR_INVALID, "ghexb_exchange_noalloc cannot be captured into a CUDA graph");
        // host tables of the batched form at the default tuning, every tile in the element kernel
        ghexb_plan_s plan;
        plan.bulk_share = 0;
        ghexb::build_tables(plan, ctx, fields, n);
        for (const auto& f : plan.fields) ghexb::check_accessible(f.data, ghexb::field_bytes(f));

        // layout: index lists | forward tiles (the tiles carry everything else the kernel needs)
        const size_t off_idx = 0;
        const size_t off_tiles = align16(off_idx + plan.idx.size() * sizeof(int32_t));
        unsigned char* dev = scratch_address(ctx->device);
        ghexb::build_tiles(plan, reinterpret_cast<const int32_t*>(dev + off_idx));
        const size_t end = align16(off_tiles + plan.xf.size() * sizeof(ghexb::xtile));
        if (end > k_noalloc_scratch_bytes)
            throw ghexb::error(GHEXB_ERR_RANGE, "ghexb_exchange_noalloc: the exchange tables need " + std::to_string(end) +
                                                    " bytes, more than the " + std::to_string(k_noalloc_scratch_bytes) +
                                                    " bytes of the no-alloc scratch; use ghexb_co_exchange");
        std::vector<unsigned char> host(end, 0);
        put(host, off_idx, plan.idx);
        put(host, off_tiles, plan.xf);

        // from pageable memory: the call returns once the data is staged, so `host` may go
        ghexb::check_cuda(cudaMemcpyAsync(dev, host.data(), end, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(no-alloc tables)");
        ghexb::check_cuda(ghexb::launch_exchange(reinterpret_cast<const ghexb::xtile*>(dev + off_tiles), (int)plan.xf.size(),
                              plan.per_thread, plan.block, s),
            "exchange kernel launch");
        return GHEXB_OK;
    }
    catch (const ghexb::error& e)
    {
        return ghexb::set_last_error(e.code, e.what());
    }
    catch (const std::exception& e)
    {
        return ghexb::set_last_error(GHEXB_ERR_INTERNAL, e.what());
    }
}

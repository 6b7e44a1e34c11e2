// ghexb_exchange_noalloc: the batched exchange without any device allocation.
//
// Some callers cannot allocate device memory at the point where they exchange halos: an
// application whose memory manager owns the device memory (a pool allocator that reserved HBM at
// start-up and treats any other cudaMalloc as a failure), or code that must not call
// cudaMalloc/cudaFree because those calls may synchronize the whole device. For them the work
// tables live in a fixed, file-scope device array instead of per-plan allocations.
//
// The array is k_noalloc_scratch_bytes large and exists once per device for as long as the
// library is loaded. Every call rebuilds the tables on the host, copies them into the array on the
// caller's stream (the scheduler counters, which must start at zero, are part of that copy) and
// launches the batched kernels on the same stream. All calls share the array, which keeps the
// contents of the last call: calls whose work overlaps on the GPU (on different streams, without
// ordering between them) race on it and must not be made.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>

#include "kernels.hpp"
#include "plan.hpp"

namespace
{
constexpr size_t k_noalloc_scratch_bytes = size_t(4) << 20; // 4 MiB per device

__device__ __align__(256) unsigned char g_noalloc_scratch[k_noalloc_scratch_bytes];

std::mutex g_scratch_mutex;
std::map<int, unsigned char*> g_scratch_address; // device -> device address of g_noalloc_scratch

// The device address of the scratch array on `device`, looked up once per device with that device
// current. In host code the array's name is only a host-side stand-in, never a device address.
unsigned char* scratch_address(int device)
{
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    auto it = g_scratch_address.find(device);
    if (it != g_scratch_address.end()) return it->second;
    int current = -1;
    ghexb::check_cuda(cudaGetDevice(&current), "cudaGetDevice");
    if (current != device)
        throw ghexb::error(GHEXB_ERR_INVALID, "ghexb_exchange_noalloc: the context's device must be the current device");
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
        // host tables of the batched form at the default tuning
        ghexb_plan_s plan;
        ghexb::build_tables(plan, ctx, fields, n);
        ghexb::build_tiles(plan);

        // layout: counters | boxes | lists | index lists | tiles of the four classes
        constexpr int k_classes = ghexb_plan_s::k_classes;
        const size_t off_ctr = 0;
        const size_t off_box = align16(off_ctr + 2 * k_classes * sizeof(unsigned));
        const size_t off_list = align16(off_box + plan.boxes.size() * sizeof(ghexb::box_desc));
        const size_t off_idx = align16(off_list + plan.lists.size() * sizeof(ghexb::list_desc));
        size_t off_tiles[k_classes];
        size_t end = align16(off_idx + plan.idx.size() * sizeof(int32_t));
        for (int c = 0; c < k_classes; ++c)
        {
            off_tiles[c] = end;
            end = align16(end + plan.ftiles[c].size() * sizeof(ghexb::tile));
        }
        if (end > k_noalloc_scratch_bytes)
            throw ghexb::error(GHEXB_ERR_RANGE, "ghexb_exchange_noalloc: the exchange tables need " + std::to_string(end) +
                                                    " bytes, more than the " + std::to_string(k_noalloc_scratch_bytes) +
                                                    " bytes of the no-alloc scratch; use ghexb_co_exchange");

        unsigned char* dev = scratch_address(ctx->device);
        // device pointers of the index lists inside the scratch
        auto* d_idx = reinterpret_cast<int32_t*>(dev + off_idx);
        for (size_t i = 0; i < plan.lists.size(); ++i)
        {
            plan.lists[i].sidx = d_idx + plan.list_idx_off[i];
            plan.lists[i].didx = d_idx + plan.list_idx_off[i] + plan.lists[i].count;
        }
        std::vector<unsigned char> host(end, 0); // counters start at zero
        put(host, off_box, plan.boxes);
        put(host, off_list, plan.lists);
        put(host, off_idx, plan.idx);
        for (int c = 0; c < k_classes; ++c) put(host, off_tiles[c], plan.ftiles[c]);

        auto s = static_cast<cudaStream_t>(stream);
        // from pageable memory: the call returns once the data is staged, so `host` may go
        ghexb::check_cuda(cudaMemcpyAsync(dev, host.data(), end, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(no-alloc tables)");
        auto* counters = reinterpret_cast<unsigned*>(dev + off_ctr);
        auto* boxes = reinterpret_cast<const ghexb::box_desc*>(dev + off_box);
        auto* lists = reinterpret_cast<const ghexb::list_desc*>(dev + off_list);
        for (int c = 0; c < k_classes; ++c)
        {
            const int nt = (int)plan.ftiles[c].size();
            if (nt == 0) continue;
            auto* tiles = reinterpret_cast<const ghexb::tile*>(dev + off_tiles[c]);
            const int grid = std::min(nt, ctx->num_sms * plan.ctas_per_sm);
            const cudaError_t e = c < 2
                ? ghexb::launch_box_exchange(boxes, tiles, nt, c == 0, counters + 2 * c, grid, plan.block, s)
                : ghexb::launch_list_exchange(lists, tiles, nt, c == 2, counters + 2 * c, grid, plan.block, s);
            ghexb::check_cuda(e, "exchange kernel launch");
        }
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

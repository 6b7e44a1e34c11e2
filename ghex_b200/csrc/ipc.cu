// CUDA IPC mappings of other processes' field memory (ipc.hpp).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "core.hpp"
#include "ipc.hpp"

namespace ghexb
{
namespace
{
PFN_cuMemGetAddressRange_v3020 g_range = nullptr;
std::once_flag g_range_once;

struct mapping
{
    char* base = nullptr;
    int refs = 0;
};
std::mutex g_mu;
std::map<std::string, mapping> g_maps; // by handle bytes

void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
    {
        (void)cudaGetLastError();
        throw error(GHEXB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
} // namespace

void ipc_export(const void* ptr, unsigned char* handle, int64_t* offset)
{
    std::call_once(g_range_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_range = reinterpret_cast<PFN_cuMemGetAddressRange_v3020>(fn);
    });
    if (!g_range) throw error(GHEXB_ERR_CUDA, "cuMemGetAddressRange is not available");
    cudaPointerAttributes a{};
    check(cudaPointerGetAttributes(&a, ptr), "cudaPointerGetAttributes");
    if (a.type != cudaMemoryTypeDevice)
        throw error(GHEXB_ERR_INVALID, "only device memory can be shared with other processes");
    CUdeviceptr base = 0;
    size_t size = 0;
    if (g_range(&base, &size, reinterpret_cast<CUdeviceptr>(ptr)) != CUDA_SUCCESS)
        throw error(GHEXB_ERR_CUDA, "cuMemGetAddressRange failed on field memory");
    cudaIpcMemHandle_t h{};
    check(cudaIpcGetMemHandle(&h, reinterpret_cast<void*>(base)),
        "cudaIpcGetMemHandle (the field's allocation cannot be shared: memory from cudaMalloc can, "
        "memory from stream-ordered or virtual-memory allocators cannot)");
    static_assert(sizeof(h) == k_ipc_handle_bytes, "IPC handle size");
    std::memcpy(handle, &h, sizeof(h));
    *offset = (int64_t)(reinterpret_cast<CUdeviceptr>(ptr) - base);
}

void* ipc_open(const unsigned char* handle, int64_t offset)
{
    if (offset < 0) throw error(GHEXB_ERR_INVALID, "negative offset into shared memory");
    const std::string key(reinterpret_cast<const char*>(handle), k_ipc_handle_bytes);
    std::lock_guard<std::mutex> lock(g_mu);
    auto& m = g_maps[key];
    if (m.refs == 0)
    {
        cudaIpcMemHandle_t h{};
        std::memcpy(&h, handle, sizeof(h));
        void* base = nullptr;
        const cudaError_t e = cudaIpcOpenMemHandle(&base, h, cudaIpcMemLazyEnablePeerAccess);
        if (e != cudaSuccess)
        {
            g_maps.erase(key);
            check(e, "cudaIpcOpenMemHandle");
        }
        m.base = static_cast<char*>(base);
    }
    ++m.refs;
    return m.base + offset;
}

void ipc_close(const unsigned char* handle)
{
    const std::string key(reinterpret_cast<const char*>(handle), k_ipc_handle_bytes);
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_maps.find(key);
    if (it == g_maps.end()) throw error(GHEXB_ERR_INVALID, "IPC handle is not open in this process");
    if (--it->second.refs == 0)
    {
        char* base = it->second.base;
        g_maps.erase(it);
        check(cudaIpcCloseMemHandle(base), "cudaIpcCloseMemHandle");
    }
}
} // namespace ghexb

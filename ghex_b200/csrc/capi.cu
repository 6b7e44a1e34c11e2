// extern "C" entry points of libghex_b200.so (declared in include/ghex_b200.h).
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "exchange.hpp"
#include "ipc.hpp"
#include "kernels.hpp"
#include "plan.hpp"
#include "stencil.hpp"

namespace
{
thread_local std::string g_last_error;

int set_error(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

template<typename F>
int guarded(F&& f)
{
    try
    {
        f();
        return GHEXB_OK;
    }
    catch (const ghexb::error& e)
    {
        return set_error(e.code, e.what());
    }
    catch (const std::bad_alloc&)
    {
        return set_error(GHEXB_ERR_ALLOC, "out of host memory");
    }
    catch (const std::exception& e)
    {
        return set_error(GHEXB_ERR_INTERNAL, e.what());
    }
}

void require(bool cond, const char* msg)
{
    if (!cond) throw ghexb::error(GHEXB_ERR_INVALID, msg);
}

std::vector<int64_t> signature(const ghexb_field* fields, int n)
{
    std::vector<int64_t> s;
    for (int i = 0; i < n; ++i)
    {
        const auto& f = *fields[i];
        s.push_back((int64_t)(intptr_t)f.pattern);
        s.push_back(f.domain_index);
        s.push_back(f.dtype);
        s.push_back((int64_t)(intptr_t)f.data);
        s.push_back(f.ndim);
        for (int a = 0; a < 4; ++a) s.push_back(f.offsets[a]), s.push_back(f.extents[a]), s.push_back(f.byte_strides[a]), s.push_back(f.layout[a]);
        s.push_back(f.num_components);
        s.push_back(f.is_vector);
        s.push_back(f.levels);
        s.push_back(f.levels_first);
        s.push_back(f.index_stride);
        s.push_back(f.level_stride);
    }
    return s;
}
} // namespace

namespace ghexb
{
// Records a failure for ghexb_last_error() from entry points defined in other files.
int set_last_error(int code, const std::string& msg) { return set_error(code, msg); }
} // namespace ghexb

struct ghexb_co_s
{
    ghexb_context_s* ctx = nullptr;
    std::map<std::vector<int64_t>, std::unique_ptr<ghexb_plan_s>> plans;
    bool in_place_receive = false;
    bool busy = false;
    cudaEvent_t done = nullptr;

    void wait()
    {
        if (!busy) return;
        ghexb::check_cuda(cudaEventSynchronize(done), "cudaEventSynchronize");
        busy = false;
    }
    bool ready()
    {
        if (!busy) return true;
        const cudaError_t e = cudaEventQuery(done);
        if (e == cudaErrorNotReady) return false;
        ghexb::check_cuda(e, "cudaEventQuery");
        busy = false;
        return true;
    }
};

struct ghexb_handle_s
{
    ghexb_co_s* co = nullptr;
};

extern "C" {

int ghexb_last_error(char* buf, size_t len)
{
    if (!buf || len == 0) return GHEXB_ERR_INVALID;
    const size_t n = std::min(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), n);
    buf[n] = 0;
    return GHEXB_OK;
}

int ghexb_version(int* major, int* minor, int* patch)
{
    return guarded([&] {
        require(major && minor && patch, "null output pointer");
        *major = 0, *minor = 1, *patch = 0;
    });
}

// ---- context ----------------------------------------------------------------------------
int ghexb_context_create(int device, ghexb_context* out)
{
    return guarded([&] {
        require(out != nullptr, "null output pointer");
        require(device >= 0, "device must be non-negative");
        auto* c = new ghexb_context_s();
        c->device = device;
        // Patterns are host-only, so a context can be made without a visible GPU; the SM count
        // is read when a device is present.
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
            c->num_sms = sms;
        else
            (void)cudaGetLastError();
        *out = c;
    });
}

int ghexb_context_destroy(ghexb_context ctx)
{
    delete ctx;
    return GHEXB_OK;
}

// ---- patterns ------------------------------------------------------------------------------
int ghexb_pattern_create_regular(ghexb_context ctx, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n_domains, const int64_t* domain_ids,
    const int* domain_first, const int* domain_last, ghexb_pattern* out)
{
    return guarded([&] {
        require(ctx && out && g_first && g_last && halos && periodic && domain_ids && domain_first && domain_last,
            "null argument");
        auto p = std::make_unique<ghexb_pattern_s>();
        p->ctx = ctx;
        ghexb::build_regular(*p, dim, g_first, g_last, halos, periodic, n_domains, domain_ids, domain_first, domain_last);
        *out = p.release();
    });
}

int ghexb_pattern_create_regular_staged(ghexb_context ctx, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n_domains, const int64_t* domain_ids, const int* domain_first,
    const int* domain_last, const int64_t* neighbor_ids, ghexb_pattern* out)
{
    return guarded([&] {
        require(ctx && g_first && g_last && halos && periodic && domain_ids && domain_first && domain_last &&
                    neighbor_ids && out,
            "null argument");
        require(dim >= 1 && dim <= 3, "regular patterns support 1 to 3 dimensions");
        std::vector<std::unique_ptr<ghexb_pattern_s>> ps;
        std::vector<ghexb_pattern_s*> raw;
        for (int i = 0; i < dim; ++i)
        {
            ps.push_back(std::make_unique<ghexb_pattern_s>());
            ps.back()->ctx = ctx;
            raw.push_back(ps.back().get());
        }
        ghexb::build_regular_staged(raw.data(), dim, g_first, g_last, halos, periodic, n_domains, domain_ids,
            domain_first, domain_last, neighbor_ids);
        for (int i = 0; i < dim; ++i) out[i] = ps[i].release();
    });
}

int ghexb_pattern_create_cubed_sphere(ghexb_context ctx, int edge_size, int levels, const int* halos,
    int n_domains, const int* tiles, const int* x_first, const int* x_last, const int* y_first,
    const int* y_last, ghexb_pattern* out)
{
    return guarded([&] {
        require(ctx && out && halos && tiles && x_first && x_last && y_first && y_last, "null argument");
        auto p = std::make_unique<ghexb_pattern_s>();
        p->ctx = ctx;
        ghexb::build_cubed_sphere(*p, edge_size, levels, halos, n_domains, tiles, x_first, x_last, y_first, y_last);
        *out = p.release();
    });
}

int ghexb_pattern_create_unstructured(ghexb_context ctx, int n_domains, const int64_t* domain_ids,
    const int64_t* gid_offsets, const int64_t* gids, const int64_t* outer_offsets,
    const int64_t* outer_lids, const int64_t* halo_gid_offsets, const int64_t* halo_gids,
    ghexb_pattern* out)
{
    return guarded([&] {
        require(ctx && out && domain_ids && gid_offsets && outer_offsets, "null argument");
        require(n_domains > 0, "a pattern needs at least one domain");
        require(gid_offsets[n_domains] == 0 || gids, "null gids");
        require(outer_offsets[n_domains] == 0 || outer_lids, "null outer lids");
        require(!halo_gid_offsets || halo_gid_offsets[n_domains] == 0 || halo_gids, "null halo gids");
        auto p = std::make_unique<ghexb_pattern_s>();
        p->ctx = ctx;
        ghexb::build_unstructured(*p, n_domains, domain_ids, gid_offsets, gids, outer_offsets, outer_lids,
            halo_gid_offsets, halo_gids);
        *out = p.release();
    });
}

int ghexb_pattern_create_unstructured_hinted(ghexb_context ctx, int n_domains, const int64_t* domain_ids,
    const int64_t* gid_offsets, const int64_t* gids, const int64_t* outer_offsets, const int64_t* outer_lids,
    const int64_t* halo_gid_offsets, const int64_t* halo_gids, const int64_t* hint_offsets,
    const int64_t* hint_domain_ids, const int64_t* hint_remote_indices, ghexb_pattern* out)
{
    return guarded([&] {
        require(ctx && out && domain_ids && gid_offsets && outer_offsets && hint_offsets, "null argument");
        require(n_domains > 0, "a pattern needs at least one domain");
        require(gid_offsets[n_domains] == 0 || gids, "null gids");
        require(outer_offsets[n_domains] == 0 || outer_lids, "null outer lids");
        require(!halo_gid_offsets || halo_gid_offsets[n_domains] == 0 || halo_gids, "null halo gids");
        require(hint_offsets[n_domains] == 0 || (hint_domain_ids && hint_remote_indices), "null hints");
        auto p = std::make_unique<ghexb_pattern_s>();
        p->ctx = ctx;
        ghexb::build_unstructured(*p, n_domains, domain_ids, gid_offsets, gids, outer_offsets, outer_lids,
            halo_gid_offsets, halo_gids, hint_offsets, hint_domain_ids, hint_remote_indices);
        *out = p.release();
    });
}

int ghexb_pattern_destroy(ghexb_pattern p)
{
    delete p;
    return GHEXB_OK;
}

int ghexb_pattern_num_domains(ghexb_pattern p, int* n)
{
    return guarded([&] {
        require(p && n, "null argument");
        *n = (int)p->domains.size();
    });
}

int ghexb_pattern_domain_id(ghexb_pattern p, int i, int64_t* id)
{
    return guarded([&] {
        require(p && id, "null argument");
        require(i >= 0 && i < (int)p->domains.size(), "domain index out of range");
        *id = p->domains[i].id;
    });
}

int ghexb_pattern_max_tag(ghexb_pattern p, int* max_tag)
{
    return guarded([&] {
        require(p && max_tag, "null argument");
        *max_tag = p->max_tag;
    });
}

int ghexb_pattern_num_spaces(ghexb_pattern p, int i, int send, int* n)
{
    return guarded([&] {
        require(p && n, "null argument");
        require(i >= 0 && i < (int)p->domains.size(), "domain index out of range");
        const auto& d = p->domains[i];
        if (p->kind == ghexb::pattern_kind::unstructured)
        {
            *n = (int)(send ? d.usend.size() : d.urecv.size());
            return;
        }
        int c = 0;
        for (const auto& e : (send ? d.send : d.recv)) c += (int)e.spaces.size();
        *n = c;
    });
}

int ghexb_pattern_space(ghexb_pattern p, int i, int send, int k, int* neighbor_index, int* local_first,
    int* local_last, int* global_first, int* global_last)
{
    return guarded([&] {
        require(p && neighbor_index && local_first && local_last && global_first && global_last, "null argument");
        require(p->kind != ghexb::pattern_kind::unstructured, "unstructured patterns hold index lists");
        require(i >= 0 && i < (int)p->domains.size(), "domain index out of range");
        const auto& d = p->domains[i];
        for (const auto& e : (send ? d.send : d.recv))
        {
            if (k < (int)e.spaces.size())
            {
                const auto& s = e.spaces[k];
                *neighbor_index = e.neighbor;
                for (int a = 0; a < 4; ++a)
                {
                    local_first[a] = s.lfirst[a];
                    local_last[a] = s.llast[a];
                    global_first[a] = s.gfirst[a];
                    global_last[a] = s.glast[a];
                }
                return;
            }
            k -= (int)e.spaces.size();
        }
        throw ghexb::error(GHEXB_ERR_INVALID, "space index out of range");
    });
}

int ghexb_pattern_space_indices(ghexb_pattern p, int i, int send, int k, int* neighbor_index,
    int64_t* lids, int64_t capacity, int64_t* count)
{
    return guarded([&] {
        require(p && neighbor_index && count, "null argument");
        require(p->kind == ghexb::pattern_kind::unstructured, "structured patterns hold iteration spaces");
        require(i >= 0 && i < (int)p->domains.size(), "domain index out of range");
        const auto& v = send ? p->domains[i].usend : p->domains[i].urecv;
        require(k >= 0 && k < (int)v.size(), "entry index out of range");
        *neighbor_index = v[k].neighbor;
        *count = (int64_t)v[k].lids.size();
        if (lids)
        {
            require(capacity >= *count, "capacity too small");
            std::copy(v[k].lids.begin(), v[k].lids.end(), lids);
        }
    });
}

// ---- fields ----------------------------------------------------------------------------------
int ghexb_field_wrap(ghexb_pattern p, int64_t domain, int dtype, void* data, int ndim, const int* offsets,
    const int* extents, const int* layout_map, const int64_t* byte_strides, int num_components, int is_vector,
    ghexb_field* out)
{
    return guarded([&] {
        require(p && out && offsets && extents, "null argument");
        require(p->kind != ghexb::pattern_kind::unstructured, "use ghexb_field_wrap_unstructured for unstructured patterns");
        require(data != nullptr, "null data pointer");
        auto f = std::make_unique<ghexb_field_s>();
        f->pattern = p;
        f->dtype = dtype;
        f->esize = ghexb::dtype_size(dtype);
        f->data = static_cast<char*>(data);
        require(reinterpret_cast<uintptr_t>(data) % f->esize == 0, "data pointer is not aligned to its element size");
        require(num_components >= 1, "number of components must be greater than 0");
        if (p->kind == ghexb::pattern_kind::regular)
        {
            f->domain_index = p->find_domain(domain);
            if (f->domain_index < 0)
                throw ghexb::error(GHEXB_ERR_INCOMPATIBLE, "field incompatible with available domains!");
            require(ndim == p->dim || ndim == p->dim + 1, "field dimension must be the domain dimension (+1 for components)");
            if (ndim == p->dim) require(num_components == 1, "this field cannot have more than 1 components");
        }
        else
        {
            require(domain >= 0 && domain < (int64_t)p->domains.size(), "cubed-sphere domain index out of range");
            f->domain_index = (int)domain;
            require(ndim == 4, "cubed-sphere fields are 4-dimensional (x, y, z, component)");
        }
        require(!is_vector || ghexb::dtype_is_float(dtype), "vector fields must be float32 or float64");
        f->ndim = ndim;
        f->num_components = num_components;
        f->is_vector = is_vector != 0;
        for (int a = 0; a < ndim; ++a)
        {
            f->offsets[a] = offsets[a];
            f->extents[a] = extents[a];
        }
        if (ndim == p->dim + 1 || p->kind == ghexb::pattern_kind::cubed_sphere)
        {
            // the trailing dimension counts components (structured/field_descriptor.hpp:175-180)
            f->offsets[ndim - 1] = 0;
            f->extents[ndim - 1] = num_components;
        }
        for (int a = 0; a < ndim; ++a) require(f->extents[a] >= 1, "extents must be positive");
        std::array<int, 4> lay{};
        for (int a = 0; a < ndim; ++a) lay[a] = layout_map ? layout_map[a] : ndim - 1 - a;
        {
            std::array<int, 4> seen{};
            for (int a = 0; a < ndim; ++a)
            {
                require(lay[a] >= 0 && lay[a] < ndim, "layout map values must be 0..ndim-1");
                require(!seen[lay[a]]++, "layout map values must be distinct");
            }
        }
        f->layout = lay;
        if (byte_strides)
        {
            for (int a = 0; a < ndim; ++a)
            {
                require(byte_strides[a] > 0, "byte strides must be positive");
                require(byte_strides[a] % f->esize == 0, "byte strides must be multiples of the element size");
                f->byte_strides[a] = byte_strides[a];
            }
        }
        else
        {
            // gridtools layout: the dimension with the largest layout value has stride sizeof(T)
            int64_t s = f->esize;
            for (int v = ndim - 1; v >= 0; --v)
            {
                int a = 0;
                while (lay[a] != v) ++a;
                f->byte_strides[a] = s;
                s *= f->extents[a];
            }
        }
        *out = f.release();
    });
}

int ghexb_field_wrap_unstructured(ghexb_pattern p, int64_t domain_id, int dtype, void* data, int64_t levels,
    int levels_first, int64_t outer_stride, ghexb_field* out)
{
    return guarded([&] {
        require(p && out, "null argument");
        require(p->kind == ghexb::pattern_kind::unstructured, "not an unstructured pattern");
        require(data != nullptr, "null data pointer");
        require(levels >= 1, "levels must be positive");
        require(outer_stride >= 0, "outer stride must be non-negative");
        auto f = std::make_unique<ghexb_field_s>();
        f->pattern = p;
        f->dtype = dtype;
        f->esize = ghexb::dtype_size(dtype);
        f->data = static_cast<char*>(data);
        require(reinterpret_cast<uintptr_t>(data) % f->esize == 0, "data pointer is not aligned to its element size");
        f->domain_index = p->find_domain(domain_id);
        if (f->domain_index < 0) throw ghexb::error(GHEXB_ERR_INCOMPATIBLE, "field incompatible with available domains!");
        const int64_t size = p->domains[f->domain_index].size;
        f->levels = levels;
        f->levels_first = levels_first != 0;
        f->index_stride = f->levels_first ? (outer_stride ? outer_stride : levels) : 1;
        f->level_stride = f->levels_first ? 1 : (outer_stride ? outer_stride : size);
        require(!outer_stride || outer_stride >= (f->levels_first ? levels : size), "outer stride too small");
        *out = f.release();
    });
}

int ghexb_field_destroy(ghexb_field f)
{
    delete f;
    return GHEXB_OK;
}

// ---- host memory for fields --------------------------------------------------------------------
namespace
{
// Ranges registered by ghexb_host_register under the pointer it was given: one range normally,
// several when part of the requested range was page-locked already by other code.
std::mutex g_host_mutex;
std::map<void*, std::vector<void*>> g_host_runs;

bool host_locked(const void* p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}
} // namespace

int ghexb_host_register(void* ptr, size_t bytes, int* owned)
{
    return guarded([&] {
        require(ptr && bytes > 0 && owned, "null argument");
        cudaPointerAttributes a{};
        ghexb::check_cuda(cudaPointerGetAttributes(&a, ptr), "cudaPointerGetAttributes");
        std::vector<void*> runs;
        // the whole range at once, unless its first page is page-locked already (a pinned
        // allocation, or a registration of other code)
        const cudaError_t e = a.type == cudaMemoryTypeHost
                                  ? cudaErrorHostMemoryAlreadyRegistered
                                  : cudaHostRegister(ptr, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable);
        if (e == cudaSuccess)
            runs.push_back(ptr);
        else if (e == cudaErrorHostMemoryAlreadyRegistered)
        {
            // part of the range is locked by other code: lock each maximal run of pages that is
            // not, page by page
            (void)cudaGetLastError();
            const size_t page = (size_t)sysconf(_SC_PAGESIZE);
            char* c = static_cast<char*>(ptr);
            char* end = c + bytes;
            try
            {
                while (c < end)
                {
                    char* next = std::min(end, reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(c) / page + 1) * page));
                    if (host_locked(c))
                    {
                        c = next;
                        continue;
                    }
                    char* q = next;
                    while (q < end && !host_locked(q))
                        q = std::min(end, reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(q) / page + 1) * page));
                    ghexb::check_cuda(cudaHostRegister(c, (size_t)(q - c), cudaHostRegisterMapped | cudaHostRegisterPortable),
                        "cudaHostRegister");
                    runs.push_back(c);
                    c = q;
                }
            }
            catch (...)
            {
                for (void* r : runs) (void)cudaHostUnregister(r);
                throw;
            }
        }
        else
            ghexb::check_cuda(e, "cudaHostRegister");
        try
        {
            ghexb::check_accessible(ptr, bytes);
        }
        catch (...)
        {
            for (void* r : runs) (void)cudaHostUnregister(r);
            throw;
        }
        *owned = runs.empty() ? 0 : 1;
        if (!runs.empty())
        {
            std::lock_guard<std::mutex> lock(g_host_mutex);
            g_host_runs[ptr] = std::move(runs);
        }
    });
}

int ghexb_host_is_mapped(const void* ptr, size_t bytes, int* mapped)
{
    return guarded([&] {
        require(ptr && bytes > 0 && mapped, "null argument");
        *mapped = 0;
        try
        {
            ghexb::check_accessible(ptr, bytes);
        }
        catch (const ghexb::error&)
        {
            (void)cudaGetLastError();
            return;
        }
        *mapped = 1;
    });
}

int ghexb_host_alloc(size_t bytes, void** out)
{
    return guarded([&] {
        require(out != nullptr && bytes > 0, "null argument or empty allocation");
        *out = nullptr;
        ghexb::check_cuda(cudaHostAlloc(out, bytes, cudaHostAllocMapped | cudaHostAllocPortable), "cudaHostAlloc");
    });
}

int ghexb_host_free(void* ptr)
{
    return guarded([&] {
        require(ptr != nullptr, "null argument");
        ghexb::check_cuda(cudaFreeHost(ptr), "cudaFreeHost");
    });
}

int ghexb_host_unregister(void* ptr)
{
    return guarded([&] {
        require(ptr != nullptr, "null argument");
        std::vector<void*> runs{ptr};
        {
            std::lock_guard<std::mutex> lock(g_host_mutex);
            auto it = g_host_runs.find(ptr);
            if (it != g_host_runs.end())
            {
                runs = it->second;
                g_host_runs.erase(it);
            }
        }
        for (void* r : runs) ghexb::check_cuda(cudaHostUnregister(r), "cudaHostUnregister");
    });
}

// ---- communication object --------------------------------------------------------------------
int ghexb_co_create(ghexb_context ctx, ghexb_co* out)
{
    return guarded([&] {
        require(ctx && out, "null argument");
        auto co = std::make_unique<ghexb_co_s>();
        co->ctx = ctx;
        *out = co.release();
    });
}

int ghexb_co_create_ipr(ghexb_context ctx, ghexb_co* out)
{
    return guarded([&] {
        require(ctx && out, "null argument");
        auto co = std::make_unique<ghexb_co_s>();
        co->ctx = ctx;
        co->in_place_receive = true;
        *out = co.release();
    });
}

int ghexb_co_destroy(ghexb_co co)
{
    if (!co) return GHEXB_OK;
    if (co->done)
    {
        cudaEventSynchronize(co->done);
        cudaEventDestroy(co->done);
    }
    delete co;
    return GHEXB_OK;
}

int ghexb_co_exchange(ghexb_co co, const ghexb_field* fields, int n, void* stream, ghexb_handle* out)
{
    return guarded([&] {
        require(co && fields && out, "null argument");
        require(n > 0, "an exchange needs at least one field");
        for (int i = 0; i < n; ++i) require(fields[i] != nullptr, "null field handle");
        if (co->busy) throw ghexb::error(GHEXB_ERR_BUSY, "earlier exchange operation was not finished");
        auto key = signature(fields, n);
        auto it = co->plans.find(key);
        if (it == co->plans.end())
        {
            if (co->plans.size() >= 64) co->plans.clear();
            auto plan = std::make_unique<ghexb_plan_s>();
            plan->in_place_receive = co->in_place_receive;
            ghexb::build_plan(*plan, co->ctx, fields, n);
            it = co->plans.emplace(std::move(key), std::move(plan)).first;
        }
        if (!co->done) ghexb::check_cuda(cudaEventCreateWithFlags(&co->done, cudaEventDisableTiming), "cudaEventCreate");
        auto s = static_cast<cudaStream_t>(stream);
        ghexb::graph_launch_plan(*it->second, s);
        ghexb::check_cuda(cudaEventRecord(co->done, s), "cudaEventRecord");
        co->busy = true;
        auto h = std::make_unique<ghexb_handle_s>();
        h->co = co;
        *out = h.release();
    });
}

int ghexb_handle_wait(ghexb_handle h)
{
    return guarded([&] {
        require(h != nullptr, "null handle");
        if (h->co) h->co->wait();
    });
}

int ghexb_handle_is_ready(ghexb_handle h, int* ready)
{
    return guarded([&] {
        require(h && ready, "null argument");
        *ready = h->co ? (h->co->ready() ? 1 : 0) : 1;
    });
}

int ghexb_handle_destroy(ghexb_handle h)
{
    delete h;
    return GHEXB_OK;
}

// ---- plans -----------------------------------------------------------------------------------
int ghexb_plan_create(ghexb_context ctx, const ghexb_field* fields, int n, ghexb_plan* out)
{
    return guarded([&] {
        require(ctx && fields && out, "null argument");
        auto plan = std::make_unique<ghexb_plan_s>();
        ghexb::build_plan(*plan, ctx, fields, n);
        *out = plan.release();
    });
}

int ghexb_plan_create_ipr(ghexb_context ctx, const ghexb_field* fields, int n, ghexb_plan* out)
{
    return guarded([&] {
        require(ctx && fields && out, "null argument");
        auto plan = std::make_unique<ghexb_plan_s>();
        plan->in_place_receive = true;
        ghexb::build_plan(*plan, ctx, fields, n);
        *out = plan.release();
    });
}

int ghexb_plan_create_sharded(ghexb_context ctx, const ghexb_field* fields, int n, const unsigned char* local, int mode,
    ghexb_plan* out)
{
    return guarded([&] {
        require(ctx && fields && local && out, "null argument");
        require(n > 0, "an exchange needs at least one field");
        auto plan = std::make_unique<ghexb_plan_s>();
        plan->shard_mode = mode;
        plan->shard_local.assign(local, local + n);
        ghexb::build_plan(*plan, ctx, fields, n);
        *out = plan.release();
    });
}

namespace
{
// host replay of every table of a plan (all staged modes and adjoint tile sizes)
int64_t check_all(ghexb_plan_s& plan)
{
    // every staged mode at two stage sizes (host geometry only), then the element kernel alone
    plan.encode_maps = false;
    if (plan.shard_mode == 0)
        for (int mode : {1, 2})
            for (int bytes : {16384, 4096})
            {
                plan.staged_mode = mode, plan.stage_bytes = bytes;
                (void)ghexb::check_tables(plan);
            }
    plan.staged_mode = 0;
    // every size of the adjoint's gather tiles
    for (int scale : {-1, 1, 2})
    {
        plan.gather_scale = scale;
        (void)ghexb::check_tables(plan);
    }
    plan.gather_scale = 0;
    // the bulk kernel taking none and half of the lists (all of them below), and the bulk gather
    // kernel taking half and all of the unstructured owners
    for (int share : {0, 2})
    {
        plan.bulk_share = share;
        (void)ghexb::check_tables(plan);
    }
    plan.bulk_share = 4;
    for (int share : {2, 4})
    {
        plan.gather_bulk = share;
        (void)ghexb::check_tables(plan);
    }
    plan.gather_bulk = 0;
    const int64_t n = ghexb::check_tables(plan);
    if (plan.shard_mode == 0) ghexb::check_relocation(plan);
    return n;
}
} // namespace

int ghexb_plan_check_sharded(ghexb_context ctx, const ghexb_field* fields, int n, const unsigned char* local, int mode,
    int64_t* elements_checked)
{
    return guarded([&] {
        require(ctx && fields && local && elements_checked, "null argument");
        require(n > 0, "an exchange needs at least one field");
        ghexb_plan_s plan;
        plan.shard_mode = mode;
        plan.shard_local.assign(local, local + n);
        ghexb::build_tables(plan, ctx, fields, n);
        (void)check_all(plan);
        *elements_checked = plan.halo_elements;
    });
}

int ghexb_ipc_export(const void* ptr, unsigned char* handle, int64_t* offset)
{
    return guarded([&] {
        require(ptr && handle && offset, "null argument");
        ghexb::ipc_export(ptr, handle, offset);
    });
}

int ghexb_ipc_open(const unsigned char* handle, int64_t offset, void** ptr)
{
    return guarded([&] {
        require(handle && ptr, "null argument");
        *ptr = ghexb::ipc_open(handle, offset);
    });
}

int ghexb_ipc_close(const unsigned char* handle)
{
    return guarded([&] {
        require(handle != nullptr, "null argument");
        ghexb::ipc_close(handle);
    });
}

int ghexb_plan_check(ghexb_context ctx, const ghexb_field* fields, int n, int64_t* elements_checked)
{
    return guarded([&] {
        require(ctx && fields && elements_checked, "null argument");
        ghexb_plan_s plan;
        ghexb::build_tables(plan, ctx, fields, n);
        *elements_checked = check_all(plan);
    });
}

int ghexb_plan_dram_floor(ghexb_context ctx, const ghexb_field* fields, int n, int sector_bytes, int64_t* read_bytes,
    int64_t* write_bytes)
{
    return guarded([&] {
        require(ctx && fields && read_bytes && write_bytes, "null argument");
        require(sector_bytes >= 16, "the sector size must be at least 16 bytes");
        ghexb_plan_s plan;
        ghexb::build_tables(plan, ctx, fields, n);
        ghexb::dram_floor(plan, sector_bytes, *read_bytes, *write_bytes);
    });
}

int ghexb_plan_destroy(ghexb_plan plan)
{
    delete plan;
    return GHEXB_OK;
}

int ghexb_plan_get_info(ghexb_plan plan, ghexb_plan_info_t* info)
{
    return guarded([&] {
        require(plan && info, "null argument");
        info->num_fields = (int64_t)plan->fields.size();
        info->num_descriptors = (int64_t)(plan->boxes.size() + plan->lists.size());
        info->num_tiles = plan->num_tiles();
        info->halo_elements = plan->halo_elements;
        info->algorithmic_bytes = plan->algorithmic_bytes;
        info->index_bytes = plan->index_bytes;
        info->adjoint_launches = plan->adjoint_launches();
        info->adjoint_cells = plan->gather_ok ? (int64_t)plan->cells.size() : 0;
        info->elems_per_thread = plan->per_thread;
        info->block = plan->block;
        info->grid = (int32_t)plan->xf.size();
        info->pairs = (int32_t)plan->pairs.size();
        info->use_pairs = plan->use_pairs ? 1 : 0;
        info->staged_mode = plan->staged_mode;
        int staged = 0;
        for (char c : plan->box_staged) staged += c != 0;
        info->staged_boxes = staged;
        info->staged_items = (int32_t)plan->sitems.size();
        info->staged_maps = (int32_t)plan->smaps.size();
        info->stages = plan->stages;
        info->stage_bytes = plan->stage_bytes;
        info->stage_consumers = plan->stage_consumers;
        info->stage_ctas_per_sm = plan->stage_ctas_per_sm;
        info->gather_scale = plan->gather_scale;
        info->bulk_share = plan->bulk_share;
        info->bulk_tiles = (int32_t)plan->bt.size();
        info->gather_bulk = plan->gather_bulk;
        info->gather_bulk_tiles = (int32_t)plan->bgt.size();
    });
}

int ghexb_plan_set_tuning(ghexb_plan plan, int elems_per_thread, int block, int use_pairs)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        if (elems_per_thread > 0)
        {
            require(elems_per_thread == 4 || elems_per_thread == 8 || elems_per_thread == 16,
                "elements per thread must be 4, 8 or 16");
            plan->per_thread = elems_per_thread;
        }
        if (block > 0)
        {
            require(block % 32 == 0 && block <= ghexb::k_max_block, "block must be a multiple of 32 and at most 512");
            plan->block = block;
        }
        if (use_pairs >= 0) plan->use_pairs = use_pairs != 0;
        ghexb::retile(*plan);
        ghexb::check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize");
    });
}

int ghexb_plan_set_staged(ghexb_plan plan, int mode, int stages, int stage_bytes, int consumers, int ctas_per_sm)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        require(mode <= 2, "staged mode must be 0, 1 or 2");
        require(stages <= 16, "at most 16 stages");
        require(stage_bytes <= 0 || (stage_bytes % 128 == 0 && stage_bytes <= 64 * 1024),
            "stage bytes must be a multiple of 128 and at most 64 KiB");
        require(consumers <= 8, "at most 8 consumer warps");
        require(ctas_per_sm <= 4, "at most 4 staged CTAs per SM");
        const int st = stages > 0 ? stages : plan->stages, sb = stage_bytes > 0 ? stage_bytes : plan->stage_bytes;
        require(st >= 2, "at least 2 stages");
        require((size_t)st * sb + 128 <= 227 * 1024, "stages x stage bytes exceed the shared memory of a CTA");
        require(mode <= 0 || plan->shard_mode == 0, "a sharded plan has no staged form");
        if (mode >= 0) plan->staged_mode = mode;
        plan->stages = st, plan->stage_bytes = sb;
        if (consumers > 0) plan->stage_consumers = consumers;
        if (ctas_per_sm > 0) plan->stage_ctas_per_sm = ctas_per_sm;
        ghexb::retile(*plan);
        ghexb::check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize");
    });
}

int ghexb_plan_set_bulk(ghexb_plan plan, int share)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        require(share >= 0 && share <= 4, "bulk share must be 0 to 4 quarters");
        plan->bulk_share = share;
        ghexb::retile(*plan);
        ghexb::check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize");
    });
}

int ghexb_plan_set_adjoint_bulk(ghexb_plan plan, int share)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        require(share >= 0 && share <= 4, "adjoint bulk share must be 0 to 4 quarters");
        plan->gather_bulk = share;
        ghexb::retile(*plan);
        ghexb::check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize");
    });
}

int ghexb_plan_set_adjoint_tuning(ghexb_plan plan, int gather_scale)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        require(gather_scale >= -1 && gather_scale <= 2, "gather scale must be -1, 0, 1 or 2");
        plan->gather_scale = gather_scale;
        ghexb::retile(*plan);
        ghexb::check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize");
    });
}

int ghexb_plan_staged_status(ghexb_plan plan, unsigned* status)
{
    return guarded([&] {
        require(plan && status, "null argument");
        *status = 0;
        if (!plan->d_status) return;
        ghexb::check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        ghexb::check_cuda(cudaMemcpy(status, plan->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost), "cudaMemcpy(status)");
        ghexb::check_cuda(cudaMemset(plan->d_status, 0, sizeof(unsigned)), "cudaMemset(status)");
    });
}

int ghexb_plan_launch(ghexb_plan plan, int form, void* stream)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        ghexb::launch_plan(*plan, form, static_cast<cudaStream_t>(stream));
    });
}

int ghexb_plan_graph_launch(ghexb_plan plan, void* stream)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        ghexb::graph_launch_plan(*plan, static_cast<cudaStream_t>(stream));
    });
}

int ghexb_plan_adjoint_launch(ghexb_plan plan, void* stream)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        ghexb::adjoint_plan(*plan, static_cast<cudaStream_t>(stream));
    });
}

int ghexb_plan_rebind(ghexb_plan plan, void* const* data, int n, void* stream)
{
    return guarded([&] {
        require(plan && data, "null argument");
        ghexb::rebind_plan(*plan, data, n, static_cast<cudaStream_t>(stream));
    });
}

int ghexb_plan_autotune(ghexb_plan plan, void* stream, int repeats, ghexb_plan_info_t* info)
{
    return guarded([&] {
        require(plan != nullptr, "null plan");
        ghexb::autotune_plan(*plan, static_cast<cudaStream_t>(stream), repeats);
        if (info)
        {
            const int rc = ghexb_plan_get_info(plan, info);
            if (rc != GHEXB_OK) throw ghexb::error(rc, g_last_error);
        }
    });
}

int ghexb_calibrate_rows(const void* src, void* dst, int64_t rows, int n, int64_t src_stride, int64_t dst_stride,
    int elem_bytes, int mode, void* stream)
{
    return guarded([&] {
        require(src && dst, "null argument");
        require(mode >= 0 && mode <= 2, "mode 0 (copy), 1 (read only) or 2 (write only)");
        require(rows >= 1 && rows < (int64_t(1) << 32) && n >= 1 && n <= 256, "rows or row length out of range");
        require(elem_bytes == 4 || elem_bytes == 8, "elements of 4 or 8 bytes");
        require(src_stride >= n && dst_stride >= n, "row strides shorter than the rows");
        ghexb::check_accessible(src, (size_t)((rows - 1) * src_stride + n) * elem_bytes);
        ghexb::check_accessible(dst, (size_t)((rows - 1) * dst_stride + n) * elem_bytes);
        ghexb::check_cuda(ghexb::launch_row_copy(src, dst, (uint32_t)rows, (uint32_t)n, src_stride, dst_stride, elem_bytes,
                              mode, static_cast<cudaStream_t>(stream)),
            "row copy launch");
    });
}

int ghexb_stencil7(int dtype, int n, const void* const* in, void* const* out, const int64_t* extents,
                   const int64_t* strides, int halo, double alpha, int adjoint, void* stream)
{
    return guarded([&] {
        require(in && out && extents && strides, "null argument");
        require(dtype == GHEXB_F32 || dtype == GHEXB_F64, "the stencil computes in float32 or float64");
        require(n >= 0, "negative domain count");
        require(halo >= 1, "the 7-point stencil needs a halo of width >= 1");
        const int64_t es = dtype == GHEXB_F64 ? 8 : 4;
        std::vector<ghexb::stencil_domain> doms(n);
        for (int i = 0; i < n; ++i)
        {
            require(in[i] && out[i], "null data pointer");
            require(reinterpret_cast<uintptr_t>(in[i]) % es == 0 && reinterpret_cast<uintptr_t>(out[i]) % es == 0,
                "data pointer not aligned to its element size");
            int64_t span = 1;
            for (int a = 0; a < 3; ++a)
            {
                require(extents[3 * i + a] > 2 * halo && extents[3 * i + a] < (int64_t(1) << 30),
                    "every extent must exceed twice the halo width");
                require(strides[3 * i + a] > 0, "strides must be positive");
                span += (extents[3 * i + a] - 1) * strides[3 * i + a];
            }
            const char* a0 = static_cast<const char*>(in[i]);
            const char* b0 = static_cast<const char*>(out[i]);
            require(a0 + span * es <= b0 || b0 + span * es <= a0, "input and output overlap");
            doms[i] = ghexb::stencil_domain{in[i], out[i], (int32_t)extents[3 * i], (int32_t)extents[3 * i + 1],
                (int32_t)extents[3 * i + 2], halo, strides[3 * i], strides[3 * i + 1], strides[3 * i + 2]};
        }
        if (n == 0) return;
        ghexb::check_cuda(ghexb::launch_stencil7(dtype == GHEXB_F64, doms.data(), n, alpha, adjoint != 0,
                              static_cast<cudaStream_t>(stream)),
            "stencil launch");
    });
}

} // extern "C"

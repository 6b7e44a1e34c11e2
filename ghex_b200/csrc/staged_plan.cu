// Host side of the staged form: which boxes the staged kernel takes, their tensor maps and work
// items, the replay check of every item element, and the launch beside the element kernel.
//
// A box descriptor copies dst[i0*d0 + i1*d1 + i2*d2] = src[i0*s0 + i1*s1 + i2*s2] (descriptors.hpp).
// The staged kernel needs source rows that are contiguous in memory and a destination axis with
// unit stride to write along:
//  * rows:       s0 = 1 and d0 = 1 (the source and destination rows run along the same axis);
//  * transposed: |s1| = 1 and d0 = 1 (the source rows run along the destination's second axis, as
//                on cubed-sphere edges whose transform swaps x and y).
// The source region is then a 3-D lattice: X (contiguous), R (rows) and P (planes). Negative
// strides are turned positive by starting the region at its lowest address (the destination
// strides change sign instead). Rows i_R = a (mod p) and planes i_P = b (mod q) form a class with
// strides p*|sR| and q*|sP| bytes, multiples of 16 as a tensor map needs; each class is one map
// whose extents are exactly the class's rows and planes and the region's X extent plus the
// elements before it down to a 16-byte boundary, so a load box reaching past the class is filled
// without reading memory.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "plan.hpp"

namespace ghexb
{
namespace
{
constexpr int k_max_box = 256; // elements of a tensor-map load box per dimension

CUtensorMapDataType map_type(int es)
{
    switch (es)
    {
        case 1: return CU_TENSOR_MAP_DATA_TYPE_UINT8;
        case 2: return CU_TENSOR_MAP_DATA_TYPE_UINT16;
        case 4: return CU_TENSOR_MAP_DATA_TYPE_UINT32;
        default: return CU_TENSOR_MAP_DATA_TYPE_UINT64;
    }
}

struct lattice
{
    int64_t n[3];  // X, R, P extents
    int64_t s[3];  // source element strides (made positive)
    int64_t d[3];  // destination element strides (sign follows the source's flip)
    int64_t src0;  // source element offset of the region's lowest element, from b.src
    int64_t dst0;  // destination element offset of that element, from b.dst
    bool transposed;
};

// The box as a source lattice, or false when the staged kernel cannot take it.
bool as_lattice(const box_desc& b, lattice& L)
{
    int ax[3];
    if (b.s0 == 1 && b.d0 == 1)
        ax[0] = 0, ax[1] = 1, ax[2] = 2, L.transposed = false;
    else if ((b.s1 == 1 || b.s1 == -1) && b.d0 == 1 && b.n1 > 1)
        ax[0] = 1, ax[1] = 0, ax[2] = 2, L.transposed = true;
    else
        return false;
    const int64_t n[3] = {b.n0, b.n1, b.n2}, s[3] = {b.s0, b.s1, b.s2}, d[3] = {b.d0, b.d1, b.d2};
    L.src0 = 0, L.dst0 = 0;
    for (int k = 0; k < 3; ++k)
    {
        const int a = ax[k];
        L.n[k] = n[a], L.s[k] = s[a], L.d[k] = d[a];
        if (L.s[k] < 0)
        {
            L.src0 += (L.n[k] - 1) * L.s[k];
            L.dst0 += (L.n[k] - 1) * L.d[k];
            L.s[k] = -L.s[k], L.d[k] = -L.d[k];
        }
    }
    return L.s[0] == 1;
}

int period(int64_t stride_bytes, int64_t extent)
{
    if (extent <= 1) return 1;
    return (int)(16 / std::gcd<int64_t>(stride_bytes % 16 == 0 ? 16 : stride_bytes % 16, 16));
}

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
} // namespace

void build_staged(ghexb_plan_s& plan)
{
    plan.box_staged.assign(plan.boxes.size(), 0);
    plan.smaps.clear();
    plan.smap_host.clear();
    plan.sitems.clear();
    plan.sitem_box.clear();
    if (plan.staged_mode <= 0) return;
    const int64_t stage = plan.stage_bytes;
    struct pending
    {
        sitem it;
        int box;
    };
    std::vector<pending> items;
    for (size_t i = 0; i < plan.boxes.size(); ++i)
    {
        const box_desc& b = plan.boxes[i];
        const ghexb_field_s& sf = plan.fields[plan.box_src_slot[i]];
        if (plan.field_on_device.size() == plan.fields.size() &&
            (!plan.field_on_device[plan.box_src_slot[i]] || !plan.field_on_device[plan.box_dst_slot[i]]))
            continue; // host fields stay on the element kernel
        if (reinterpret_cast<uintptr_t>(sf.data) % 16) continue;
        lattice L;
        if (!as_lattice(b, L)) continue;
        const int es = (int)b.esize;
        const int64_t al = 16 / es; // elements per 16 bytes
        if (L.n[0] + al - 1 > k_max_box) continue;
        if (plan.staged_mode == 1 && !L.transposed && L.n[0] * es > 64) continue;
        const int p = period(L.s[1] * es, L.n[1]), q = period(L.s[2] * es, L.n[2]);
        // every class's load box must fit a stage
        if (round_up(L.n[0] + al - 1, al) * es > stage) continue;
        plan.box_staged[i] = 1;
        for (int a = 0; a < std::min<int64_t>(p, L.n[1]); ++a)
            for (int c = 0; c < std::min<int64_t>(q, L.n[2]); ++c)
            {
                const int64_t rows = (L.n[1] - a + p - 1) / p, planes = (L.n[2] - c + q - 1) / q;
                const char* origin = b.src + (L.src0 + a * L.s[1] + c * L.s[2]) * es;
                const int64_t delta = (int64_t)(reinterpret_cast<uintptr_t>(origin) % 16) / es;
                const char* base = origin - delta * es;
                const int64_t w = round_up(delta + L.n[0], al);
                const int64_t h = std::min<int64_t>({rows, k_max_box, std::max<int64_t>(1, stage / (w * es))});
                const int64_t dd = std::min<int64_t>({planes, k_max_box, std::max<int64_t>(1, stage / (w * es * h))});
                const int64_t rstride = rows > 1 ? p * L.s[1] * es : round_up(w * es, 16);
                const int64_t pstride = planes > 1 ? q * L.s[2] * es : rstride * rows;
                ghexb_plan_s::smap_info mi{base, {delta + L.n[0], rows, planes}, {rstride, pstride}, es, (int)w, (int)h,
                    (int)dd, plan.box_src_slot[i]};
                CUtensorMap m;
                std::memset(&m, 0, sizeof m);
                if (plan.encode_maps)
                {
                    const cuuint64_t dims[3] = {(cuuint64_t)mi.dims[0], (cuuint64_t)rows, (cuuint64_t)planes};
                    const cuuint64_t strides[2] = {(cuuint64_t)rstride, (cuuint64_t)pstride};
                    const cuuint32_t box[3] = {(cuuint32_t)w, (cuuint32_t)h, (cuuint32_t)dd};
                    const CUresult r = encode_tensor_map(&m, map_type(es), 3, const_cast<char*>(base), dims, strides, box,
                        w * es <= 64 ? CU_TENSOR_MAP_L2_PROMOTION_NONE : CU_TENSOR_MAP_L2_PROMOTION_L2_128B);
                    if (r != CUDA_SUCCESS)
                        throw error(GHEXB_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) +
                                                        ") for box " + std::to_string(i));
                }
                const uint32_t map_index = (uint32_t)plan.smaps.size();
                plan.smaps.push_back(m);
                plan.smap_host.push_back(mi);
                for (int64_t j0 = 0; j0 < rows; j0 += h)
                    for (int64_t z0 = 0; z0 < planes; z0 += dd)
                    {
                        const int64_t nr = std::min(h, rows - j0), nz = std::min(dd, planes - z0);
                        sitem it{};
                        const int64_t first = L.dst0 + (a + p * j0) * L.d[1] + (c + q * z0) * L.d[2];
                        it.dst = b.dst + first * es;
                        it.map = map_index;
                        it.c1 = (int32_t)j0, it.c2 = (int32_t)z0;
                        it.bytes = (uint32_t)(w * h * dd * es);
                        it.sbase = (uint32_t)delta;
                        it.sz = (uint32_t)(w * h);
                        it.dz = (int32_t)(q * L.d[2]);
                        int64_t nu, nv;
                        if (!L.transposed)
                        {
                            // u along X (the destination's unit stride), v along the class rows
                            nu = L.n[0], nv = nr;
                            it.su = 1, it.sv = (uint32_t)w;
                            it.du = (int32_t)L.d[0], it.dv = (int32_t)(p * L.d[1]);
                        }
                        else
                        {
                            // u along the class rows (the destination's unit stride), v along X
                            nu = nr, nv = L.n[0];
                            it.su = (uint32_t)w, it.sv = 1;
                            it.du = (int32_t)(p * L.d[1]), it.dv = (int32_t)L.d[0];
                        }
                        const fast_div fu = fast_div::make((uint32_t)nu), fv = fast_div::make((uint32_t)nv);
                        it.nu = fu.d, it.mu = fu.m, it.lu = (uint8_t)fu.l;
                        it.nv = fv.d, it.mv = fv.m, it.lv = (uint8_t)fv.l;
                        it.count = (uint32_t)(nu * nv * nz);
                        it.es = (uint8_t)es;
                        it.neg = b.xor_mask != 0;
                        items.push_back({it, (int)i});
                    }
            }
    }
    // the largest loads first: with items dealt round-robin to the CTAs, each CTA gets a share of
    // every size
    std::stable_sort(items.begin(), items.end(), [](const pending& x, const pending& y) { return x.it.bytes > y.it.bytes; });
    for (const auto& pi : items)
    {
        plan.sitems.push_back(pi.it);
        plan.sitem_box.push_back(pi.box);
    }
}

int64_t check_staged(const ghexb_plan_s& plan)
{
    int64_t checked = 0;
    std::vector<std::vector<std::pair<const char*, const char*>>> got(plan.boxes.size());
    for (size_t k = 0; k < plan.sitems.size(); ++k)
    {
        const sitem& it = plan.sitems[k];
        const int bi = plan.sitem_box[k];
        const box_desc& b = plan.boxes[bi];
        if (it.map >= plan.smap_host.size()) throw error(GHEXB_ERR_INTERNAL, "staged item names no tensor map");
        const auto& m = plan.smap_host[it.map];
        if ((int64_t)m.w * m.h * m.d * m.es != it.bytes || it.bytes > (uint32_t)plan.stage_bytes)
            throw error(GHEXB_ERR_INTERNAL, "staged item bytes differ from its load box");
        if (it.es != b.esize || m.slot != plan.box_src_slot[bi]) throw error(GHEXB_ERR_INTERNAL, "staged item of the wrong field");
        const char* fsrc = plan.fields[m.slot].data;
        const char* fdst = plan.fields[plan.box_dst_slot[bi]].data;
        const int64_t sspan = (int64_t)field_bytes(plan.fields[m.slot]);
        const int64_t dspan = (int64_t)field_bytes(plan.fields[plan.box_dst_slot[bi]]);
        for (uint32_t e = 0; e < it.count; ++e)
        {
            const uint32_t q = fast_div{it.nu, it.mu, it.lu}.div(e);
            const uint32_t u = e - q * it.nu;
            const uint32_t z = fast_div{it.nv, it.mv, it.lv}.div(q);
            const uint32_t v = q - z * it.nv;
            const int64_t sidx = (int64_t)it.sbase + (int64_t)u * it.su + (int64_t)v * it.sv + (int64_t)z * it.sz;
            // the shared-memory element as load-box coordinates, which must lie inside the map
            const int64_t x = sidx % m.w, j = (sidx / m.w) % m.h, zz = sidx / ((int64_t)m.w * m.h);
            if (zz >= m.d) throw error(GHEXB_ERR_INTERNAL, "staged element beyond its load box");
            if (x >= m.dims[0] || it.c1 + j >= m.dims[1] || it.c2 + zz >= m.dims[2])
                throw error(GHEXB_ERR_INTERNAL, "staged element outside its tensor map (a filled element)");
            const char* src = m.base + x * m.es + (it.c1 + j) * m.strides[0] + (it.c2 + zz) * m.strides[1];
            const char* dst = it.dst + ((int64_t)u * it.du + (int64_t)v * it.dv + (int64_t)z * it.dz) * it.es;
            if (src < fsrc || src + m.es > fsrc + sspan) throw error(GHEXB_ERR_RANGE, "staged source outside its field");
            if (dst < fdst || dst + it.es > fdst + dspan) throw error(GHEXB_ERR_RANGE, "staged destination outside its field");
            if (reinterpret_cast<uintptr_t>(m.base) % 16 || m.strides[0] % 16 || m.strides[1] % 16)
                throw error(GHEXB_ERR_INTERNAL, "tensor map base or stride not 16-byte aligned");
            got[bi].emplace_back(dst, src);
            ++checked;
        }
    }
    // every staged box's elements, each once, with the box's own source for its destination
    for (size_t i = 0; i < plan.boxes.size(); ++i)
    {
        if (!plan.box_staged.empty() && plan.box_staged[i])
        {
            const box_desc& b = plan.boxes[i];
            std::vector<std::pair<const char*, const char*>> want;
            for (int32_t i2 = 0; i2 < b.n2; ++i2)
                for (int32_t i1 = 0; i1 < b.n1; ++i1)
                    for (int32_t i0 = 0; i0 < b.n0; ++i0)
                        want.emplace_back(b.dst + ((int64_t)i0 * b.d0 + (int64_t)i1 * b.d1 + (int64_t)i2 * b.d2) * b.esize,
                            b.src + ((int64_t)i0 * b.s0 + (int64_t)i1 * b.s1 + (int64_t)i2 * b.s2) * b.esize);
            std::sort(want.begin(), want.end());
            std::sort(got[i].begin(), got[i].end());
            if (want != got[i]) throw error(GHEXB_ERR_INTERNAL, "staged items differ from box " + std::to_string(i));
        }
        else if (!got[i].empty())
            throw error(GHEXB_ERR_INTERNAL, "staged items of a box that is not staged");
    }
    return checked;
}

void ensure_side_stream(ghexb_plan_s& plan)
{
    if (plan.side_stream) return;
    check_cuda(cudaStreamCreateWithFlags(&plan.side_stream, cudaStreamNonBlocking), "cudaStreamCreate(side)");
    check_cuda(cudaEventCreateWithFlags(&plan.fork_event, cudaEventDisableTiming), "cudaEventCreate(fork)");
    check_cuda(cudaEventCreateWithFlags(&plan.join_event, cudaEventDisableTiming), "cudaEventCreate(join)");
}

void launch_staged_plan(ghexb_plan_s& plan, cudaStream_t stream)
{
    if (plan.sitems.empty()) return;
    ensure_side_stream(plan);
    staged_launch a{};
    a.items = plan.d_sitems;
    a.maps = plan.d_smaps;
    a.status = plan.d_status;
    a.nitems = (int)plan.sitems.size();
    a.stages = plan.stages;
    a.stage_bytes = plan.stage_bytes;
    a.consumers = plan.stage_consumers;
    a.grid = std::max(1, std::min(a.nitems, (plan.ctx ? plan.ctx->num_sms : 148) * plan.stage_ctas_per_sm));
    check_cuda(staged_prepare(a.stages * a.stage_bytes + 128), "staged kernel shared memory");
    check_cuda(cudaEventRecord(plan.fork_event, stream), "cudaEventRecord(fork)");
    check_cuda(cudaStreamWaitEvent(plan.side_stream, plan.fork_event, 0), "cudaStreamWaitEvent(fork)");
    check_cuda(launch_staged(a, plan.side_stream), "staged kernel launch");
    check_cuda(cudaEventRecord(plan.join_event, plan.side_stream), "cudaEventRecord(join)");
}
} // namespace ghexb

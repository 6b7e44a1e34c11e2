// Lowering of a field set into the work-descriptor table, tiling, adjoint phases, launches,
// graph capture and autotuning.
//
// Field matching follows communication_object::allocate (communication_object.hpp:558-624): the
// message between two domains carries their fields in argument order, so the k-th field given
// for a receiving domain pairs with the k-th field given for the sending domain of the same
// pattern. The fused form copies each halo element straight from the sender's interior
// (structured/regular/field_descriptor.hpp:72-96 packs it into a buffer, :85-96 unpacks it) to
// the receiver's halo; the cubed-sphere unpack transform and component negation
// (structured/cubed_sphere/field_descriptor.hpp:80-108,142-167) become signed source strides and
// a sign-bit mask; the unstructured gather/scatter (unstructured/user_concepts.hpp:549-581)
// becomes one index-list descriptor per neighbour pair.
#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <tuple>
#include <unordered_map>
#include <unordered_set>

#include "exchange.hpp"
#include "kernels.hpp"
#include "plan.hpp"

namespace ghexb
{
void check_cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
        throw error(GHEXB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace
{
constexpr int64_t k_i32max = 0x7fffffffLL;

// Host-to-device copies of a plan's tables, stream-ordered, through the plan's page-locked
// staging buffers: put() queues a copy; commit() takes the next buffer of the ring, waits until
// the copies of its previous use have left it, packs the queued tables into it and issues the
// copies on `stream`.
class host_stager
{
  public:
    host_stager(ghexb_plan_s& plan, cudaStream_t stream)
    : m_plan(plan)
    , m_stream(stream)
    {
    }
    template<typename T>
    void put(T* dptr, const std::vector<T>& v)
    {
        if (!v.empty()) m_q.push_back({dptr, v.data(), v.size() * sizeof(T)});
    }
    void commit()
    {
        size_t total = 0;
        for (const auto& c : m_q) total += (c.bytes + 255) / 256 * 256;
        if (total == 0) return;
        auto& B = m_plan.h_stage[m_plan.h_stage_next];
        m_plan.h_stage_next = (m_plan.h_stage_next + 1) % 4;
        if (B.done) check_cuda(cudaEventSynchronize(B.done), "cudaEventSynchronize(staging)");
        else
            check_cuda(cudaEventCreateWithFlags(&B.done, cudaEventDisableTiming), "cudaEventCreate(staging)");
        if (total > B.cap)
        {
            if (B.ptr) cudaFreeHost(B.ptr), B.ptr = nullptr, B.cap = 0;
            check_cuda(cudaMallocHost(&B.ptr, total), "cudaMallocHost(plan staging)");
            B.cap = total;
        }
        char* buf = static_cast<char*>(B.ptr);
        size_t off = 0;
        for (const auto& c : m_q)
        {
            std::memcpy(buf + off, c.src, c.bytes);
            check_cuda(cudaMemcpyAsync(c.dst, buf + off, c.bytes, cudaMemcpyHostToDevice, m_stream),
                "cudaMemcpyAsync(plan table)");
            off += (c.bytes + 255) / 256 * 256;
        }
        check_cuda(cudaEventRecord(B.done, m_stream), "cudaEventRecord(staging)");
        m_q.clear();
    }

  private:
    struct copy
    {
        void* dst;
        const void* src;
        size_t bytes;
    };
    ghexb_plan_s& m_plan;
    cudaStream_t m_stream;
    std::vector<copy> m_q;
};

template<typename T>
void upload(T*& dptr, const std::vector<T>& v, host_stager& st)
{
    if (dptr) cudaFree(dptr), dptr = nullptr;
    if (v.empty()) return;
    check_cuda(cudaMalloc(&dptr, v.size() * sizeof(T)), "cudaMalloc(plan table)");
    st.put(dptr, v);
}

// One axis of a box: extent, first source/destination coordinates in field memory and the
// element strides the axis moves by.
struct axis
{
    int n;
    int64_t ss, ds;   // element strides
    int order;        // destination layout value (larger = faster)
};

struct owner_region
{
    int field;
    std::array<int64_t, 4> lo, hi; // source-field coordinates (inclusive)
};

struct builder
{
    ghexb_plan_s& plan;
    std::vector<owner_region> box_owner;  // per box desc, source region for adjoint phases
    std::vector<int> list_src_field;      // per adjoint list desc

    explicit builder(ghexb_plan_s& p)
    : plan(p)
    {
    }

    static int64_t estride(const ghexb_field_s& f, int a)
    {
        return f.byte_strides[a] / f.esize;
    }

    // Emits box descriptors from a list of axes (any order) and the element offsets of the box
    // origin in source and destination. Rows longer than 256 elements are split.
    void emit_box(const ghexb_field_s& src, int src_slot, const ghexb_field_s& dst, int dst_slot,
        std::vector<axis> ax, int64_t src_origin, int64_t dst_origin, uint64_t xor_mask,
        int logical, const owner_region& reg)
    {
        std::stable_sort(ax.begin(), ax.end(), [](const axis& a, const axis& b) { return a.order > b.order; });
        while (ax.size() < 3) ax.push_back(axis{1, 0, 0, -1});
        if (ax.size() > 3) throw error(GHEXB_ERR_INTERNAL, "box descriptors are 3-dimensional");
        int64_t nelem = 1, sspan = 0, dspan = 0;
        for (const auto& a : ax)
        {
            if (a.n <= 0) return;
            nelem *= a.n;
            sspan += (int64_t)(a.n - 1) * (a.ss < 0 ? -a.ss : a.ss);
            dspan += (int64_t)(a.n - 1) * (a.ds < 0 ? -a.ds : a.ds);
        }
        if (nelem > k_i32max || sspan > k_i32max || dspan > k_i32max)
            throw error(GHEXB_ERR_RANGE, "a halo box spans more than 2^31 elements");
        constexpr int k_max_row = 256;
        for (int x0 = 0; x0 < ax[0].n; x0 += k_max_row)
        {
            box_desc b{};
            b.n0 = std::min(k_max_row, ax[0].n - x0);
            b.src = src.data + (src_origin + x0 * ax[0].ss) * src.esize;
            b.dst = dst.data + (dst_origin + x0 * ax[0].ds) * dst.esize;
            b.n1 = ax[1].n, b.n2 = ax[2].n;
            b.s0 = (int32_t)ax[0].ss, b.s1 = (int32_t)ax[1].ss, b.s2 = (int32_t)ax[2].ss;
            b.d0 = (int32_t)ax[0].ds, b.d1 = (int32_t)ax[1].ds, b.d2 = (int32_t)ax[2].ds;
            b.esize = (uint32_t)dst.esize;
            b.field = (uint32_t)logical;
            b.map = row_map::make(b.n0);
            b.xor_mask = xor_mask;
            b.div1 = fast_div::make((uint32_t)b.n1);
            plan.boxes.push_back(b);
            plan.box_src_slot.push_back(src_slot);
            plan.box_dst_slot.push_back(dst_slot);
            plan.box_src_off.push_back(b.src - src.data);
            plan.box_dst_off.push_back(b.dst - dst.data);
            box_owner.push_back(reg);
            box_owner.back().field = src_slot;
        }
        plan.halo_elements += nelem;
        plan.algorithmic_bytes += nelem * dst.esize * 2;
    }

    static void check_range(const ghexb_field_s& f, int a, int64_t lo, int64_t hi, const char* which)
    {
        if (lo < 0 || hi >= f.extents[a])
            throw error(GHEXB_ERR_RANGE,
                std::string(which) + " halo box exceeds the wrapped field memory along dimension " +
                    std::to_string(a) + " (coordinates " + std::to_string(lo) + ".." + std::to_string(hi) +
                    ", extent " + std::to_string(f.extents[a]) + ")");
    }

    void regular_space(const ghexb_pattern_s& P, int e, const ghexb_field_s& dst, int dst_slot,
        const ghexb_field_s& src, int src_slot, const space_pair& sp, int logical)
    {
        const int D = P.dim;
        const auto& sdom = P.domains[e];
        std::vector<axis> ax;
        int64_t so = 0, dof = 0;
        owner_region reg{};
        for (int a = 0; a < D; ++a)
        {
            const int64_t dl = sp.lfirst[a] + dst.offsets[a], dh = sp.llast[a] + dst.offsets[a];
            const int64_t sl = (sp.has_src ? sp.sfirst[a] : sp.gfirst[a] - sdom.first[a]) + src.offsets[a];
            const int64_t sh = sl + (sp.llast[a] - sp.lfirst[a]);
            check_range(dst, a, dl, dh, "destination");
            check_range(src, a, sl, sh, "source");
            dof += dl * estride(dst, a);
            so += sl * estride(src, a);
            ax.push_back(axis{(int)(dh - dl + 1), estride(src, a), estride(dst, a), dst.layout[a]});
            reg.lo[a] = sl, reg.hi[a] = sh;
        }
        if (dst.ndim == D + 1)
        {
            // one descriptor per component: the kernels walk 3-D boxes
            for (int c = 0; c < dst.num_components; ++c)
            {
                owner_region rc = reg;
                rc.lo[D] = rc.hi[D] = c;
                emit_box(src, src_slot, dst, dst_slot, ax, so + c * estride(src, D), dof + c * estride(dst, D), 0,
                    logical, rc);
            }
            return;
        }
        emit_box(src, src_slot, dst, dst_slot, ax, so, dof, 0, logical, reg);
    }

    void cubed_space(const ghexb_pattern_s& P, int d, int e, const ghexb_field_s& dst, int dst_slot,
        const ghexb_field_s& src, int src_slot, const space_pair& sp, int logical)
    {
        const auto& ddom = P.domains[d];
        const auto& sdom = P.domains[e];
        const int c = P.edge_size;
        const cs_transform* t = &cs_identity();
        if (sp.gfirst[0] != ddom.tile)
        {
            int n = 0;
            while (n < 4 && cs_neighbor_tile(ddom.tile, n) != sp.gfirst[0]) ++n;
            if (n == 4) throw error(GHEXB_ERR_INTERNAL, "receive space on a tile that is not a neighbour");
            t = &cs_forward(ddom.tile, n);
        }
        const auto& r = t->rot;
        // source local coordinate of destination local (x, y):
        //   sx = r0 x + r1 y + cx, sy = r2 x + r3 y + cy
        const int64_t cx = (int64_t)r[0] * ddom.first[1] + (int64_t)r[1] * ddom.first[2] +
                           (int64_t)t->trans[0] * c + t->off[0] - sdom.first[1];
        const int64_t cy = (int64_t)r[2] * ddom.first[1] + (int64_t)r[3] * ddom.first[2] +
                           (int64_t)t->trans[1] * c + t->off[1] - sdom.first[2];
        const int lx0 = sp.lfirst[1], lx1 = sp.llast[1], ly0 = sp.lfirst[2], ly1 = sp.llast[2];
        const int lz0 = sp.lfirst[3], lz1 = sp.llast[3];
        // bounds: destination box, and the source image of its four corners
        check_range(dst, 0, lx0 + dst.offsets[0], lx1 + dst.offsets[0], "destination");
        check_range(dst, 1, ly0 + dst.offsets[1], ly1 + dst.offsets[1], "destination");
        check_range(dst, 2, lz0 + dst.offsets[2], lz1 + dst.offsets[2], "destination");
        const int64_t zs = lz0 + (ddom.first[3] - sdom.first[3]);
        check_range(src, 2, zs + src.offsets[2], zs + (lz1 - lz0) + src.offsets[2], "source");
        int64_t sx_lo = INT64_MAX, sx_hi = INT64_MIN, sy_lo = INT64_MAX, sy_hi = INT64_MIN;
        for (int cx_i = 0; cx_i < 2; ++cx_i)
            for (int cy_i = 0; cy_i < 2; ++cy_i)
            {
                const int64_t x = cx_i ? lx1 : lx0, y = cy_i ? ly1 : ly0;
                const int64_t sx = r[0] * x + r[1] * y + cx, sy = r[2] * x + r[3] * y + cy;
                sx_lo = std::min(sx_lo, sx), sx_hi = std::max(sx_hi, sx);
                sy_lo = std::min(sy_lo, sy), sy_hi = std::max(sy_hi, sy);
            }
        check_range(src, 0, sx_lo + src.offsets[0], sx_hi + src.offsets[0], "source");
        check_range(src, 1, sy_lo + src.offsets[1], sy_hi + src.offsets[1], "source");

        const int64_t sX = estride(src, 0), sY = estride(src, 1), sZ = estride(src, 2), sC = estride(src, 3);
        const int64_t sx0 = r[0] * lx0 + r[1] * ly0 + cx, sy0 = r[2] * lx0 + r[3] * ly0 + cy;
        const int64_t src_origin = (sx0 + src.offsets[0]) * sX + (sy0 + src.offsets[1]) * sY + (zs + src.offsets[2]) * sZ;
        const int64_t dst_origin = (lx0 + dst.offsets[0]) * estride(dst, 0) +
                                   (ly0 + dst.offsets[1]) * estride(dst, 1) +
                                   (lz0 + dst.offsets[2]) * estride(dst, 2);
        std::vector<axis> ax{
            axis{lx1 - lx0 + 1, r[0] * sX + r[2] * sY, estride(dst, 0), dst.layout[0]},
            axis{ly1 - ly0 + 1, r[1] * sX + r[3] * sY, estride(dst, 1), dst.layout[1]},
            axis{lz1 - lz0 + 1, sZ, estride(dst, 2), dst.layout[2]},
        };
        owner_region reg{};
        reg.lo = {sx_lo + src.offsets[0], sy_lo + src.offsets[1], zs + src.offsets[2], 0};
        reg.hi = {sx_hi + src.offsets[0], sy_hi + src.offsets[1], zs + (lz1 - lz0) + src.offsets[2], 0};
        const int nc = dst.num_components;
        const uint64_t sign = dst.esize == 8 ? (1ull << 63) : (1ull << 31);
        const bool neg0 = dst.is_vector && r[2] == -1;
        const bool neg1 = dst.is_vector && r[1] == -1;
        for (int comp = 0; comp < nc; ++comp)
        {
            const uint64_t xm = (comp == 0 && neg0) || (comp == 1 && neg1) ? sign : 0;
            owner_region rc = reg;
            rc.lo[3] = rc.hi[3] = comp;
            emit_box(src, src_slot, dst, dst_slot, ax, src_origin + comp * sC, dst_origin + comp * estride(dst, 3),
                xm, logical, rc);
        }
    }

    void list_pair(const ghexb_field_s& dst, int dst_slot, const ghexb_field_s& src, int src_slot,
        const std::vector<int64_t>& R, const std::vector<int64_t>& S, int logical)
    {
        if (R.size() != S.size() || R.empty()) return;
        const int64_t cnt = (int64_t)R.size();
        const int64_t L = dst.levels;
        const int es = dst.esize;
        int64_t smax = 0, dmax = 0;
        for (int64_t k = 0; k < cnt; ++k)
        {
            if (S[k] < 0 || R[k] < 0) throw error(GHEXB_ERR_INTERNAL, "negative local index");
            smax = std::max(smax, S[k]);
            dmax = std::max(dmax, R[k]);
        }
        if (smax > k_i32max || dmax > k_i32max) throw error(GHEXB_ERR_RANGE, "local index exceeds 2^31");
        const int64_t idx0 = (int64_t)plan.idx.size();
        for (auto v : S) plan.idx.push_back((int32_t)v);
        for (auto v : R) plan.idx.push_back((int32_t)v);

        // forward descriptors: 16-byte columns when every column is 16-byte aligned; columns of
        // more than 256 units are split into level segments
        const bool cols = dst.level_stride == 1 && src.level_stride == 1;
        const bool vec16 = cols && (L * es) % 16 == 0 && (dst.index_stride * es) % 16 == 0 &&
                           (src.index_stride * es) % 16 == 0 &&
                           reinterpret_cast<uintptr_t>(dst.data) % 16 == 0 &&
                           reinterpret_cast<uintptr_t>(src.data) % 16 == 0;
        const int unit = vec16 ? 16 : es;
        const int64_t k = unit / es;
        const int64_t levels_u = L / k;
        const int64_t s_is = src.index_stride / k, d_is = dst.index_stride / k;
        const int64_t s_ls = vec16 ? 1 : src.level_stride, d_ls = vec16 ? 1 : dst.level_stride;
        const int64_t span_s = smax * s_is + (levels_u - 1) * s_ls;
        const int64_t span_d = dmax * d_is + (levels_u - 1) * d_ls;
        if (span_s > k_i32max || span_d > k_i32max)
            throw error(GHEXB_ERR_RANGE, "an index-list descriptor spans more than 2^31 elements");
        constexpr int64_t k_max_row = 256;
        for (int64_t l0 = 0; l0 < levels_u; l0 += k_max_row)
        {
            list_desc l{};
            l.src = src.data + l0 * s_ls * unit;
            l.dst = dst.data + l0 * d_ls * unit;
            l.count = (int32_t)cnt;
            l.levels = (int32_t)std::min(k_max_row, levels_u - l0);
            l.s_is = (int32_t)s_is, l.s_ls = (int32_t)s_ls;
            l.d_is = (int32_t)d_is, l.d_ls = (int32_t)d_ls;
            l.unit = (uint32_t)unit;
            l.field = (uint32_t)logical;
            l.map = row_map::make(l.levels);
            plan.lists.push_back(l);
            plan.list_idx_off.push_back(idx0);
            plan.list_src_slot.push_back(src_slot);
            plan.list_dst_slot.push_back(dst_slot);
            plan.list_src_off.push_back(l.src - src.data);
            plan.list_dst_off.push_back(l.dst - dst.data);
        }
        plan.halo_elements += cnt * L;
        plan.algorithmic_bytes += cnt * L * es * 2;
        plan.index_bytes += cnt * 8;

        // adjoint descriptors: element units, split so that no owner repeats inside one
        if (!dtype_is_float(dst.dtype)) return;
        int64_t b = 0;
        while (b < cnt)
        {
            std::unordered_map<int64_t, int> seen;
            int64_t e = b;
            while (e < cnt && seen.emplace(S[e], 1).second) ++e;
            for (int64_t l0 = 0; l0 < L; l0 += k_max_row)
            {
                list_desc a{};
                a.src = src.data + l0 * src.level_stride * es;
                a.dst = dst.data + l0 * dst.level_stride * es;
                a.count = (int32_t)(e - b);
                a.levels = (int32_t)std::min(k_max_row, L - l0);
                a.s_is = (int32_t)src.index_stride;
                a.s_ls = (int32_t)src.level_stride;
                a.d_is = (int32_t)dst.index_stride;
                a.d_ls = (int32_t)dst.level_stride;
                a.unit = (uint32_t)es;
                a.field = (uint32_t)logical;
                a.map = row_map::make(a.levels);
                plan.adj_lists.push_back(a);
                plan.adj_idx_off.push_back(idx0 + b);
                plan.adj_didx_off.push_back(idx0 + cnt + b);
                plan.adj_src_slot.push_back(src_slot);
                plan.adj_dst_slot.push_back(dst_slot);
                plan.adj_src_off.push_back(a.src - src.data);
                plan.adj_dst_off.push_back(a.dst - dst.data);
                list_src_field.push_back(src_slot);
            }
            b = e;
        }
    }
};


// ---- box adjoint in gather form ---------------------------------------------------------------
// The owner elements of a field decompose uniquely into coordinates when its axes, sorted by
// decreasing element stride, nest: every stride is at least the span of the axes below it.
struct owner_geometry
{
    int nd = 0;
    std::array<int64_t, 4> os{}, ext{};
    std::array<int, 4> order{}; // axes by decreasing stride
    bool ok = false;

    static owner_geometry of(const ghexb_field_s& f)
    {
        owner_geometry g;
        g.nd = f.ndim;
        for (int a = 0; a < f.ndim; ++a)
        {
            if (f.byte_strides[a] <= 0 || f.byte_strides[a] % f.esize) return g;
            g.os[a] = f.byte_strides[a] / f.esize;
            g.ext[a] = f.extents[a];
            g.order[a] = a;
        }
        std::stable_sort(g.order.begin(), g.order.begin() + g.nd, [&](int a, int b) { return g.os[a] > g.os[b]; });
        for (int k = 0; k + 1 < g.nd; ++k)
        {
            const int hi = g.order[k], lo = g.order[k + 1];
            if (g.os[hi] < g.os[lo] * g.ext[lo]) return g;
        }
        g.ok = g.nd >= 1 && g.os[g.order[g.nd - 1]] >= 1;
        return g;
    }

    bool decompose(int64_t off, std::array<int64_t, 4>& c) const
    {
        c = {0, 0, 0, 0};
        for (int k = 0; k < nd; ++k)
        {
            const int a = order[k];
            c[a] = off / os[a];
            off -= c[a] * os[a];
            if (c[a] < 0 || c[a] >= ext[a]) return false;
        }
        return off == 0;
    }
};

// Cuts the owner regions of the box descriptors of every source field into cells covered by the
// same descriptors. Returns false (with the reason) when a field's layout has no unique
// coordinates, a box stride matches no owner axis, or a cell has more than k_max_images images.
bool build_cells(ghexb_plan_s& plan, std::string& why)
{
    plan.cells.clear();
    struct omap
    {
        std::array<int64_t, 4> lo, hi, t;
        int64_t dst_lo;
        int dst_slot;
        uint32_t neg;
    };
    std::vector<omap> maps(plan.boxes.size());
    std::map<int, std::vector<int>> by_slot;
    for (int i = 0; i < (int)plan.boxes.size(); ++i)
    {
        const auto& b = plan.boxes[i];
        const int slot = plan.box_src_slot[i];
        const auto& f = plan.fields[slot];
        const owner_geometry G = owner_geometry::of(f);
        if (!G.ok)
        {
            why = "a field's strides do not nest";
            return false;
        }
        if (plan.box_src_off[i] % f.esize || plan.box_dst_off[i] % f.esize)
        {
            why = "a box origin is not element-aligned";
            return false;
        }
        std::array<int64_t, 4> c;
        if (!G.decompose(plan.box_src_off[i] / f.esize, c))
        {
            why = "a box origin has no owner coordinates";
            return false;
        }
        omap m{c, c, {0, 0, 0, 0}, plan.box_dst_off[i] / f.esize, plan.box_dst_slot[i], b.xor_mask != 0 ? 1u : 0u};
        const int64_t n[3] = {b.n0, b.n1, b.n2}, st[3] = {b.s0, b.s1, b.s2}, dt[3] = {b.d0, b.d1, b.d2};
        std::array<bool, 4> used{};
        for (int a = 0; a < 3; ++a)
        {
            if (n[a] <= 1) continue;
            int ax = -1;
            for (int q = 0; q < G.nd && ax < 0; ++q)
                if (!used[q] && G.os[q] == (st[a] < 0 ? -st[a] : st[a]) && G.ext[q] >= n[a]) ax = q;
            if (ax < 0)
            {
                why = "a box stride matches no owner axis";
                return false;
            }
            used[ax] = true;
            if (st[a] > 0) m.hi[ax] = c[ax] + n[a] - 1;
            else
            {
                m.lo[ax] = c[ax] - (n[a] - 1);
                m.dst_lo += (n[a] - 1) * dt[a];
            }
            m.t[ax] = st[a] > 0 ? dt[a] : -dt[a];
            if (m.lo[ax] < 0 || m.hi[ax] >= G.ext[ax])
            {
                why = "a box leaves its owner field";
                return false;
            }
        }
        maps[i] = m;
        by_slot[slot].push_back(i);
    }
    for (const auto& kv : by_slot)
    {
        const int slot = kv.first;
        const auto& ids = kv.second;
        const auto& f = plan.fields[slot];
        const owner_geometry G = owner_geometry::of(f);
        std::array<std::vector<int64_t>, 4> bp;
        int64_t ncells = 1;
        for (int a = 0; a < G.nd; ++a)
        {
            for (int i : ids)
            {
                bp[a].push_back(maps[i].lo[a]);
                bp[a].push_back(maps[i].hi[a] + 1);
            }
            std::sort(bp[a].begin(), bp[a].end());
            bp[a].erase(std::unique(bp[a].begin(), bp[a].end()), bp[a].end());
            ncells *= (int64_t)bp[a].size() - 1;
        }
        if (ncells > (int64_t(1) << 22))
        {
            why = "too many adjoint cells";
            return false;
        }
        std::array<int64_t, 4> j{0, 0, 0, 0};
        for (int64_t cell = 0; cell < ncells; ++cell)
        {
            int64_t r = cell;
            std::array<int64_t, 4> lo{0, 0, 0, 0}, hi{0, 0, 0, 0};
            for (int a = 0; a < G.nd; ++a)
            {
                const int64_t m = (int64_t)bp[a].size() - 1;
                j[a] = r % m;
                r /= m;
                lo[a] = bp[a][j[a]];
                hi[a] = bp[a][j[a] + 1] - 1;
            }
            std::vector<int> cover;
            for (int i : ids)
            {
                bool in = true;
                for (int a = 0; a < G.nd && in; ++a) in = maps[i].lo[a] <= lo[a] && hi[a] <= maps[i].hi[a];
                if (in) cover.push_back(i);
            }
            if (cover.empty()) continue;
            if ((int)cover.size() > k_max_images)
            {
                why = "an owner element has more than " + std::to_string(k_max_images) + " halo images";
                return false;
            }
            // cell axes: extents > 1 by increasing owner stride; axes beyond three are unrolled
            std::vector<int> axes;
            for (int a = 0; a < G.nd; ++a)
                if (hi[a] > lo[a]) axes.push_back(a);
            std::stable_sort(axes.begin(), axes.end(), [&](int a, int b) { return G.os[a] < G.os[b]; });
            std::vector<int> extra(axes.begin() + std::min<size_t>(3, axes.size()), axes.end());
            axes.resize(std::min<size_t>(3, axes.size()));
            int64_t nsub = 1;
            for (int a : extra) nsub *= hi[a] - lo[a] + 1;
            for (int64_t sub = 0; sub < nsub; ++sub)
            {
                std::array<int64_t, 4> base = lo;
                int64_t rr = sub;
                for (int a : extra)
                {
                    base[a] = lo[a] + rr % (hi[a] - lo[a] + 1);
                    rr /= hi[a] - lo[a] + 1;
                }
                gcell g{};
                g.own_slot = slot;
                g.esize = f.esize;
                g.own_off = 0;
                for (int a = 0; a < G.nd; ++a) g.own_off += base[a] * G.os[a];
                for (int q = 0; q < 3; ++q)
                {
                    g.n[q] = q < (int)axes.size() ? (int32_t)(hi[axes[q]] - lo[axes[q]] + 1) : 1;
                    g.o[q] = q < (int)axes.size() ? (int32_t)G.os[axes[q]] : 0;
                }
                g.nimg = (int)cover.size();
                for (int k = 0; k < g.nimg; ++k)
                {
                    const omap& m = maps[cover[k]];
                    auto& im = g.img[k];
                    im.slot = m.dst_slot;
                    im.off = m.dst_lo;
                    for (int a = 0; a < G.nd; ++a) im.off += (base[a] - m.lo[a]) * m.t[a];
                    for (int q = 0; q < 3; ++q) im.t[q] = q < (int)axes.size() ? (int32_t)m.t[axes[q]] : 0;
                    im.neg = m.neg;
                }
                plan.cells.push_back(g);
            }
        }
    }
    return true;
}

// Pairs of x-face boxes in one destination field whose rows interleave in memory: rows of at most
// 64 bytes along the destination's contiguous axis, the same rows and planes, and B's row r + 1
// starting where A's row r ends. Each box joins at most one pair.
void find_pairs(ghexb_plan_s& plan)
{
    plan.pairs.clear();
    plan.box_pair.assign(plan.boxes.size(), -1);
    std::map<std::pair<int, int64_t>, int> by_dst; // (destination slot, byte offset) -> box
    auto short_row = [&](const box_desc& b) {
        return (b.esize == 8 || b.esize == 4) && b.d0 == 1 && (int64_t)b.n0 * b.esize <= 64 && b.n1 >= 2;
    };
    for (int i = 0; i < (int)plan.boxes.size(); ++i)
        if (short_row(plan.boxes[i])) by_dst[{plan.box_dst_slot[i], plan.box_dst_off[i]}] = i;
    for (int a = 0; a < (int)plan.boxes.size(); ++a)
    {
        const auto& A = plan.boxes[a];
        if (!short_row(A) || plan.box_pair[a] >= 0) continue;
        const int64_t want = plan.box_dst_off[a] + ((int64_t)A.n0 - A.d1) * A.esize;
        auto it = by_dst.find({plan.box_dst_slot[a], want});
        if (it == by_dst.end()) continue;
        const int b = it->second;
        const auto& B = plan.boxes[b];
        if (b == a || plan.box_pair[b] >= 0 || B.esize != A.esize || B.n1 != A.n1 || B.n2 != A.n2 ||
            B.d1 != A.d1 || B.d2 != A.d2 || B.field != A.field)
            continue;
        plan.box_pair[a] = plan.box_pair[b] = (int)plan.pairs.size();
        plan.pairs.push_back({a, b});
    }
}

// Owner columns of the unstructured adjoint lists, each with its image columns in receive order.
// Returns false when an owner has more than k_max_images images or its images differ in levels
// or level stride.
bool build_list_owners(ghexb_plan_s& plan, std::string& why)
{
    plan.lowners.clear();
    std::map<std::pair<int, int64_t>, int> index; // (slot, byte offset) -> owner
    for (size_t i = 0; i < plan.adj_lists.size(); ++i)
    {
        const auto& l = plan.adj_lists[i];
        const int ss = plan.adj_src_slot[i], ds = plan.adj_dst_slot[i];
        const int es = plan.fields[ss].esize;
        for (int32_t k = 0; k < l.count; ++k)
        {
            const int64_t so = plan.adj_src_off[i] + (int64_t)plan.idx[plan.adj_idx_off[i] + k] * l.s_is * es;
            const int64_t dof = plan.adj_dst_off[i] + (int64_t)plan.idx[plan.adj_didx_off[i] + k] * l.d_is * es;
            auto it = index.find({ss, so});
            if (it == index.end())
            {
                ghexb_plan_s::list_owner o{};
                o.slot = ss, o.off = so, o.levels = l.levels, o.s_ls = l.s_ls, o.d_ls = l.d_ls, o.esize = es;
                it = index.emplace(std::make_pair(ss, so), (int)plan.lowners.size()).first;
                plan.lowners.push_back(o);
            }
            auto& o = plan.lowners[it->second];
            if (o.levels != l.levels || o.s_ls != l.s_ls || o.d_ls != l.d_ls)
            {
                why = "an owner column's images differ in levels or level stride";
                return false;
            }
            if (o.nimg == k_max_images)
            {
                why = "an owner column has more than " + std::to_string(k_max_images) + " images";
                return false;
            }
            o.img_slot[o.nimg] = ds;
            o.img_off[o.nimg] = dof;
            ++o.nimg;
        }
    }
    std::stable_sort(plan.lowners.begin(), plan.lowners.end(), [](const auto& a, const auto& b) {
        return std::make_tuple(a.esize, a.nimg, a.levels, a.s_ls, a.d_ls) <
               std::make_tuple(b.esize, b.nimg, b.levels, b.s_ls, b.d_ls);
    });
    return true;
}

// Receive rows of an in-place receive: GHEX receives the message of a neighbour as raw bytes at
// the address of its first receive index (communication_object_ipr.hpp:127-141), so the k-th
// value lands on row front + k whatever the receive list says. Those rows must be halo rows of
// the domain, received once: otherwise the outcome would depend on the order of the copies.
std::vector<std::vector<int64_t>> in_place_rows(const ghexb_pattern_s& P, int d)
{
    const auto& dom = P.domains[d];
    std::vector<std::vector<int64_t>> rows;
    std::unordered_set<int64_t> claimed;
    for (const auto& re : dom.urecv)
    {
        std::vector<int64_t> r(re.lids.size());
        for (size_t k = 0; k < r.size(); ++k)
        {
            r[k] = re.lids[0] + (int64_t)k;
            if (!std::binary_search(dom.outer.begin(), dom.outer.end(), r[k]) || !claimed.insert(r[k]).second)
                throw error(GHEXB_ERR_INVALID,
                    "in-place receive: the halo of domain " + std::to_string(dom.id) + " received from domain " +
                        std::to_string(P.domains[re.neighbor].id) + " is not stored on consecutive halo rows from " +
                        "local index " + std::to_string(re.lids[0]));
        }
        rows.push_back(std::move(r));
    }
    return rows;
}

} // namespace

void build_tables(ghexb_plan_s& plan, ghexb_context_s* ctx, const ghexb_field* fields, int n)
{
    if (n < 1) throw error(GHEXB_ERR_INVALID, "an exchange needs at least one field");
    plan.ctx = ctx;
    for (int i = 0; i < n; ++i)
    {
        if (!fields[i]) throw error(GHEXB_ERR_INVALID, "null field handle");
        plan.fields.push_back(*fields[i]);
    }
    if (plan.shard_mode != 0)
    {
        if (plan.shard_mode != 1 && plan.shard_mode != 2) throw error(GHEXB_ERR_INVALID, "sharded mode must be 1 (pull) or 2 (push)");
        if ((int)plan.shard_local.size() != n) throw error(GHEXB_ERR_INVALID, "one locality flag per field");
        if (plan.in_place_receive) throw error(GHEXB_ERR_INVALID, "an in-place receive is not sharded");
        if (plan.shard_mode == 1)
        {
            plan.adjoint_ok = false;
            plan.adjoint_reason = "the pull form of a sharded exchange has no adjoint (its push form has)";
        }
    }
    // descriptors of a sharded plan: those writing (pull) or reading (push) a local field
    auto kept = [&](int dst_slot, int src_slot) {
        if (plan.shard_mode == 1) return plan.shard_local[dst_slot] != 0;
        if (plan.shard_mode == 2) return plan.shard_local[src_slot] != 0;
        return true;
    };
    // patterns in order of first appearance; per (pattern, domain) the field slots in order
    std::vector<ghexb_pattern_s*> pats;
    std::vector<std::vector<std::vector<int>>> groups;
    for (int i = 0; i < n; ++i)
    {
        auto* P = plan.fields[i].pattern;
        auto it = std::find(pats.begin(), pats.end(), P);
        int pi = (int)(it - pats.begin());
        if (it == pats.end())
        {
            pats.push_back(P);
            groups.emplace_back(P->domains.size());
        }
        groups[pi][plan.fields[i].domain_index].push_back(i);
    }
    builder B(plan);
    std::map<std::pair<int, int>, int> logical;
    auto logical_of = [&](int pi, int k) {
        auto it = logical.find({pi, k});
        if (it != logical.end()) return it->second;
        const int id = (int)logical.size();
        logical[{pi, k}] = id;
        return id;
    };
    for (int pi = 0; pi < (int)pats.size(); ++pi)
    {
        const auto& P = *pats[pi];
        for (int d = 0; d < (int)P.domains.size(); ++d)
        {
            const auto& Fd = groups[pi][d];
            if (Fd.empty()) continue;
            auto partner = [&](int e) -> const std::vector<int>& {
                const auto& Fe = groups[pi][e];
                if (Fe.size() != Fd.size())
                    throw error(GHEXB_ERR_INCOMPATIBLE,
                        "field incompatible with available domains! domain " + std::to_string(P.domains[d].id) +
                            " exchanges " + std::to_string(Fd.size()) + " field(s) but its neighbour " +
                            std::to_string(P.domains[e].id) + " provides " + std::to_string(Fe.size()));
                return Fe;
            };
            auto check_pair = [&](const ghexb_field_s& a, const ghexb_field_s& b) {
                if (a.dtype != b.dtype) throw error(GHEXB_ERR_INCOMPATIBLE, "paired fields differ in dtype");
                if (a.num_components != b.num_components || a.is_vector != b.is_vector)
                    throw error(GHEXB_ERR_INCOMPATIBLE, "paired fields differ in components");
                if (a.levels != b.levels) throw error(GHEXB_ERR_INCOMPATIBLE, "paired fields differ in levels");
            };
            if (plan.in_place_receive && P.kind != pattern_kind::unstructured)
                throw error(GHEXB_ERR_INVALID, "an in-place receive needs an unstructured pattern");
            if (P.kind == pattern_kind::unstructured)
            {
                std::vector<std::vector<int64_t>> placed;
                if (plan.in_place_receive)
                {
                    placed = in_place_rows(P, d);
                    for (int slot : Fd)
                    {
                        const auto& f = plan.fields[slot];
                        const bool rows = f.levels == 1 ? f.index_stride == 1
                                                        : f.level_stride == 1 && f.index_stride == f.levels;
                        if (!rows)
                            throw error(GHEXB_ERR_INVALID,
                                "in-place receive needs the levels of a halo element stored contiguously "
                                "(levels first, rows without padding)");
                    }
                }
                for (size_t ri = 0; ri < P.domains[d].urecv.size(); ++ri)
                {
                    const auto& re = P.domains[d].urecv[ri];
                    const auto& rlids = plan.in_place_receive ? placed[ri] : re.lids;
                    const auto& Fe = partner(re.neighbor);
                    const list_entry* se = nullptr;
                    for (const auto& s : P.domains[re.neighbor].usend)
                        if (s.neighbor == d && s.tag == re.tag) se = &s;
                    if (!se) throw error(GHEXB_ERR_INTERNAL, "unmatched receive list");
                    for (size_t k = 0; k < Fd.size(); ++k)
                    {
                        const auto& dst = plan.fields[Fd[k]];
                        const auto& src = plan.fields[Fe[k]];
                        check_pair(dst, src);
                        const int lg = logical_of(pi, (int)k);
                        if (kept(Fd[k], Fe[k])) B.list_pair(dst, Fd[k], src, Fe[k], rlids, se->lids, lg);
                    }
                }
                continue;
            }
            for (const auto& re : P.domains[d].recv)
            {
                const auto& Fe = partner(re.neighbor);
                for (size_t k = 0; k < Fd.size(); ++k)
                {
                    const auto& dst = plan.fields[Fd[k]];
                    const auto& src = plan.fields[Fe[k]];
                    check_pair(dst, src);
                    const int lg = logical_of(pi, (int)k);
                    if (!kept(Fd[k], Fe[k])) continue;
                    for (const auto& sp : re.spaces)
                    {
                        if (P.kind == pattern_kind::regular) B.regular_space(P, re.neighbor, dst, Fd[k], src, Fe[k], sp, lg);
                        else
                            B.cubed_space(P, d, re.neighbor, dst, Fd[k], src, Fe[k], sp, lg);
                    }
                }
            }
        }
    }
    plan.n_logical = (int)logical.size();

    // adjoint phases: a descriptor runs after every earlier descriptor whose owner elements it
    // shares, so every owner accumulates its halos in descriptor order
    for (const auto& f : plan.fields)
        if (!dtype_is_float(f.dtype))
        {
            plan.adjoint_ok = false;
            plan.adjoint_reason = "the adjoint needs float32 or float64 fields";
        }
    plan.box_phase.assign(plan.boxes.size(), 0);
    {
        std::map<int, std::vector<int>> by_field;
        for (int i = 0; i < (int)plan.boxes.size(); ++i)
        {
            auto& mine = B.box_owner[i];
            int ph = 0;
            for (int j : by_field[mine.field])
            {
                const auto& o = B.box_owner[j];
                bool overlap = true;
                for (int a = 0; a < 4; ++a)
                    if (o.hi[a] < mine.lo[a] || mine.hi[a] < o.lo[a]) overlap = false;
                if (overlap) ph = std::max(ph, plan.box_phase[j] + 1);
            }
            plan.box_phase[i] = ph;
            by_field[mine.field].push_back(i);
        }
    }
    plan.list_phase.assign(plan.adj_lists.size(), 0);
    {
        std::map<int, std::unordered_map<int32_t, int>> last; // per source field: owner -> phase
        for (int i = 0; i < (int)plan.adj_lists.size(); ++i)
        {
            const auto& a = plan.adj_lists[i];
            auto& m = last[B.list_src_field[i]];
            int ph = 0;
            const int64_t s0 = plan.adj_idx_off[i];
            for (int32_t k = 0; k < a.count; ++k)
            {
                auto it = m.find(plan.idx[s0 + k]);
                if (it != m.end()) ph = std::max(ph, it->second + 1);
            }
            for (int32_t k = 0; k < a.count; ++k) m[plan.idx[s0 + k]] = ph;
            plan.list_phase[i] = ph;
        }
    }
    plan.gather_ok = plan.adjoint_ok && build_cells(plan, plan.gather_reason);
    std::string list_reason;
    plan.list_gather_ok = plan.adjoint_ok && build_list_owners(plan, list_reason);
    find_pairs(plan);
}

namespace
{
int64_t field_span(const ghexb_field_s& f);

// memory type of the byte at p; host memory must be mapped at its own address
cudaMemoryType accessible_type(const void* p)
{
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess)
    {
        (void)cudaGetLastError();
        throw error(GHEXB_ERR_INVALID, std::string("field memory: cudaPointerGetAttributes failed: ") +
                                           cudaGetErrorString(e));
    }
    switch (a.type)
    {
        case cudaMemoryTypeDevice:
        case cudaMemoryTypeManaged: return a.type;
        case cudaMemoryTypeHost:
            if (a.devicePointer == p) return a.type;
            throw error(GHEXB_ERR_INVALID, "page-locked host memory of a field is not mapped at the same address on the device");
        default:
            throw error(GHEXB_ERR_INVALID,
                "field memory is neither device memory nor page-locked host memory (a host field's pages must be "
                "locked for the device: ghexb_host_register)");
    }
}
} // namespace

void check_accessible(const void* p) { (void)accessible_type(p); }

void check_accessible(const void* p, size_t bytes)
{
    // page-locked host memory is locked page by page, possibly by several registrations: every
    // page of the range is checked, not only its first byte
    if (accessible_type(p) != cudaMemoryTypeHost || bytes <= 1) return;
    const char* c = static_cast<const char*>(p);
    for (size_t off = 4096 - reinterpret_cast<uintptr_t>(c) % 4096; off < bytes; off += 4096) (void)accessible_type(c + off);
    (void)accessible_type(c + bytes - 1);
}

void upload_plan(ghexb_plan_s& plan)
{
    for (const auto& f : plan.fields) check_accessible(f.data, (size_t)(field_span(f) * f.esize));
    plan.field_on_device.clear();
    for (const auto& f : plan.fields) plan.field_on_device.push_back(accessible_type(f.data) == cudaMemoryTypeDevice);
    // upload index lists, patch device pointers, upload descriptor tables
    host_stager st(plan, nullptr);
    upload(plan.d_idx, plan.idx, st);
    for (size_t i = 0; i < plan.lists.size(); ++i)
    {
        plan.lists[i].sidx = plan.d_idx + plan.list_idx_off[i];
        plan.lists[i].didx = plan.d_idx + plan.list_idx_off[i] + plan.lists[i].count;
    }
    for (size_t i = 0; i < plan.adj_lists.size(); ++i)
    {
        plan.adj_lists[i].sidx = plan.d_idx + plan.adj_idx_off[i];
        plan.adj_lists[i].didx = plan.d_idx + plan.adj_didx_off[i];
    }
    upload(plan.d_boxes, plan.boxes, st);
    upload(plan.d_lists, plan.lists, st);
    // two scheduler counters per phased adjoint kernel
    const std::vector<unsigned> zeros(4, 0u);
    upload(plan.d_counters, zeros, st);
    upload(plan.d_adj_lists, plan.adj_lists, st);
    st.commit();
    check_cuda(cudaStreamCreateWithFlags(&plan.cap_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    retile(plan);
    check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize");
}

void build_plan(ghexb_plan_s& plan, ghexb_context_s* ctx, const ghexb_field* fields, int n)
{
    build_tables(plan, ctx, fields, n);
    upload_plan(plan);
}

namespace
{
// memory span of a field in elements: every valid element offset lies in [0, span)
int64_t field_span(const ghexb_field_s& f)
{
    if (f.pattern && f.pattern->kind == pattern_kind::unstructured)
    {
        const int64_t size = f.pattern->domains[f.domain_index].size;
        return (size - 1) * f.index_stride + (f.levels - 1) * f.level_stride + 1;
    }
    int64_t span = 1;
    for (int a = 0; a < f.ndim; ++a) span += (int64_t)(f.extents[a] - 1) * (f.byte_strides[a] / f.esize);
    return span;
}

void check_offset(const ghexb_field_s& f, const char* base, int64_t rel, int64_t span, const char* what)
{
    const int64_t e = (base - f.data) / f.esize + rel;
    if (e < 0 || e >= span)
        throw error(GHEXB_ERR_RANGE, std::string(what) + " element offset " + std::to_string(e) +
                                         " outside the field's memory span " + std::to_string(span));
}
} // namespace

size_t field_bytes(const ghexb_field_s& f) { return (size_t)(field_span(f) * f.esize); }

namespace
{
// Approximate DRAM bytes of a run of `count` elements in rows of `row` elements of `unit` bytes:
// a row touches about one 32-byte sector more than its bytes.
double run_cost(int64_t count, int unit, int64_t row)
{
    const double w = (double)row * unit;
    return (double)count * unit * (w + 32.0) / w;
}

// A forward tile's rows run along its first axis where source and destination are both
// contiguous along it (pairs: segments of n0 elements); otherwise every element is a row.
double tile_cost(const xtile& t)
{
    auto unit_stride = [](int32_t v) { return v == 1 || v == -1; };
    const bool contiguous = t.kind == 2 || (t.kind == 0 ? unit_stride(t.s0) && unit_stride(t.d0) : t.s1 == 1 && t.d1 == 1);
    return run_cost(t.count, t.unit, contiguous ? t.n0 : 1);
}

// A gather tile's accesses are rows along its first axis only where the owner and every image
// are contiguous along it; otherwise every element is a row of its own.
double tile_cost(const gtile& t)
{
    bool contiguous = t.o0 == 1;
    for (int i = 0; i < t.nimg && contiguous; ++i) contiguous = t.kind ? t.img[0].t0 == 1 : (t.img[i].t0 == 1 || t.img[i].t0 == -1);
    return run_cost(t.count, t.esize, contiguous ? t.n0 : 1) * 2.0 * (1 + t.nimg);
}

// Appends the tiles of one launch range; returns [begin, count) in out.
template<typename R>
std::pair<int, int> append_range(std::vector<R>& out, const std::vector<R>& tiles)
{
    const int begin = (int)out.size();
    out.insert(out.end(), tiles.begin(), tiles.end());
    return {begin, (int)tiles.size()};
}

int class_of_x(const xtile& t) { return forward_class_of(t.kind, t.unit, t.neg != 0); }

// The elements of a pair tile that exist, with the decomposition of exchange.cu's pair_elements:
// fn(a, c, s, i2) with a = element of box A.
template<typename F>
void for_pair_elements(const xtile& t, F&& fn)
{
    for (uint32_t e = 0; e < t.count; ++e)
    {
        const uint32_t g = t.e0 + e;
        const uint32_t q = fast_div{t.n0, t.m0, t.l0}.div(g);
        const int64_t c = g - (int64_t)q * t.n0;
        const uint32_t i2 = fast_div{t.n1, t.m1, t.l1}.div(q);
        const int64_t s = q - (int64_t)i2 * t.n1;
        if (c < 0 || c >= t.n0 || s < 0 || s >= t.n1) throw error(GHEXB_ERR_INTERNAL, "pair element decomposition out of range");
        const bool a = c < (int64_t)t.na;
        if (a ? s >= 1 : s + 1 < (int64_t)t.n1) fn(a, c, s, (int64_t)i2);
    }
}

int64_t valid_elements(const gtile& t) { return t.count; }

int64_t valid_elements(const xtile& t)
{
    if (t.kind != 2) return t.count;
    int64_t n = 0;
    for_pair_elements(t, [&](bool, int64_t, int64_t, int64_t) { ++n; });
    return n;
}
int class_of_g(const gtile& t) { return t.kind ? list_gather_class(t.esize, t.nimg) : gather_class(t.esize, t.nimg); }
} // namespace

void dram_floor(const ghexb_plan_s& plan, int sector, int64_t& read_bytes, int64_t& write_bytes)
{
    if (sector < 1 || (sector & (sector - 1))) throw error(GHEXB_ERR_INVALID, "the sector size must be a power of two");
    // every element's source and destination address as (sector << 5) | bytes: elements are aligned
    // to their size (at most 16 bytes), so none straddles a sector of 16 bytes or more
    std::vector<uint64_t> rd, wr;
    rd.reserve((size_t)plan.halo_elements);
    wr.reserve((size_t)plan.halo_elements);
    auto add = [&](const char* src, const char* dst, uint64_t bytes) {
        rd.push_back((reinterpret_cast<uintptr_t>(src) / sector) << 5 | bytes);
        wr.push_back((reinterpret_cast<uintptr_t>(dst) / sector) << 5 | bytes);
    };
    for (const auto& b : plan.boxes)
        for (int32_t i2 = 0; i2 < b.n2; ++i2)
            for (int32_t i1 = 0; i1 < b.n1; ++i1)
                for (int32_t i0 = 0; i0 < b.n0; ++i0)
                    add(b.src + ((int64_t)i0 * b.s0 + (int64_t)i1 * b.s1 + (int64_t)i2 * b.s2) * b.esize,
                        b.dst + ((int64_t)i0 * b.d0 + (int64_t)i1 * b.d1 + (int64_t)i2 * b.d2) * b.esize, b.esize);
    for (size_t i = 0; i < plan.lists.size(); ++i)
    {
        const auto& l = plan.lists[i];
        const int32_t* sidx = plan.idx.data() + plan.list_idx_off[i];
        const int32_t* didx = sidx + l.count;
        for (int32_t k = 0; k < l.count; ++k)
            for (int32_t v = 0; v < l.levels; ++v)
                add(l.src + ((int64_t)sidx[k] * l.s_is + (int64_t)v * l.s_ls) * l.unit,
                    l.dst + ((int64_t)didx[k] * l.d_is + (int64_t)v * l.d_ls) * l.unit, l.unit);
    }
    std::sort(rd.begin(), rd.end());
    std::sort(wr.begin(), wr.end());
    std::vector<uint64_t> rs; // sectors read
    for (uint64_t v : rd)
        if (rs.empty() || rs.back() != (v >> 5)) rs.push_back(v >> 5);
    int64_t written = 0, fill = 0;
    for (size_t a = 0; a < wr.size();)
    {
        const uint64_t sec = wr[a] >> 5;
        uint64_t bytes = 0;
        size_t b = a;
        for (; b < wr.size() && (wr[b] >> 5) == sec; ++b) bytes += wr[b] & 31u;
        ++written;
        // a sector written in part whose other bytes were not read is filled from DRAM first
        if (bytes < (uint64_t)sector && !std::binary_search(rs.begin(), rs.end(), sec)) ++fill;
        a = b;
    }
    read_bytes = ((int64_t)rs.size() + fill) * sector;
    write_bytes = written * sector;
}

namespace
{
// Moves the pointers of a plan's tile tables from the fields' old memory to their new memory:
// every pointer that lies in an old field's span moves by that field's displacement. Every table
// pointer that the kernels dereference addresses an element of a field (tile records, gather
// cells, the column table) or the index lists, which do not move. Not applicable (ok == false)
// when two old spans overlap.
struct relocator
{
    struct span
    {
        uintptr_t lo, hi;
        intptr_t delta;
    };
    std::vector<span> spans; // sorted by lo
    bool ok = true;

    relocator(const std::vector<ghexb_field_s>& fields, void* const* data)
    {
        for (size_t i = 0; i < fields.size(); ++i)
        {
            const uintptr_t lo = reinterpret_cast<uintptr_t>(fields[i].data);
            spans.push_back({lo, lo + field_bytes(fields[i]), reinterpret_cast<intptr_t>(data[i]) - (intptr_t)lo});
        }
        std::sort(spans.begin(), spans.end(), [](const span& a, const span& b) { return a.lo < b.lo; });
        for (size_t i = 1; i < spans.size(); ++i)
            if (spans[i].lo < spans[i - 1].hi) ok = false;
    }
    template<typename P>
    void operator()(P*& p) const
    {
        const uintptr_t a = reinterpret_cast<uintptr_t>(p);
        auto it = std::upper_bound(spans.begin(), spans.end(), a, [](uintptr_t v, const span& s) { return v < s.lo; });
        if (it == spans.begin()) return;
        --it;
        if (a < it->hi) p = reinterpret_cast<P*>(a + it->delta);
    }
    void operator()(uint64_t& v) const
    {
        char* p = reinterpret_cast<char*>(v);
        (*this)(p);
        v = reinterpret_cast<uint64_t>(p);
    }
};

void relocate_tiles(ghexb_plan_s& plan, const relocator& R)
{
    for (auto* tab : {&plan.xf, &plan.xp, &plan.xb, &plan.xpair})
        for (auto& t : *tab)
        {
            R(t.src), R(t.dst);
            if (t.src2) R(t.src2);
        }
    for (auto& g : plan.gt)
    {
        if (g.own) R(g.own);
        for (int k = 0; k < k_max_images; ++k)
            if (g.img[k].ptr) R(g.img[k].ptr);
    }
    for (auto& c : plan.lcols) R(c);
    for (auto& c : plan.gblk) R(c);
    for (auto& t : plan.bt) R(t.src), R(t.dst);
    for (auto& c : plan.bgt_blk) R(c);
}

} // namespace

void check_relocation(ghexb_plan_s& plan)
{
    // the tables built for the fields at a second address, against the current tables moved there
    build_tiles(plan, plan.idx.data());
    std::vector<void*> moved;
    for (size_t i = 0; i < plan.fields.size(); ++i) moved.push_back(plan.fields[i].data + (int64_t)4096 * (int64_t)(i + 1) * 3);
    const relocator R(plan.fields, moved.data());
    if (!R.ok) return;
    ghexb_plan_s copy;
    copy.xf = plan.xf, copy.xp = plan.xp, copy.xb = plan.xb, copy.xpair = plan.xpair, copy.gt = plan.gt, copy.lcols = plan.lcols;
    copy.gblk = plan.gblk, copy.bt = plan.bt, copy.bgt_blk = plan.bgt_blk;
    relocate_tiles(copy, R);
    const auto old_data = plan.fields;
    const auto old_boxes = plan.boxes;
    const auto old_lists = plan.lists;
    for (size_t i = 0; i < plan.fields.size(); ++i) plan.fields[i].data = static_cast<char*>(moved[i]);
    for (size_t i = 0; i < plan.boxes.size(); ++i)
    {
        plan.boxes[i].src = plan.fields[plan.box_src_slot[i]].data + plan.box_src_off[i];
        plan.boxes[i].dst = plan.fields[plan.box_dst_slot[i]].data + plan.box_dst_off[i];
    }
    for (size_t i = 0; i < plan.lists.size(); ++i)
    {
        plan.lists[i].src = plan.fields[plan.list_src_slot[i]].data + plan.list_src_off[i];
        plan.lists[i].dst = plan.fields[plan.list_dst_slot[i]].data + plan.list_dst_off[i];
    }
    build_tiles(plan, plan.idx.data());
    auto same = [](const auto& a, const auto& b) {
        return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(a[0])) == 0);
    };
    const bool equal = same(copy.xf, plan.xf) && same(copy.xp, plan.xp) && same(copy.xb, plan.xb) &&
                       same(copy.xpair, plan.xpair) && same(copy.gt, plan.gt) && same(copy.lcols, plan.lcols) &&
                       same(copy.gblk, plan.gblk) && same(copy.bt, plan.bt) && same(copy.bgt_blk, plan.bgt_blk);
    plan.fields = old_data, plan.boxes = old_boxes, plan.lists = old_lists;
    build_tiles(plan, plan.idx.data());
    if (!equal) throw error(GHEXB_ERR_INTERNAL, "moved tile tables differ from the tables built at the new address");
}

int64_t check_tables(ghexb_plan_s& plan)
{
    build_tiles(plan, plan.idx.data());
    int64_t checked = 0;
    // forward tiles, with the element decomposition of exchange.cu
    auto replay = [&](const xtile& t, const ghexb_field_s& sf, const ghexb_field_s& df) {
        const int64_t k = t.unit / sf.esize; // elements per unit
        const int64_t ss = field_span(sf), ds = field_span(df);
        for (uint32_t e = 0; e < t.count; ++e)
        {
            const uint32_t g = t.e0 + e;
            int64_t so, dof;
            if (t.kind == 0)
            {
                const uint32_t r = fast_div{t.n0, t.m0, t.l0}.div(g);
                const int64_t i0 = g - r * t.n0;
                const uint32_t i2 = fast_div{t.n1, t.m1, t.l1}.div(r);
                const int64_t i1 = r - i2 * t.n1;
                if (i0 < 0 || i0 >= t.n0 || i1 < 0 || i1 >= t.n1)
                    throw error(GHEXB_ERR_INTERNAL, "box element decomposition out of range");
                so = i0 * t.s0 + i1 * t.s1 + (int64_t)i2 * t.s2;
                dof = i0 * t.d0 + i1 * t.d1 + (int64_t)i2 * t.d2;
            }
            else
            {
                const uint32_t col = fast_div{t.n0, t.m0, t.l0}.div(g);
                const int64_t lev = g - col * t.n0;
                so = (int64_t)t.sidx[col] * t.s0 + lev * t.s1;
                dof = (int64_t)t.didx[col] * t.d0 + lev * t.d1;
            }
            check_offset(sf, t.src, so * k, ss, "source");
            check_offset(sf, t.src, so * k + k - 1, ss, "source");
            check_offset(df, t.dst, dof * k, ds, "destination");
            check_offset(df, t.dst, dof * k + k - 1, ds, "destination");
        }
        return (int64_t)t.count;
    };
    auto replay_range = [&](std::pair<int, int> r, int src_slot, int dst_slot) {
        for (int k = r.first; k < r.first + r.second; ++k)
        {
            const xtile& t = plan.xb[k];
            if ((int)t.count > forward_per_thread(plan.per_thread, t.unit) * plan.block)
                throw error(GHEXB_ERR_INTERNAL, "forward tile too large");
            if (t.count) checked += replay(t, plan.fields[src_slot], plan.fields[dst_slot]);
        }
    };
    for (size_t i = 0; i < plan.boxes.size(); ++i) replay_range(plan.xb_box[i], plan.box_src_slot[i], plan.box_dst_slot[i]);
    for (size_t i = 0; i < plan.lists.size(); ++i)
        replay_range(plan.xb_list[i], plan.list_src_slot[i], plan.list_dst_slot[i]);
    // pairs: every element's source and destination, against the two boxes' own mapping
    for (size_t p = 0; p < plan.pairs.size(); ++p)
    {
        const int ia = plan.pairs[p].first, ib = plan.pairs[p].second;
        const auto& A = plan.boxes[ia];
        const auto& Bx = plan.boxes[ib];
        std::vector<std::tuple<const char*, const char*, int>> want, got;
        for (int which = 0; which < 2; ++which)
        {
            const auto& b = which ? Bx : A;
            for (int32_t i2 = 0; i2 < b.n2; ++i2)
                for (int32_t i1 = 0; i1 < b.n1; ++i1)
                    for (int32_t i0 = 0; i0 < b.n0; ++i0)
                        want.emplace_back(b.dst + ((int64_t)i0 * b.d0 + (int64_t)i1 * b.d1 + (int64_t)i2 * b.d2) * b.esize,
                            b.src + ((int64_t)i0 * b.s0 + (int64_t)i1 * b.s1 + (int64_t)i2 * b.s2) * b.esize,
                            b.xor_mask != 0);
        }
        const auto& sa = plan.fields[plan.box_src_slot[ia]];
        const auto& sb = plan.fields[plan.box_src_slot[ib]];
        const auto& df = plan.fields[plan.box_dst_slot[ia]];
        const int64_t spa = field_span(sa), spb = field_span(sb), spd = field_span(df);
        for (int k = plan.xpair_range[p].first; k < plan.xpair_range[p].first + plan.xpair_range[p].second; ++k)
        {
            const xtile& t = plan.xpair[k];
            if ((int)t.count > forward_per_thread(plan.per_thread, t.unit) * plan.block)
                throw error(GHEXB_ERR_INTERNAL, "forward tile too large");
            for_pair_elements(t, [&](bool a, int64_t c, int64_t s, int64_t i2) {
                const int64_t so = a ? c * t.s0 + (s - 1) * t.s1 + i2 * t.s2 : (c - t.na) * t.u0 + s * t.u1 + i2 * t.u2;
                const int64_t dof = c + (s - 1) * t.d1 + i2 * t.d2;
                check_offset(a ? sa : sb, a ? t.src : t.src2, so, a ? spa : spb, "source");
                check_offset(df, t.dst, dof, spd, "destination");
                got.emplace_back(t.dst + dof * t.unit, (a ? t.src : t.src2) + so * t.unit, a ? t.neg : t.neg2);
            });
        }
        std::sort(want.begin(), want.end());
        std::sort(got.begin(), got.end());
        if (want != got) throw error(GHEXB_ERR_INTERNAL, "a pair's segments differ from its two boxes");
    }
    // every table: tile classes consistent with their elements, and the same
    // work in the batched, per-field and per-box tables
    auto check_tiles = [](const auto& tiles, int begin, int count, auto class_of) {
        int64_t elems = 0;
        for (int u = begin; u < begin + count; ++u)
        {
            const auto& t = tiles[u];
            if (t.count == 0 || class_of(t) != t.cls) throw error(GHEXB_ERR_INTERNAL, "a tile's class differs from its elements");
            elems += valid_elements(t);
        }
        return elems;
    };
    const int64_t nf = check_tiles(plan.xf, 0, (int)plan.xf.size(), class_of_x);
    int64_t np = 0, nb = 0;
    for (const auto& r : plan.xp_field) np += check_tiles(plan.xp, r.first, r.second, class_of_x);
    for (const auto& r : plan.xb_box) nb += check_tiles(plan.xb, r.first, r.second, class_of_x);
    for (const auto& r : plan.xb_list) nb += check_tiles(plan.xb, r.first, r.second, class_of_x);
    // index blocks: a flagged list tile finds every column's indices in its block, as the lists hold them
    auto check_blocks = [&](const std::vector<xtile>& tiles, const std::vector<int32_t>& blocks) {
        for (size_t p = 0; p < tiles.size(); ++p)
        {
            const xtile& t = tiles[p];
            if (!t.pad[0]) continue;
            if (t.kind != 1 || blocks.size() < (p + 1) * k_block_ints)
                throw error(GHEXB_ERR_INTERNAL, "index block of a tile that has none");
            for (uint32_t e = 0; e < t.count; ++e)
            {
                const uint32_t col = fast_div{t.n0, t.m0, t.l0}.div(t.e0 + e);
                const uint32_t c = col - (uint32_t)t.u0;
                if (c >= (uint32_t)k_block_columns || blocks[p * k_block_ints + c] != t.sidx[col] ||
                    blocks[p * k_block_ints + k_block_columns + c] != t.didx[col])
                    throw error(GHEXB_ERR_INTERNAL, "index block differs from the lists");
            }
        }
    };
    check_blocks(plan.xf, plan.xf_blk);
    check_blocks(plan.xp, plan.xp_blk);
    check_blocks(plan.xb, plan.xb_blk);
    const int64_t ns = check_staged(plan);
    checked += ns;
    // bulk column tiles: every column inside its fields, 16-byte aligned, its indices as the list
    // holds them; the lists they take have no element tiles in the batched table
    int64_t nbulk = 0;
    if (plan.bt_blk.size() != plan.bt.size() * k_bulk_block_ints || plan.bt_list.size() != plan.bt.size())
        throw error(GHEXB_ERR_INTERNAL, "bulk tiles and their index blocks differ in number");
    for (size_t u = 0; u < plan.bt.size(); ++u)
    {
        const auto& t = plan.bt[u];
        const int i = plan.bt_list[u];
        const auto& l = plan.lists[i];
        const auto& sf = plan.fields[plan.list_src_slot[i]];
        const auto& df = plan.fields[plan.list_dst_slot[i]];
        const int64_t sbytes = field_span(sf) * sf.esize, dbytes = field_span(df) * df.esize;
        if (t.ncols == 0 || t.ncols > (uint32_t)k_bulk_columns || t.col_bytes % 16 || t.col_bytes != (uint32_t)l.levels * 16u ||
            (int64_t)t.ncols * t.col_bytes > k_bulk_stage || t.src != l.src || t.dst != l.dst)
            throw error(GHEXB_ERR_INTERNAL, "bulk tile out of shape");
        const bool four = t.smap >= 0;
        if (four != (t.dmap >= 0) || (four && (t.smap >= (int32_t)plan.bmap_geo.size() || t.dmap >= (int32_t)plan.bmap_geo.size() ||
                                                  (int64_t)(t.ncols + 3) / 4 * 4 * t.col_bytes > k_bulk_stage || (4 * t.col_bytes) % 128)))
            throw error(GHEXB_ERR_INTERNAL, "bulk tile's tensor maps out of shape");
        if (four)
            for (const auto& [g, base, is] : {std::tuple{plan.bmap_geo[t.smap], t.src, t.s_is}, std::tuple{plan.bmap_geo[t.dmap], (const char*)t.dst, t.d_is}})
                if (g.base != base || g.stride != is || (int64_t)g.width * g.es != (int64_t)t.col_bytes || g.stride % 16 ||
                    reinterpret_cast<uintptr_t>(g.base) % 16 || g.width > 256)
                    throw error(GHEXB_ERR_INTERNAL, "bulk tile's tensor map differs from its columns");
        const int32_t* S = plan.idx.data() + plan.list_idx_off[i];
        for (uint32_t c = 0; c < t.ncols; ++c)
        {
            const int32_t col = plan.bt_col0[u] + (int32_t)c;
            if (col >= l.count || plan.bt_blk[u * k_bulk_block_ints + c] != S[col] ||
                plan.bt_blk[u * k_bulk_block_ints + k_bulk_columns + c] != S[l.count + col])
                throw error(GHEXB_ERR_INTERNAL, "bulk index block differs from the list");
            const int64_t so = (t.src - sf.data) + (int64_t)S[col] * t.s_is;
            const int64_t dof = (t.dst - df.data) + (int64_t)S[l.count + col] * t.d_is;
            if (so < 0 || so + t.col_bytes > sbytes || dof < 0 || dof + t.col_bytes > dbytes)
                throw error(GHEXB_ERR_RANGE, "bulk column outside its field's memory");
            if (four && (S[col] < 0 || S[col] >= plan.bmap_geo[t.smap].rows || S[l.count + col] < 0 ||
                            S[l.count + col] >= plan.bmap_geo[t.dmap].rows))
                throw error(GHEXB_ERR_RANGE, "bulk column outside its tensor map");
            if ((reinterpret_cast<uintptr_t>(sf.data) + (uint64_t)so) % 16 || (reinterpret_cast<uintptr_t>(df.data) + (uint64_t)dof) % 16)
                throw error(GHEXB_ERR_INTERNAL, "bulk column not 16-byte aligned");
        }
        nbulk += (int64_t)t.ncols * l.levels;
    }
    for (const auto& t : plan.xf)
        if (t.kind == 1)
            for (size_t u = 0; u < plan.bt.size(); ++u)
                if (t.src == plan.bt[u].src && t.dst == plan.bt[u].dst && t.sidx == plan.idx.data() + plan.list_idx_off[plan.bt_list[u]])
                    throw error(GHEXB_ERR_INTERNAL, "a list is both in bulk and in element tiles");
    checked += nbulk;
    if (nf + ns + nbulk != nb || np != nb) throw error(GHEXB_ERR_INTERNAL, "batched, per-field and per-box tables differ");
    if (plan.gather_ok)
    {
        check_tiles(plan.gt, 0, (int)plan.gt.size(), class_of_g);
        for (const auto& t : plan.gt)
            if ((int)t.count > gather_per_thread(t.nimg) * k_gather_block)
                throw error(GHEXB_ERR_INTERNAL, "gather tile too large");
    }

    // gather cells: every element in bounds, every owner and every image touched exactly once,
    // and the images are exactly the destination elements of the box descriptors
    if (plan.gather_ok)
    {
        std::vector<std::pair<int, int64_t>> owners, images, box_dst;
        for (const auto& g : plan.cells)
        {
            const auto& of = plan.fields[g.own_slot];
            const int64_t os = field_span(of);
            for (int32_t c = 0; c < g.n[2]; ++c)
                for (int32_t b = 0; b < g.n[1]; ++b)
                    for (int32_t a = 0; a < g.n[0]; ++a)
                    {
                        const int64_t o = g.own_off + (int64_t)a * g.o[0] + (int64_t)b * g.o[1] + (int64_t)c * g.o[2];
                        if (o < 0 || o >= os) throw error(GHEXB_ERR_RANGE, "adjoint owner outside its field");
                        owners.push_back({g.own_slot, o});
                        for (int k = 0; k < g.nimg; ++k)
                        {
                            const auto& im = g.img[k];
                            const int64_t h = im.off + (int64_t)a * im.t[0] + (int64_t)b * im.t[1] + (int64_t)c * im.t[2];
                            if (h < 0 || h >= field_span(plan.fields[im.slot]))
                                throw error(GHEXB_ERR_RANGE, "adjoint image outside its field");
                            images.push_back({im.slot, h});
                        }
                    }
        }
        for (size_t i = 0; i < plan.boxes.size(); ++i)
        {
            const auto& b = plan.boxes[i];
            const int slot = plan.box_dst_slot[i];
            const int64_t base = plan.box_dst_off[i] / plan.fields[slot].esize;
            for (int32_t c = 0; c < b.n2; ++c)
                for (int32_t r = 0; r < b.n1; ++r)
                    for (int32_t a = 0; a < b.n0; ++a)
                        box_dst.push_back({slot, base + (int64_t)a * b.d0 + (int64_t)r * b.d1 + (int64_t)c * b.d2});
        }
        std::sort(owners.begin(), owners.end());
        if (std::adjacent_find(owners.begin(), owners.end()) != owners.end())
            throw error(GHEXB_ERR_INTERNAL, "an owner element lies in two adjoint cells");
        std::sort(images.begin(), images.end());
        std::sort(box_dst.begin(), box_dst.end());
        if (images != box_dst) throw error(GHEXB_ERR_INTERNAL, "adjoint images differ from the forward destinations");
        checked += (int64_t)images.size();
    }
    // unstructured owner columns: every level in bounds, owners pairwise distinct, images equal to
    // the destinations of the adjoint lists, and the tiles cover every owner level once
    if (plan.list_gather_ok)
    {
        std::vector<std::pair<int, int64_t>> owners, images, list_dst;
        int64_t levels = 0;
        for (const auto& o : plan.lowners)
        {
            const int64_t es = o.esize;
            for (int32_t lev = 0; lev < o.levels; ++lev)
            {
                const int64_t oe = o.off / es + (int64_t)lev * o.s_ls;
                if (o.off % es || oe < 0 || oe >= field_span(plan.fields[o.slot]))
                    throw error(GHEXB_ERR_RANGE, "adjoint owner column outside its field");
                owners.push_back({o.slot, oe});
                for (int i = 0; i < o.nimg; ++i)
                {
                    const int64_t he = o.img_off[i] / es + (int64_t)lev * o.d_ls;
                    if (o.img_off[i] % es || he < 0 || he >= field_span(plan.fields[o.img_slot[i]]))
                        throw error(GHEXB_ERR_RANGE, "adjoint image column outside its field");
                    images.push_back({o.img_slot[i], he});
                }
            }
            levels += o.levels;
        }
        for (size_t i = 0; i < plan.adj_lists.size(); ++i)
        {
            const auto& l = plan.adj_lists[i];
            const int slot = plan.adj_dst_slot[i];
            const int64_t es = plan.fields[slot].esize;
            for (int32_t k = 0; k < l.count; ++k)
                for (int32_t lev = 0; lev < l.levels; ++lev)
                    list_dst.push_back({slot, plan.adj_dst_off[i] / es + (int64_t)plan.idx[plan.adj_didx_off[i] + k] * l.d_is +
                                                  (int64_t)lev * l.d_ls});
        }
        std::sort(owners.begin(), owners.end());
        if (std::adjacent_find(owners.begin(), owners.end()) != owners.end())
            throw error(GHEXB_ERR_INTERNAL, "an owner element appears in two adjoint columns");
        std::sort(images.begin(), images.end());
        std::sort(list_dst.begin(), list_dst.end());
        if (images != list_dst) throw error(GHEXB_ERR_INTERNAL, "adjoint images differ from the list destinations");
        int64_t covered = 0;
        for (const auto& t : plan.gt)
            if (t.kind == 1)
            {
                covered += t.count;
                if ((int64_t)t.col0 + (int64_t)(t.e0 + t.count - 1) / t.n0 * (t.nimg + 1) + t.nimg >= (int64_t)plan.lcols.size())
                    throw error(GHEXB_ERR_INTERNAL, "adjoint tile outside the column table");
            }
        // bulk gather tiles: their column addresses as the column table holds them, 16-byte aligned,
        // within the shared stage; their owners are covered by them and by no element tile
        if (plan.bgt_blk.size() != plan.bgt.size() * k_bgather_entries || plan.bgt_first.size() != plan.bgt.size())
            throw error(GHEXB_ERR_INTERNAL, "bulk gather tiles and their blocks differ in number");
        for (size_t u = 0; u < plan.bgt.size(); ++u)
        {
            const auto& t = plan.bgt[u];
            const uint64_t per = (uint64_t)t.nimg + 1, n = t.nown * per;
            if (t.nown == 0 || n > (uint64_t)k_bgather_entries || t.col_bytes % 16 || t.col_bytes > (uint32_t)k_bgather_zero ||
                n * t.col_bytes > (uint64_t)k_bulk_stage || t.col_bytes != t.levels * t.esize ||
                (uint64_t)plan.bgt_first[u] + n > plan.lcols.size())
                throw error(GHEXB_ERR_INTERNAL, "bulk gather tile out of shape");
            for (uint64_t c = 0; c < n; ++c)
            {
                const uint64_t a = plan.bgt_blk[u * k_bgather_entries + c];
                if (a != plan.lcols[plan.bgt_first[u] + c] || a % 16)
                    throw error(GHEXB_ERR_INTERNAL, "bulk gather block differs from the column table");
            }
            covered += (int64_t)t.nown * t.levels;
        }
        if (covered != levels) throw error(GHEXB_ERR_INTERNAL, "adjoint tiles do not cover every owner level");
        // column blocks: the flagged tiles' blocks hold their slices of the column table
        if (plan.gblk.size() != (plan.gt.size() - (size_t)plan.gt_boxes) * k_gblock_entries)
            throw error(GHEXB_ERR_INTERNAL, "column blocks do not match the gather tiles");
        for (size_t i = (size_t)plan.gt_boxes; i < plan.gt.size(); ++i)
        {
            const auto& t = plan.gt[i];
            if (!t.pad[0]) continue;
            const uint64_t per = (uint64_t)t.nimg + 1, j0 = t.e0 / t.n0, j1 = (t.e0 + t.count - 1) / t.n0;
            if ((j1 - j0 + 1) * per > (uint64_t)k_gblock_entries) throw error(GHEXB_ERR_INTERNAL, "column block overflow");
            for (uint64_t j = j0; j <= j1; ++j)
                for (uint64_t c = 0; c < per; ++c)
                    if (plan.gblk[(i - plan.gt_boxes) * k_gblock_entries + (j - j0) * per + c] != plan.lcols[t.col0 + j * per + c])
                        throw error(GHEXB_ERR_INTERNAL, "column block differs from the column table");
        }
        checked += (int64_t)images.size();
    }
    // phased adjoint lists
    for (size_t i = 0; i < plan.adj_lists.size(); ++i)
    {
        const auto& l = plan.adj_lists[i];
        const auto& sf = plan.fields[plan.adj_src_slot[i]];
        const auto& df = plan.fields[plan.adj_dst_slot[i]];
        const int64_t k = l.unit / sf.esize;
        const int64_t ss = field_span(sf), ds = field_span(df);
        for (int32_t col = 0; col < l.count; ++col)
            for (int32_t lev = 0; lev < l.levels; ++lev)
            {
                check_offset(sf, l.src, ((int64_t)plan.idx[plan.adj_idx_off[i] + col] * l.s_is + (int64_t)lev * l.s_ls) * k, ss, "source");
                check_offset(df, l.dst, ((int64_t)plan.idx[plan.adj_didx_off[i] + col] * l.d_is + (int64_t)lev * l.d_ls) * k, ds, "destination");
            }
        checked += (int64_t)l.count * l.levels;
    }
    // a sharded plan: every forward descriptor writes (pull) or reads (push) a local field, and
    // every adjoint owner is local
    if (plan.shard_mode != 0)
    {
        const bool pull = plan.shard_mode == 1;
        auto local = [&](int slot) { return plan.shard_local[slot] != 0; };
        for (size_t i = 0; i < plan.boxes.size(); ++i)
            if (!local(pull ? plan.box_dst_slot[i] : plan.box_src_slot[i]))
                throw error(GHEXB_ERR_INTERNAL, "a sharded plan holds a box of another process");
        for (size_t i = 0; i < plan.lists.size(); ++i)
            if (!local(pull ? plan.list_dst_slot[i] : plan.list_src_slot[i]))
                throw error(GHEXB_ERR_INTERNAL, "a sharded plan holds a list of another process");
        if (plan.gather_ok)
            for (const auto& g : plan.cells)
                if (!local(g.own_slot)) throw error(GHEXB_ERR_INTERNAL, "a sharded adjoint gathers into another process's field");
        if (plan.list_gather_ok)
            for (const auto& o : plan.lowners)
                if (!local(o.slot)) throw error(GHEXB_ERR_INTERNAL, "a sharded adjoint gathers into another process's field");
        for (size_t i = 0; i < plan.adj_lists.size() && plan.adjoint_ok; ++i)
            if (!local(plan.adj_src_slot[i]))
                throw error(GHEXB_ERR_INTERNAL, "a sharded adjoint accumulates into another process's owner");
    }
    return checked;
}

namespace
{
// device buffer of at least n elements; returns true when it was (re)allocated
template<typename T>
bool ensure(T*& dptr, size_t& cap, size_t n)
{
    if (n <= cap && dptr) return false;
    if (dptr) cudaFree(dptr), dptr = nullptr;
    cap = 0;
    if (n == 0) return true;
    check_cuda(cudaMalloc(&dptr, n * sizeof(T)), "cudaMalloc(plan tiles)");
    cap = n;
    return true;
}

} // namespace

void retile(ghexb_plan_s& plan, cudaStream_t stream)
{
    release_graph(plan);
    build_tiles(plan, plan.d_idx);
    ensure(plan.d_xf, plan.cap_xf, plan.xf.size());
    ensure(plan.d_xp, plan.cap_xp, plan.xp.size());
    ensure(plan.d_xb, plan.cap_xb, plan.xb.size());
    ensure(plan.d_gt, plan.cap_gt, plan.gt.size());
    ensure(plan.d_lcols, plan.cap_lcols, plan.lcols.size());
    ensure(plan.d_gblk, plan.cap_gblk, plan.gblk.size());
    ensure(plan.d_bt, plan.cap_bt, plan.bt.size());
    ensure(plan.d_bt_blk, plan.cap_bt_blk, plan.bt_blk.size());
    ensure(plan.d_bmaps, plan.cap_bmaps, plan.bmaps.size());
    ensure(plan.d_bgt, plan.cap_bgt, plan.bgt.size());
    ensure(plan.d_bgt_blk, plan.cap_bgt_blk, plan.bgt_blk.size());
    ensure(plan.d_smaps, plan.cap_smaps, plan.smaps.size());
    ensure(plan.d_sitems, plan.cap_sitems, plan.sitems.size());
    ensure(plan.d_xf_blk, plan.cap_xf_blk, plan.xf_blk.size());
    ensure(plan.d_xp_blk, plan.cap_xp_blk, plan.xp_blk.size());
    ensure(plan.d_xb_blk, plan.cap_xb_blk, plan.xb_blk.size());
    host_stager st(plan, stream);
    st.put(plan.d_xf_blk, plan.xf_blk);
    st.put(plan.d_xp_blk, plan.xp_blk);
    st.put(plan.d_xb_blk, plan.xb_blk);
    st.put(plan.d_xf, plan.xf);
    st.put(plan.d_xp, plan.xp);
    st.put(plan.d_xb, plan.xb);
    st.put(plan.d_gt, plan.gt);
    st.put(plan.d_lcols, plan.lcols);
    st.put(plan.d_gblk, plan.gblk);
    st.put(plan.d_bt, plan.bt);
    st.put(plan.d_bt_blk, plan.bt_blk);
    st.put(plan.d_bmaps, plan.bmaps);
    st.put(plan.d_bgt, plan.bgt);
    st.put(plan.d_bgt_blk, plan.bgt_blk);
    st.put(plan.d_smaps, plan.smaps);
    st.put(plan.d_sitems, plan.sitems);
    if ((!plan.sitems.empty() || !plan.bt.empty() || !plan.bgt.empty()) && !plan.d_status)
    {
        check_cuda(cudaMalloc(&plan.d_status, sizeof(unsigned)), "cudaMalloc(staged status)");
        check_cuda(cudaMemsetAsync(plan.d_status, 0, sizeof(unsigned), stream), "cudaMemsetAsync(staged status)");
    }
    upload(plan.d_adj_btiles, plan.adj_btiles, st);
    upload(plan.d_adj_ltiles, plan.adj_ltiles, st);
    st.commit();
    plan.forms_stale = false;
}

// Index blocks of a tile table: for every list tile whose columns number at most
// k_block_columns, the source then destination indices of its columns (k_block_ints per tile, at
// the tile's position), which the kernel loads beside the tile record; the tile is flagged
// (pad[0] = 1). Empty when the plan has no lists.
void build_index_blocks(ghexb_plan_s& plan, std::vector<xtile>& tiles, std::vector<int32_t>& blocks, const int32_t* idx)
{
    blocks.clear();
    if (plan.lists.empty() || !idx) return;
    blocks.assign(tiles.size() * k_block_ints, 0);
    for (size_t p = 0; p < tiles.size(); ++p)
    {
        xtile& t = tiles[p];
        t.pad[0] = 0;
        if (t.kind != 1 || t.count == 0) continue;
        const uint32_t first = t.e0 / t.n0, last = (t.e0 + t.count - 1) / t.n0;
        if ((uint32_t)t.u0 != first || last - first + 1 > (uint32_t)k_block_columns) continue;
        const int64_t so = t.sidx - idx, dof = t.didx - idx; // offsets of the lists in plan.idx
        for (uint32_t c = first; c <= last; ++c)
        {
            blocks[p * k_block_ints + (c - first)] = plan.idx[so + c];
            blocks[p * k_block_ints + k_block_columns + (c - first)] = plan.idx[dof + c];
        }
        t.pad[0] = 1;
    }
}

void build_tiles(ghexb_plan_s& plan, const int32_t* idx)
{
    // ---- staged boxes (batched form): tensor maps and items
    build_staged(plan);
    auto staged = [&](int box) { return !plan.box_staged.empty() && plan.box_staged[box]; };
    // ---- forward
    const int B = plan.block;
    auto cap = [&](int unit) { return (uint32_t)(forward_per_thread(plan.per_thread, unit) * B); };
    // Short rows cost a memory request per row rather than per 32 elements: their tiles shrink by
    // the row's useful bytes over the bytes of the sectors it touches, so that the requests of
    // x-face boxes spread over as many CTAs (and SMs) as their bytes would.
    auto row_cap = [&](int unit, int64_t row_elems) {
        const int64_t w = row_elems * unit;
        const int64_t c = (int64_t)cap(unit) * w / (w + 32);
        return (uint32_t)std::max<int64_t>(B, std::min<int64_t>(cap(unit), c));
    };
    auto box_tiles = [&](int i, std::vector<xtile>& out) {
        const auto& b = plan.boxes[i];
        const fast_div f0 = fast_div::make((uint32_t)b.n0), f1 = fast_div::make((uint32_t)b.n1);
        const uint32_t n = (uint32_t)((int64_t)b.n0 * b.n1 * b.n2), c = row_cap((int)b.esize, b.n0);
        for (uint32_t e0 = 0; e0 < n; e0 += c)
        {
            xtile t{};
            t.src = b.src, t.dst = b.dst;
            t.e0 = e0, t.count = std::min(c, n - e0);
            t.s0 = b.s0, t.s1 = b.s1, t.s2 = b.s2;
            t.d0 = b.d0, t.d1 = b.d1, t.d2 = b.d2;
            t.n0 = f0.d, t.m0 = f0.m, t.l0 = (uint8_t)f0.l;
            t.n1 = f1.d, t.m1 = f1.m, t.l1 = (uint8_t)f1.l;
            t.unit = (uint8_t)b.esize;
            t.kind = 0;
            t.neg = b.xor_mask != 0;
            out.push_back(t);
        }
    };
    auto list_tiles = [&](int i, std::vector<xtile>& out) {
        const auto& l = plan.lists[i];
        const fast_div f0 = fast_div::make((uint32_t)l.levels);
        const uint32_t n = (uint32_t)((int64_t)l.count * l.levels);
        uint32_t c = row_cap((int)l.unit, l.levels);
        // whole columns, at most k_block_columns of them, when a tile holds at least one: the
        // tile's index block (below) then covers its columns
        if ((uint32_t)l.levels <= c) c = std::min<uint32_t>(c / l.levels, k_block_columns) * (uint32_t)l.levels;
        for (uint32_t e0 = 0; e0 < n; e0 += c)
        {
            xtile t{};
            t.src = l.src, t.dst = l.dst;
            t.sidx = idx ? idx + plan.list_idx_off[i] : nullptr;
            t.didx = idx ? idx + plan.list_idx_off[i] + l.count : nullptr;
            t.e0 = e0, t.count = std::min(c, n - e0);
            t.s0 = l.s_is, t.s1 = l.s_ls, t.d0 = l.d_is, t.d1 = l.d_ls;
            t.n0 = f0.d, t.m0 = f0.m, t.l0 = (uint8_t)f0.l;
            t.n1 = 1, t.m1 = 1, t.l1 = 0;
            t.unit = (uint8_t)l.unit;
            t.kind = 1;
            t.u0 = (int32_t)(e0 / (uint32_t)l.levels); // first column of the tile
            out.push_back(t);
        }
    };
    auto pair_tiles = [&](int p, std::vector<xtile>& out) {
        const auto& A = plan.boxes[plan.pairs[p].first];
        const auto& Bx = plan.boxes[plan.pairs[p].second];
        const uint32_t w = (uint32_t)(A.n0 + Bx.n0), segs = (uint32_t)A.n1 + 1;
        const fast_div f0 = fast_div::make(w), f1 = fast_div::make(segs);
        const uint32_t n = (uint32_t)((int64_t)w * segs * A.n2), c = row_cap((int)A.esize, std::max(A.n0, Bx.n0));
        for (uint32_t e0 = 0; e0 < n; e0 += c)
        {
            xtile t{};
            t.src = A.src, t.dst = A.dst, t.src2 = Bx.src;
            t.e0 = e0, t.count = std::min(c, n - e0);
            t.s0 = A.s0, t.s1 = A.s1, t.s2 = A.s2;
            t.u0 = Bx.s0, t.u1 = Bx.s1, t.u2 = Bx.s2;
            t.d0 = 1, t.d1 = A.d1, t.d2 = A.d2;
            t.n0 = f0.d, t.m0 = f0.m, t.l0 = (uint8_t)f0.l;
            t.n1 = f1.d, t.m1 = f1.m, t.l1 = (uint8_t)f1.l;
            t.na = (uint32_t)A.n0;
            t.unit = (uint8_t)A.esize;
            t.kind = 2;
            t.neg = A.xor_mask != 0, t.neg2 = Bx.xor_mask != 0;
            t.cls = (uint8_t)class_of_x(t);
            out.push_back(t);
        }
    };
    std::vector<std::vector<xtile>> ptiles(plan.pairs.size());
    plan.xpair.clear();
    plan.xpair_range.clear();
    for (size_t p = 0; p < plan.pairs.size(); ++p)
    {
        pair_tiles((int)p, ptiles[p]);
        plan.xpair_range.push_back({(int)plan.xpair.size(), (int)ptiles[p].size()});
        plan.xpair.insert(plan.xpair.end(), ptiles[p].begin(), ptiles[p].end());
    }
    // tiles per descriptor, with their element class
    std::vector<std::vector<xtile>> btiles(plan.boxes.size()), ltiles(plan.lists.size());
    for (size_t i = 0; i < plan.boxes.size(); ++i)
    {
        box_tiles((int)i, btiles[i]);
        for (auto& t : btiles[i]) t.cls = (uint8_t)class_of_x(t);
    }
    for (size_t i = 0; i < plan.lists.size(); ++i)
    {
        list_tiles((int)i, ltiles[i]);
        for (auto& t : ltiles[i]) t.cls = (uint8_t)class_of_x(t);
    }
    // per box: one range per descriptor
    plan.xb.clear();
    plan.xb_box.assign(plan.boxes.size(), {0, 0});
    plan.xb_list.assign(plan.lists.size(), {0, 0});
    for (size_t i = 0; i < plan.boxes.size(); ++i) plan.xb_box[i] = append_range(plan.xb, btiles[i]);
    for (size_t i = 0; i < plan.lists.size(); ++i) plan.xb_list[i] = append_range(plan.xb, ltiles[i]);
    // per field: one range per logical field
    plan.xp.clear();
    plan.xp_field.assign(plan.n_logical, {0, 0});
    for (int lg = 0; lg < plan.n_logical; ++lg)
    {
        std::vector<xtile> f;
        for (size_t i = 0; i < plan.boxes.size(); ++i)
            if ((int)plan.boxes[i].field == lg && (!plan.use_pairs || plan.box_pair[i] < 0))
                f.insert(f.end(), btiles[i].begin(), btiles[i].end());
        for (size_t p = 0; p < plan.pairs.size() && plan.use_pairs; ++p)
            if ((int)plan.boxes[plan.pairs[p].first].field == lg) f.insert(f.end(), ptiles[p].begin(), ptiles[p].end());
        for (size_t i = 0; i < plan.lists.size(); ++i)
            if ((int)plan.lists[i].field == lg) f.insert(f.end(), ltiles[i].begin(), ltiles[i].end());
        plan.xp_field[lg] = append_range(plan.xp, f);
    }
    // batched: one range, the most DRAM bytes per element (short rows) first, so that the first
    // wave of CTAs starts on the most expensive tiles; staged boxes are the staged kernel's, and
    // a pair moves as a pair only when neither of its boxes is staged
    {
        auto paired = [&](int i) {
            if (!plan.use_pairs || plan.box_pair[i] < 0) return false;
            const auto& pr = plan.pairs[plan.box_pair[i]];
            return !staged(pr.first) && !staged(pr.second);
        };
        std::vector<xtile> all;
        for (size_t i = 0; i < plan.boxes.size(); ++i)
            if (!staged((int)i) && !paired((int)i)) all.insert(all.end(), btiles[i].begin(), btiles[i].end());
        if (plan.use_pairs)
            for (size_t p = 0; p < ptiles.size(); ++p)
                if (!staged(plan.pairs[p].first) && !staged(plan.pairs[p].second))
                    all.insert(all.end(), ptiles[p].begin(), ptiles[p].end());
        // lists in 16-byte units between device fields: bulk column tiles, else element tiles
        plan.bt.clear(), plan.bt_blk.clear(), plan.bt_list.clear(), plan.bt_col0.clear();
        plan.bmaps.clear(), plan.bmap_geo.clear();
        auto on_device = [&](int slot) { return plan.field_on_device.empty() || plan.field_on_device[slot]; };
        // the tensor map of a field's columns from `base` (a row per index, `width` elements a
        // row): its index in bmaps, or -1 when it cannot be had (a column wider than a load box)
        auto bmap = [&](int slot, const char* base, int width) -> int32_t {
            const auto& f = plan.fields[slot];
            const int64_t rows = f.pattern->domains[f.domain_index].size, stride = f.index_stride * f.esize;
            if (width < 1 || width > 256 || rows < 1 || rows > k_i32max || stride % 16 || reinterpret_cast<uintptr_t>(base) % 16)
                return -1;
            for (size_t m = 0; m < plan.bmap_geo.size(); ++m)
            {
                const auto& g = plan.bmap_geo[m];
                if (g.base == base && g.rows == rows && g.stride == stride && g.width == width && g.es == f.esize) return (int32_t)m;
            }
            CUtensorMap map{};
            if (plan.encode_maps)
            {
                const cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)rows};
                const cuuint64_t strides[1] = {(cuuint64_t)stride};
                const cuuint32_t box[2] = {(cuuint32_t)width, 1};
                const CUtensorMapDataType type = f.esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : f.esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32
                                                 : f.esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8;
                if (encode_tensor_map(&map, type, 2, const_cast<char*>(base), dims, strides, box, CU_TENSOR_MAP_L2_PROMOTION_NONE) !=
                    CUDA_SUCCESS)
                    return -1;
            }
            plan.bmaps.push_back(map);
            plan.bmap_geo.push_back({base, rows, stride, width, f.esize});
            return (int32_t)plan.bmaps.size() - 1;
        };
        for (size_t i = 0; i < plan.lists.size(); ++i)
        {
            const auto& l = plan.lists[i];
            const uint32_t cb = (uint32_t)l.levels * 16u;
            // (not on a sharded plan: its fields include other processes' memory)
            if (!((int)(i % 4) < plan.bulk_share && plan.shard_mode == 0 && l.unit == 16 && cb <= (uint32_t)k_bulk_stage &&
                    on_device(plan.list_src_slot[i]) && on_device(plan.list_dst_slot[i])))
            {
                all.insert(all.end(), ltiles[i].begin(), ltiles[i].end());
                continue;
            }
            // four columns at a time through tensor maps when both fields have one, else one at a time
            const int es = plan.fields[plan.list_src_slot[i]].esize;
            int32_t smap = bmap(plan.list_src_slot[i], l.src, (int)(cb / es));
            int32_t dmap = smap >= 0 ? bmap(plan.list_dst_slot[i], l.dst, (int)(cb / es)) : -1;
            const uint32_t four = (uint32_t)k_bulk_stage / (4 * cb) * 4;
            // (each group of four starts on a 128-byte boundary of the shared stage)
            if (smap < 0 || dmap < 0 || four < 4 || (4 * cb) % 128) smap = dmap = -1;
            const int32_t per = (int32_t)std::min<uint32_t>(k_bulk_columns, smap >= 0 ? four : (uint32_t)k_bulk_stage / cb);
            const int32_t* S = plan.idx.data() + plan.list_idx_off[i];
            const int32_t* D = S + l.count;
            for (int32_t c0 = 0; c0 < l.count; c0 += per)
            {
                btile t{};
                t.src = l.src, t.dst = l.dst;
                t.s_is = (int64_t)l.s_is * 16, t.d_is = (int64_t)l.d_is * 16;
                t.ncols = (uint32_t)std::min(per, l.count - c0);
                t.col_bytes = cb;
                t.smap = smap, t.dmap = dmap;
                const size_t b = plan.bt_blk.size();
                plan.bt_blk.resize(b + k_bulk_block_ints, 0);
                for (uint32_t c = 0; c < t.ncols; ++c)
                {
                    plan.bt_blk[b + c] = S[c0 + c];
                    plan.bt_blk[b + k_bulk_columns + c] = D[c0 + c];
                }
                plan.bt.push_back(t);
                plan.bt_list.push_back((int)i);
                plan.bt_col0.push_back(c0);
            }
        }
        auto per_elem = [](const xtile& t) { return tile_cost(t) / std::max<uint32_t>(1u, t.count); };
        std::stable_sort(all.begin(), all.end(), [&](const xtile& x, const xtile& y) { return per_elem(x) > per_elem(y); });
        plan.xf.clear();
        append_range(plan.xf, all);
    }
    build_index_blocks(plan, plan.xf, plan.xf_blk, idx);
    build_index_blocks(plan, plan.xp, plan.xp_blk, idx);
    build_index_blocks(plan, plan.xb, plan.xb_blk, idx);

    // ---- box adjoint, gather form
    plan.gt.clear();
    if (plan.gather_ok)
    {
        std::vector<gtile> all;
        for (const auto& g : plan.cells)
        {
            // tiles of short rows shrink as the forward's do (row_cap): rows along the first axis
            // only where the owner and every image are contiguous along it
            bool contiguous = g.o[0] == 1;
            for (int k = 0; k < g.nimg && contiguous; ++k) contiguous = g.img[k].t[0] == 1 || g.img[k].t[0] == -1;
            const int64_t w = (contiguous ? g.n[0] : 1) * (int64_t)g.esize;
            const int64_t full = (int64_t)gather_per_thread(g.nimg) * k_gather_block;
            int64_t sized = std::max<int64_t>(k_gather_block, std::min<int64_t>(full, full * w / (w + 32)));
            // tuning: halved (gather_scale -1) or grown towards a full tile (1: x2, 2: x4)
            if (plan.gather_scale < 0) sized = std::max<int64_t>(k_gather_block / 2, sized / 2);
            else if (plan.gather_scale > 0) sized = std::min<int64_t>(full, sized << plan.gather_scale);
            const uint32_t gc = (uint32_t)sized;
            const auto& of = plan.fields[g.own_slot];
            const fast_div f0 = fast_div::make((uint32_t)g.n[0]), f1 = fast_div::make((uint32_t)g.n[1]);
            const uint32_t n = (uint32_t)((int64_t)g.n[0] * g.n[1] * g.n[2]);
            for (uint32_t e0 = 0; e0 < n; e0 += gc)
            {
                gtile t{};
                t.own = of.data + g.own_off * of.esize;
                t.e0 = e0, t.count = std::min(gc, n - e0);
                t.o0 = g.o[0], t.o1 = g.o[1], t.o2 = g.o[2];
                t.n0 = f0.d, t.m0 = f0.m, t.l0 = (uint8_t)f0.l;
                t.n1 = f1.d, t.m1 = f1.m, t.l1 = (uint8_t)f1.l;
                t.esize = (uint8_t)g.esize;
                t.nimg = (uint8_t)g.nimg;
                for (int k = 0; k < g.nimg; ++k)
                {
                    const auto& df = plan.fields[g.img[k].slot];
                    t.img[k].ptr = df.data + g.img[k].off * df.esize;
                    t.img[k].t0 = g.img[k].t[0], t.img[k].t1 = g.img[k].t[1], t.img[k].t2 = g.img[k].t[2];
                    t.img[k].neg = g.img[k].neg;
                }
                t.cls = (uint8_t)class_of_g(t);
                all.push_back(t);
            }
        }
        // the most expensive tiles (most bytes, short rows) first: the first wave starts on them
        std::stable_sort(all.begin(), all.end(), [](const gtile& a, const gtile& b) { return tile_cost(a) > tile_cost(b); });
        append_range(plan.gt, all);
    }
    plan.gt_boxes = (int)plan.gt.size();
    // ---- unstructured adjoint, gather form: owner groups and their column table; of a group whose
    // columns are contiguous and 16-byte aligned, the first gather_bulk quarters of its owners go
    // to the bulk gather kernel
    plan.lcols.clear();
    plan.bgt.clear(), plan.bgt_blk.clear(), plan.bgt_first.clear();
    if (plan.list_gather_ok)
    {
        for (size_t a = 0; a < plan.lowners.size();)
        {
            const auto& o0 = plan.lowners[a];
            size_t b = a;
            while (b < plan.lowners.size() && plan.lowners[b].esize == o0.esize && plan.lowners[b].nimg == o0.nimg &&
                   plan.lowners[b].levels == o0.levels && plan.lowners[b].s_ls == o0.s_ls && plan.lowners[b].d_ls == o0.d_ls)
                ++b;
            const uint32_t group0 = (uint32_t)plan.lcols.size();
            bool aligned = true;
            for (size_t j = a; j < b; ++j)
            {
                const auto& o = plan.lowners[j];
                plan.lcols.push_back((uint64_t)(uintptr_t)(plan.fields[o.slot].data + o.off));
                for (int i = 0; i < o.nimg; ++i)
                    plan.lcols.push_back((uint64_t)(uintptr_t)(plan.fields[o.img_slot[i]].data + o.img_off[i]));
            }
            for (size_t c = group0; c < plan.lcols.size(); ++c) aligned = aligned && plan.lcols[c] % 16 == 0;
            const uint32_t per = (uint32_t)o0.nimg + 1, cb = (uint32_t)(o0.levels * o0.esize);
            auto on_device = [&](int slot) { return plan.field_on_device.empty() || plan.field_on_device[slot]; };
            bool devices = true;
            for (size_t j = a; j < b && devices; ++j)
            {
                devices = on_device(plan.lowners[j].slot);
                for (int i = 0; i < plan.lowners[j].nimg; ++i) devices = devices && on_device(plan.lowners[j].img_slot[i]);
            }
            const bool bulkable = plan.gather_bulk > 0 && plan.shard_mode == 0 && aligned && devices && o0.s_ls == 1 &&
                                  o0.d_ls == 1 && cb % 16 == 0 && cb <= (uint32_t)k_bgather_zero &&
                                  per * cb <= (uint32_t)k_bulk_stage;
            const size_t nb = bulkable ? (b - a) * (size_t)plan.gather_bulk / 4 : 0;
            if (nb > 0)
            {
                const uint32_t cap = std::min<uint32_t>((uint32_t)k_bulk_stage / (per * cb), (uint32_t)k_bgather_entries / per);
                for (size_t j = 0; j < nb; j += cap)
                {
                    bgtile t{};
                    t.nown = (uint32_t)std::min<size_t>(cap, nb - j), t.nimg = per - 1, t.col_bytes = cb;
                    t.levels = (uint32_t)o0.levels, t.esize = (uint32_t)o0.esize;
                    const size_t blk0 = plan.bgt_blk.size();
                    plan.bgt_blk.resize(blk0 + k_bgather_entries, 0);
                    std::copy(plan.lcols.begin() + (int64_t)(group0 + j * per), plan.lcols.begin() + (int64_t)(group0 + (j + t.nown) * per),
                        plan.bgt_blk.begin() + (int64_t)blk0);
                    plan.bgt.push_back(t);
                    plan.bgt_first.push_back((int)(group0 + j * per));
                }
            }
            // the other owners of the group: element tiles of list_gather_kernel
            const uint32_t col0 = group0 + (uint32_t)(nb * per);
            const uint32_t gc = (uint32_t)(gather_per_thread(o0.nimg) * k_gather_block);
            const uint32_t n = (uint32_t)((int64_t)(b - a - nb) * o0.levels);
            const fast_div f0 = fast_div::make((uint32_t)o0.levels);
            for (uint32_t e0 = 0; e0 < n; e0 += gc)
            {
                gtile t{};
                t.e0 = e0, t.count = std::min(gc, n - e0);
                t.o0 = o0.s_ls;
                t.img[0].t0 = o0.d_ls;
                t.n0 = f0.d, t.m0 = f0.m, t.l0 = (uint8_t)f0.l;
                t.n1 = 1, t.m1 = 1, t.l1 = 0;
                t.esize = (uint8_t)o0.esize;
                t.nimg = (uint8_t)o0.nimg;
                t.kind = 1;
                t.col0 = col0;
                t.cls = (uint8_t)class_of_g(t);
                plan.gt.push_back(t);
            }
            a = b;
        }
    }
    // column blocks of the unstructured gather tiles: a tile's slice of the column table, which
    // its CTA loads beside the record instead of after it (one dependent round trip fewer)
    plan.gblk.assign((plan.gt.size() - (size_t)plan.gt_boxes) * k_gblock_entries, 0);
    for (size_t i = (size_t)plan.gt_boxes; i < plan.gt.size(); ++i)
    {
        auto& t = plan.gt[i];
        const uint64_t per = (uint64_t)t.nimg + 1;
        const uint64_t first = t.col0 + (uint64_t)(t.e0 / t.n0) * per;
        const uint64_t n = ((uint64_t)(t.e0 + t.count - 1) / t.n0 - t.e0 / t.n0 + 1) * per;
        t.pad[0] = n <= (uint64_t)k_gblock_entries ? 1 : 0;
        if (t.pad[0])
            std::copy(plan.lcols.begin() + (int64_t)first, plan.lcols.begin() + (int64_t)(first + n),
                plan.gblk.begin() + (int64_t)(i - plan.gt_boxes) * k_gblock_entries);
    }

    // ---- phased adjoint kernels (boxes without a gather form, lists without one)
    auto box_rows = [&](int i) { return (int64_t)plan.boxes[i].n1 * plan.boxes[i].n2; };
    auto box_len = [&](int i) { return std::max<int64_t>(1, 4096 / plan.boxes[i].n0); };
    auto list_len = [&](const list_desc& l) { return std::max<int64_t>(1, 4096 / l.levels); };
    auto split = [&](int desc, int kind, int64_t rows, int64_t len, std::vector<tile>& out) {
        for (int64_t st = 0; st < rows; st += len)
            out.push_back(tile{desc, kind, (uint32_t)st, (uint32_t)std::min<int64_t>(len, rows - st)});
    };
    plan.adj_btiles.clear();
    plan.adj_ltiles.clear();
    plan.adj_bphase_range.clear();
    plan.adj_lphase_range.clear();
    int nph = 0;
    if (!plan.gather_ok)
        for (int p : plan.box_phase) nph = std::max(nph, p + 1);
    if (!plan.list_gather_ok)
        for (int p : plan.list_phase) nph = std::max(nph, p + 1);
    for (int ph = 0; ph < nph; ++ph)
    {
        int begin = (int)plan.adj_btiles.size();
        if (!plan.gather_ok)
            for (int i = 0; i < (int)plan.boxes.size(); ++i)
                if (plan.box_phase[i] == ph) split(i, 0, box_rows(i), box_len(i), plan.adj_btiles);
        plan.adj_bphase_range.push_back({begin, (int)plan.adj_btiles.size() - begin});
        begin = (int)plan.adj_ltiles.size();
        if (!plan.list_gather_ok)
            for (int i = 0; i < (int)plan.adj_lists.size(); ++i)
                if (plan.list_phase[i] == ph) split(i, 1, plan.adj_lists[i].count, list_len(plan.adj_lists[i]), plan.adj_ltiles);
        plan.adj_lphase_range.push_back({begin, (int)plan.adj_ltiles.size() - begin});
    }
}

void release_graph(ghexb_plan_s& plan)
{
    if (plan.exec) cudaGraphExecDestroy(plan.exec), plan.exec = nullptr;
    if (plan.graph) cudaGraphDestroy(plan.graph), plan.graph = nullptr;
    if (plan.adj_exec) cudaGraphExecDestroy(plan.adj_exec), plan.adj_exec = nullptr;
    if (plan.adj_graph) cudaGraphDestroy(plan.adj_graph), plan.adj_graph = nullptr;
}

void launch_plan(ghexb_plan_s& plan, int form, cudaStream_t stream)
{
    if (plan.forms_stale && (form == GHEXB_FORM_PER_FIELD || form == GHEXB_FORM_PER_BOX))
    {
        host_stager st(plan, stream);
        st.put(plan.d_xp, plan.xp);
        st.put(plan.d_xb, plan.xb);
        st.commit();
        plan.forms_stale = false;
    }
    auto run = [&](const xtile* base, const int32_t* blocks, std::pair<int, int> r) {
        if (r.second <= 0) return;
        check_cuda(launch_exchange(base + r.first, r.second, plan.per_thread, plan.block, stream, plan.d_idx,
                       plan.idx.size() * sizeof(int32_t), blocks ? blocks + (size_t)r.first * k_block_ints : nullptr),
            "exchange kernel launch");
    };
    switch (form)
    {
        case GHEXB_FORM_BATCHED:
        {
            // the staged kernel, and the bulk kernel when the element kernel has work too, run on
            // the second stream beside the element kernel
            launch_staged_plan(plan, stream);
            const bool side_bulk = !plan.bt.empty() && !plan.xf.empty();
            if (side_bulk)
            {
                if (plan.sitems.empty())
                {
                    ensure_side_stream(plan);
                    check_cuda(cudaEventRecord(plan.fork_event, stream), "cudaEventRecord(fork)");
                    check_cuda(cudaStreamWaitEvent(plan.side_stream, plan.fork_event, 0), "cudaStreamWaitEvent(fork)");
                }
                check_cuda(launch_bulk(plan.d_bt, plan.d_bt_blk, plan.bmaps.empty() ? nullptr : plan.d_bmaps, (int)plan.bt.size(),
                               plan.d_status, plan.side_stream),
                    "bulk kernel launch");
                check_cuda(cudaEventRecord(plan.join_event, plan.side_stream), "cudaEventRecord(join)");
            }
            else
                check_cuda(launch_bulk(plan.d_bt, plan.d_bt_blk, plan.bmaps.empty() ? nullptr : plan.d_bmaps, (int)plan.bt.size(),
                           plan.d_status, stream),
                    "bulk kernel launch");
            run(plan.d_xf, plan.xf_blk.empty() ? nullptr : plan.d_xf_blk, {0, (int)plan.xf.size()});
            if (!plan.sitems.empty() || side_bulk)
                check_cuda(cudaStreamWaitEvent(stream, plan.join_event, 0), "cudaStreamWaitEvent(join)");
            break;
        }
        case GHEXB_FORM_PER_FIELD:
            for (const auto& r : plan.xp_field) run(plan.d_xp, plan.xp_blk.empty() ? nullptr : plan.d_xp_blk, r);
            break;
        case GHEXB_FORM_PER_BOX:
            for (const auto& r : plan.xb_box) run(plan.d_xb, plan.xb_blk.empty() ? nullptr : plan.d_xb_blk, r);
            for (const auto& r : plan.xb_list) run(plan.d_xb, plan.xb_blk.empty() ? nullptr : plan.d_xb_blk, r);
            break;
        default: throw error(GHEXB_ERR_INVALID, "unknown exchange form " + std::to_string(form));
    }
}

void graph_launch_plan(ghexb_plan_s& plan, cudaStream_t stream)
{
    if (!plan.exec)
    {
        check_cuda(cudaStreamBeginCapture(plan.cap_stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        std::string err;
        try
        {
            launch_plan(plan, GHEXB_FORM_BATCHED, plan.cap_stream);
        }
        catch (const error& e)
        {
            err = e.what();
        }
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(plan.cap_stream, &g);
        if (!err.empty())
        {
            if (g) cudaGraphDestroy(g);
            throw error(GHEXB_ERR_CUDA, err);
        }
        check_cuda(ce, "cudaStreamEndCapture");
        plan.graph = g;
        check_cuda(cudaGraphInstantiate(&plan.exec, plan.graph, 0), "cudaGraphInstantiate");
    }
    check_cuda(cudaGraphLaunch(plan.exec, stream), "cudaGraphLaunch");
}

namespace
{
// Launches of one adjoint: the gather kernels, then the phases of what has no gather form.
void adjoint_launches(ghexb_plan_s& plan, cudaStream_t stream)
{
    check_cuda(launch_gather(plan.d_gt, plan.gt_boxes, stream), "adjoint kernel launch");
    check_cuda(launch_list_gather(plan.d_gt + plan.gt_boxes, (int)plan.gt.size() - plan.gt_boxes, plan.d_lcols,
                   plan.gblk.empty() ? nullptr : plan.d_gblk, stream),
        "adjoint kernel launch");
    // the bulk gather kernel, on the second stream when other adjoint kernels run (its owners and
    // images are no other kernel's)
    const bool side_bulk = !plan.bgt.empty() && (!plan.gt.empty() || !plan.adj_btiles.empty() || !plan.adj_ltiles.empty());
    if (side_bulk)
    {
        ensure_side_stream(plan);
        check_cuda(cudaEventRecord(plan.fork_event, stream), "cudaEventRecord(fork)");
        check_cuda(cudaStreamWaitEvent(plan.side_stream, plan.fork_event, 0), "cudaStreamWaitEvent(fork)");
        check_cuda(launch_bulk_gather(plan.d_bgt, plan.d_bgt_blk, (int)plan.bgt.size(), plan.d_status, plan.side_stream),
            "bulk gather kernel launch");
        check_cuda(cudaEventRecord(plan.join_event, plan.side_stream), "cudaEventRecord(join)");
    }
    else
        check_cuda(launch_bulk_gather(plan.d_bgt, plan.d_bgt_blk, (int)plan.bgt.size(), plan.d_status, stream),
            "bulk gather kernel launch");
    const int sms = plan.ctx ? plan.ctx->num_sms : 148;
    auto grid = [&](int n) { return std::min(n, 4 * sms); };
    for (size_t ph = 0; ph < plan.adj_bphase_range.size(); ++ph)
    {
        const auto rb = plan.adj_bphase_range[ph];
        const auto rl = plan.adj_lphase_range[ph];
        if (rb.second > 0)
            check_cuda(launch_box_adjoint(plan.d_boxes, plan.d_adj_btiles + rb.first, rb.second, plan.d_counters,
                           grid(rb.second), 256, stream),
                "adjoint kernel launch");
        if (rl.second > 0)
            check_cuda(launch_list_adjoint(plan.d_adj_lists, plan.d_adj_ltiles + rl.first, rl.second, plan.d_counters + 2,
                           grid(rl.second), 256, stream),
                "adjoint kernel launch");
    }
    if (side_bulk) check_cuda(cudaStreamWaitEvent(stream, plan.join_event, 0), "cudaStreamWaitEvent(join)");
}
} // namespace

void adjoint_plan(ghexb_plan_s& plan, cudaStream_t stream)
{
    if (!plan.adjoint_ok) throw error(GHEXB_ERR_INVALID, plan.adjoint_reason);
    // one kernel is launched as it is (a one-node graph was never faster than the kernel alone)
    if (plan.adjoint_launches() == 1)
    {
        adjoint_launches(plan, stream);
        return;
    }
    if (!plan.adj_exec)
    {
        check_cuda(cudaStreamBeginCapture(plan.cap_stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        std::string err;
        try
        {
            adjoint_launches(plan, plan.cap_stream);
        }
        catch (const error& e)
        {
            err = e.what();
        }
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(plan.cap_stream, &g);
        if (!err.empty())
        {
            if (g) cudaGraphDestroy(g);
            throw error(GHEXB_ERR_CUDA, err);
        }
        check_cuda(ce, "cudaStreamEndCapture");
        plan.adj_graph = g;
        check_cuda(cudaGraphInstantiate(&plan.adj_exec, plan.adj_graph, 0), "cudaGraphInstantiate");
    }
    check_cuda(cudaGraphLaunch(plan.adj_exec, stream), "cudaGraphLaunch");
}

namespace
{
// stream-ordered rewrite of the descriptor tables the phased adjoint kernels read
void put_descriptors(ghexb_plan_s& plan, cudaStream_t stream)
{
    host_stager st(plan, stream);
    st.put(plan.d_boxes, plan.boxes);
    st.put(plan.d_lists, plan.lists);
    st.put(plan.d_adj_lists, plan.adj_lists);
    st.commit();
}
} // namespace

void rebind_plan(ghexb_plan_s& plan, void* const* data, int n, cudaStream_t stream)
{
    if (plan.shard_mode != 0) throw error(GHEXB_ERR_INVALID, "a sharded plan cannot be rebound: build a new one");
    if (n != (int)plan.fields.size())
        throw error(GHEXB_ERR_INVALID, "rebind needs one pointer per field of the plan (" +
                                           std::to_string(plan.fields.size()) + ")");
    for (int i = 0; i < n; ++i)
    {
        if (!data[i]) throw error(GHEXB_ERR_INVALID, "null data pointer");
        if (reinterpret_cast<uintptr_t>(data[i]) % plan.fields[i].esize != 0)
            throw error(GHEXB_ERR_INVALID, "data pointer is not aligned to its element size");
    }
    for (size_t i = 0; i < plan.lists.size(); ++i)
        if (plan.lists[i].unit == 16 && (reinterpret_cast<uintptr_t>(data[plan.list_src_slot[i]]) % 16 ||
                                           reinterpret_cast<uintptr_t>(data[plan.list_dst_slot[i]]) % 16))
            throw error(GHEXB_ERR_INVALID, "rebind: 16-byte column alignment of the plan is not met by the new memory");
    for (int i = 0; i < n; ++i) check_accessible(data[i], (size_t)(field_span(plan.fields[i]) * plan.fields[i].esize));
    const relocator R(plan.fields, data);
    for (int i = 0; i < n; ++i) plan.fields[i].data = static_cast<char*>(data[i]);
    for (size_t i = 0; i < plan.boxes.size(); ++i)
    {
        plan.boxes[i].src = plan.fields[plan.box_src_slot[i]].data + plan.box_src_off[i];
        plan.boxes[i].dst = plan.fields[plan.box_dst_slot[i]].data + plan.box_dst_off[i];
    }
    for (size_t i = 0; i < plan.lists.size(); ++i)
    {
        plan.lists[i].src = plan.fields[plan.list_src_slot[i]].data + plan.list_src_off[i];
        plan.lists[i].dst = plan.fields[plan.list_dst_slot[i]].data + plan.list_dst_off[i];
    }
    for (size_t i = 0; i < plan.adj_lists.size(); ++i)
    {
        plan.adj_lists[i].src = plan.fields[plan.adj_src_slot[i]].data + plan.adj_src_off[i];
        plan.adj_lists[i].dst = plan.fields[plan.adj_dst_slot[i]].data + plan.adj_dst_off[i];
    }
    if (plan.staged_mode > 0 || !plan.bmaps.empty())
    {
        // tensor maps hold addresses, and which boxes a map can load depends on the alignment of
        // the new memory: the tables are rebuilt (and the graph recaptured on its next launch)
        put_descriptors(plan, stream);
        retile(plan, stream);
        return;
    }
    // stream-ordered rewrite of the tables. The tile tables keep their size and device address,
    // so a captured graph stays valid. Their pointers move with the fields (the same tables as a
    // rebuild gives: ghexb_plan_check compares the two), else they are rebuilt.
    // Moved tables keep their index blocks (indices do not move), and the per-field and per-box
    // tables are uploaded when one of those forms is launched next (forms_stale).
    host_stager st(plan, stream);
    if (R.ok)
    {
        relocate_tiles(plan, R);
        plan.forms_stale = true;
    }
    else
    {
        build_tiles(plan, plan.d_idx);
        st.put(plan.d_xf_blk, plan.xf_blk);
        st.put(plan.d_xp_blk, plan.xp_blk);
        st.put(plan.d_xb_blk, plan.xb_blk);
        st.put(plan.d_xp, plan.xp);
        st.put(plan.d_xb, plan.xb);
        plan.forms_stale = false;
    }
    st.put(plan.d_xf, plan.xf);
    st.put(plan.d_gt, plan.gt);
    st.put(plan.d_lcols, plan.lcols);
    st.put(plan.d_gblk, plan.gblk);
    st.put(plan.d_bt, plan.bt);
    st.put(plan.d_bt_blk, plan.bt_blk);
    st.put(plan.d_bgt, plan.bgt);
    st.put(plan.d_bgt_blk, plan.bgt_blk);
    st.put(plan.d_boxes, plan.boxes);
    st.put(plan.d_lists, plan.lists);
    st.put(plan.d_adj_lists, plan.adj_lists);
    st.commit();
}

// The size of the adjoint's gather tiles of short rows (gather_scale -1, 0, 1, 2), timed like the
// forward candidates: each adjoint after a cold-L2 read outside its events, the mean per launch.
// The adjoint updates the fields in place, so their memory (merged spans) is saved to a device
// buffer first and restored after; the tuning is skipped, keeping the current size, when a field
// is in host memory or the device has no room for the copy.
void autotune_adjoint(ghexb_plan_s& plan, cudaStream_t stream, int repeats)
{
    std::vector<std::pair<uintptr_t, uintptr_t>> spans;
    for (size_t i = 0; i < plan.fields.size(); ++i)
    {
        if (i < plan.field_on_device.size() && !plan.field_on_device[i]) return;
        const uintptr_t lo = reinterpret_cast<uintptr_t>(plan.fields[i].data);
        spans.push_back({lo, lo + field_bytes(plan.fields[i])});
    }
    std::sort(spans.begin(), spans.end());
    std::vector<std::pair<uintptr_t, uintptr_t>> merged;
    for (const auto& sp : spans)
        if (!merged.empty() && sp.first <= merged.back().second) merged.back().second = std::max(merged.back().second, sp.second);
        else merged.push_back(sp);
    size_t saved_bytes = 0;
    for (const auto& m : merged) saved_bytes += (m.second - m.first + 255) & ~(size_t)255;
    char* saved = nullptr;
    if (cudaMalloc(&saved, std::max<size_t>(saved_bytes, 1)) != cudaSuccess)
    {
        cudaGetLastError();
        return;
    }
    auto copy_fields = [&](bool restore) {
        size_t off = 0;
        for (const auto& m : merged)
        {
            char* f = reinterpret_cast<char*>(m.first);
            const size_t n = m.second - m.first;
            check_cuda(cudaMemcpyAsync(restore ? f : saved + off, restore ? saved + off : f, n, cudaMemcpyDeviceToDevice, stream),
                       "cudaMemcpyAsync(adjoint tuning copy)");
            off += (n + 255) & ~(size_t)255;
        }
    };
    int l2 = 0;
    check_cuda(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, plan.ctx->device), "cudaDeviceGetAttribute");
    const size_t flush_bytes = std::max<size_t>(2 * (size_t)l2, 64u << 20);
    uint4* flush = nullptr;
    unsigned* sink = nullptr;
    std::vector<cudaEvent_t> ev(2 * (size_t)repeats, nullptr);
    auto cleanup = [&]() {
        if (flush) cudaFree(flush);
        if (sink) cudaFree(sink);
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    };
    const int start = plan.gather_scale, start_bulk = plan.gather_bulk;
    int best_scale = start, best_bulk = start_bulk;
    float best = 1e30f;
    bool bulk_candidates = false;
    for (const auto& o : plan.lowners) bulk_candidates = bulk_candidates || (o.s_ls == 1 && o.d_ls == 1);
    try
    {
        copy_fields(false);
        check_cuda(cudaMalloc(&flush, flush_bytes), "cudaMalloc(l2 flush)");
        check_cuda(cudaMemsetAsync(flush, 0, flush_bytes, stream), "cudaMemsetAsync(l2 flush)");
        check_cuda(cudaMalloc(&sink, sizeof(unsigned)), "cudaMalloc(l2 flush sink)");
        for (auto& e : ev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        const int fgrid = (plan.ctx ? plan.ctx->num_sms : 148) * 8;
        // the gather-tile sizes of the box cells, then, at the best size, the bulk gather kernel's
        // shares of the unstructured owners
        std::vector<std::pair<int, int>> cands;
        for (int scale : {-1, 0, 1, 2}) cands.push_back({scale, start_bulk});
        for (size_t ci = 0; ci < cands.size(); ++ci)
        {
            const int scale = cands[ci].first;
            plan.gather_scale = scale, plan.gather_bulk = cands[ci].second;
            retile(plan, stream);
            if (ci > 3 && plan.gather_bulk > 0 && plan.bgt.empty()) continue; // nothing for the bulk kernel
            for (int w = 0; w < 3; ++w) adjoint_plan(plan, stream);
            for (int r = 0; r < repeats; ++r)
            {
                check_cuda(launch_l2_flush(flush, flush_bytes / 16, sink, fgrid, stream), "l2 flush");
                check_cuda(cudaEventRecord(ev[2 * r], stream), "cudaEventRecord");
                adjoint_plan(plan, stream);
                check_cuda(cudaEventRecord(ev[2 * r + 1], stream), "cudaEventRecord");
            }
            check_cuda(cudaEventSynchronize(ev[2 * repeats - 1]), "cudaEventSynchronize");
            float total = 0.f;
            for (int r = 0; r < repeats; ++r)
            {
                float ms = 0.f;
                check_cuda(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]), "cudaEventElapsedTime");
                total += ms;
            }
            // a bulk candidate whose waits gave up is not a result
            bool failed = false;
            if (!plan.bgt.empty() && plan.d_status)
            {
                unsigned st = 0;
                check_cuda(cudaMemcpyAsync(&st, plan.d_status, sizeof st, cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync(status)");
                check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
                if (st) check_cuda(cudaMemsetAsync(plan.d_status, 0, sizeof st, stream), "cudaMemsetAsync(status)");
                failed = st != 0;
            }
            if (!failed && total < best) best = total, best_scale = scale, best_bulk = plan.gather_bulk;
            if (ci == 3 && bulk_candidates)
                for (int share : {0, 1, 2, 3, 4})
                    if (share != start_bulk) cands.push_back({best_scale, share});
        }
    }
    catch (...)
    {
        try
        {
            copy_fields(true);
        }
        catch (...)
        {
        }
        cudaStreamSynchronize(stream);
        cleanup();
        cudaFree(saved);
        plan.gather_scale = start, plan.gather_bulk = start_bulk;
        throw;
    }
    cleanup();
    plan.gather_scale = best_scale, plan.gather_bulk = best_bulk;
    retile(plan, stream);
    copy_fields(true);
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    cudaFree(saved);
}

void autotune_plan(ghexb_plan_s& plan, cudaStream_t stream, int repeats)
{
    if (repeats < 1) repeats = 10;
    struct cand
    {
        int k, block;
        bool pairs;
        int mode, stages, stage_bytes, consumers, ctas;
        int bulk;
    };
    const cand start{plan.per_thread, plan.block, plan.use_pairs, plan.staged_mode, plan.stages, plan.stage_bytes,
        plan.stage_consumers, plan.stage_ctas_per_sm, plan.bulk_share};
    // the element kernel alone first; then, with its best shape, the bulk kernel taking a share of
    // the lists beside it, and the staged form beside it
    std::vector<cand> cands;
    for (int k : {4, 8, 16})
        for (int block : {128, 256, 512})
            for (bool pairs : {false, true})
                if (!pairs || !plan.pairs.empty()) cands.push_back({k, block, pairs, 0, start.stages, start.stage_bytes,
                                                       start.consumers, start.ctas, 0});
    const bool stageable = !plan.boxes.empty() && plan.shard_mode == 0;
    bool bulkable = false;
    for (const auto& l : plan.lists) bulkable = bulkable || (l.unit == 16 && plan.shard_mode == 0);
    const size_t n_element = cands.size();

    // every timed launch starts with a cold L2: read a buffer of twice the L2 size first
    int l2 = 0;
    check_cuda(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, plan.ctx->device), "cudaDeviceGetAttribute");
    const size_t flush_bytes = std::max<size_t>(2 * (size_t)l2, 64u << 20);
    uint4* flush = nullptr;
    unsigned* sink = nullptr;
    std::vector<cudaEvent_t> ev(2 * (size_t)repeats, nullptr);
    auto cleanup = [&]() {
        if (flush) cudaFree(flush);
        if (sink) cudaFree(sink);
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    };
    float best = 1e30f;
    cand bestc = start;
    auto apply = [&](const cand& c) {
        plan.per_thread = c.k, plan.block = c.block, plan.use_pairs = c.pairs;
        plan.staged_mode = c.mode, plan.stages = c.stages, plan.stage_bytes = c.stage_bytes;
        plan.stage_consumers = c.consumers, plan.stage_ctas_per_sm = c.ctas;
        plan.bulk_share = c.bulk;
        retile(plan, stream);
    };
    try
    {
        check_cuda(cudaMalloc(&flush, flush_bytes), "cudaMalloc(l2 flush)");
        check_cuda(cudaMemsetAsync(flush, 0, flush_bytes, stream), "cudaMemsetAsync(l2 flush)");
        check_cuda(cudaMalloc(&sink, sizeof(unsigned)), "cudaMalloc(l2 flush sink)");
        for (auto& e : ev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        const int fgrid = (plan.ctx ? plan.ctx->num_sms : 148) * 8;
        for (size_t ci = 0; ci < cands.size(); ++ci)
        {
            const cand& c = cands[ci];
            apply(c);
            if (c.mode > 0 && plan.sitems.empty()) continue; // nothing to stage
            if (c.bulk > 0 && plan.bt.empty()) continue;      // nothing for the bulk kernel
            for (int w = 0; w < 3; ++w) graph_launch_plan(plan, stream); // capture and warm-up
            // the graph launches queued back to back (the form the batched exchange runs in, where
            // a second stream's fork and join are graph edges), each after a cold-L2 read outside
            // its events, as an application's exchanges follow its other kernels; the mean time
            for (int r = 0; r < repeats; ++r)
            {
                check_cuda(launch_l2_flush(flush, flush_bytes / 16, sink, fgrid, stream), "l2 flush");
                check_cuda(cudaEventRecord(ev[2 * r], stream), "cudaEventRecord");
                graph_launch_plan(plan, stream);
                check_cuda(cudaEventRecord(ev[2 * r + 1], stream), "cudaEventRecord");
            }
            check_cuda(cudaEventSynchronize(ev[2 * repeats - 1]), "cudaEventSynchronize");
            float total = 0.f;
            for (int r = 0; r < repeats; ++r)
            {
                float ms = 0.f;
                check_cuda(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]), "cudaEventElapsedTime");
                total += ms;
            }
            // a staged or bulk candidate whose waits gave up is not a result
            if ((c.mode > 0 || c.bulk > 0) && plan.d_status)
            {
                unsigned st = 0;
                check_cuda(cudaMemcpyAsync(&st, plan.d_status, sizeof st, cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync(status)");
                check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
                if (st)
                {
                    check_cuda(cudaMemsetAsync(plan.d_status, 0, sizeof st, stream), "cudaMemsetAsync(status)");
                    continue;
                }
            }
            if (total < best) best = total, bestc = c;
            if (ci + 1 == n_element)
            {
                const cand e = bestc;
                // the bulk kernel beside the best element-kernel shape
                if (bulkable)
                    for (int share : {1, 2, 3, 4})
                        cands.push_back({e.k, e.block, e.pairs, 0, e.stages, e.stage_bytes, e.consumers, e.ctas, share});
                // the staged form beside it
                if (stageable)
                    for (int mode : {1, 2})
                        for (const auto& sh : std::vector<std::array<int, 4>>{{8, 16384, 4, 1}, {6, 16384, 8, 1},
                                 {4, 16384, 4, 2}, {12, 8192, 4, 1}})
                            cands.push_back({e.k, e.block, e.pairs, mode, sh[0], sh[1], sh[2], sh[3], 0});
            }
        }
    }
    catch (...)
    {
        cleanup();
        throw;
    }
    cleanup();
    apply(bestc);
    // (not on a sharded plan: its adjoint zeroes halos in other processes' memory)
    if (plan.adjoint_ok && plan.gather_ok && plan.shard_mode == 0) autotune_adjoint(plan, stream, repeats);
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}
} // namespace ghexb

ghexb_plan_s::~ghexb_plan_s()
{
    ghexb::release_graph(*this);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (side_stream) cudaStreamDestroy(side_stream);
    for (auto& b : h_stage)
    {
        if (b.done) cudaEventSynchronize(b.done), cudaEventDestroy(b.done);
        if (b.ptr) cudaFreeHost(b.ptr);
    }
    if (fork_event) cudaEventDestroy(fork_event);
    if (join_event) cudaEventDestroy(join_event);
    for (void* p : {(void*)d_smaps, (void*)d_sitems, (void*)d_status, (void*)d_xf_blk, (void*)d_xp_blk, (void*)d_xb_blk,
             (void*)d_gblk, (void*)d_bt, (void*)d_bt_blk, (void*)d_bgt, (void*)d_bgt_blk, (void*)d_bmaps})
        if (p) cudaFree(p);
    for (void* p : {(void*)d_boxes, (void*)d_lists, (void*)d_adj_lists, (void*)d_idx, (void*)d_xf, (void*)d_xp,
             (void*)d_xb, (void*)d_gt, (void*)d_lcols, (void*)d_adj_btiles, (void*)d_adj_ltiles, (void*)d_counters})
        if (p) cudaFree(p);
}

int64_t ghexb_plan_s::num_tiles() const
{
    int64_t n = 0;
    for (const auto& t : xf) n += t.count > 0;
    return n;
}

int ghexb_plan_s::adjoint_launches() const
{
    int n = (gt_boxes > 0) + ((int)gt.size() > gt_boxes) + !bgt.empty();
    for (size_t ph = 0; ph < adj_bphase_range.size(); ++ph)
        n += (adj_bphase_range[ph].second > 0) + (adj_lphase_range[ph].second > 0);
    return n;
}

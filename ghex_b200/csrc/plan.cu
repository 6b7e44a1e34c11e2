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
#include <cstring>
#include <map>
#include <unordered_map>

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

template<typename T>
void upload(T*& dptr, const std::vector<T>& v)
{
    if (dptr) cudaFree(dptr), dptr = nullptr;
    if (v.empty()) return;
    check_cuda(cudaMalloc(&dptr, v.size() * sizeof(T)), "cudaMalloc(plan table)");
    check_cuda(cudaMemcpy(dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice),
        "cudaMemcpy(plan table)");
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

    // Emits a box descriptor from a list of axes (any order) and the element offsets of the
    // box origin in source and destination.
    void emit_box(const ghexb_field_s& src, int src_slot, const ghexb_field_s& dst, int dst_slot,
        std::vector<axis> ax, int64_t src_origin, int64_t dst_origin, uint64_t xor_mask,
        int logical, const owner_region& reg)
    {
        std::stable_sort(ax.begin(), ax.end(), [](const axis& a, const axis& b) { return a.order > b.order; });
        while (ax.size() < 4) ax.push_back(axis{1, 0, 0, -1});
        if (ax.size() > 4) throw error(GHEXB_ERR_INTERNAL, "box with more than 4 axes");
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
        box_desc b{};
        b.src = src.data + src_origin * src.esize;
        b.dst = dst.data + dst_origin * dst.esize;
        b.n0 = ax[0].n, b.n1 = ax[1].n, b.n2 = ax[2].n, b.n3 = ax[3].n;
        b.s0 = (int32_t)ax[0].ss, b.s1 = (int32_t)ax[1].ss, b.s2 = (int32_t)ax[2].ss, b.s3 = (int32_t)ax[3].ss;
        b.d0 = (int32_t)ax[0].ds, b.d1 = (int32_t)ax[1].ds, b.d2 = (int32_t)ax[2].ds, b.d3 = (int32_t)ax[3].ds;
        b.esize = (uint32_t)dst.esize;
        b.field = (uint32_t)logical;
        b.xor_mask = xor_mask;
        b.div0 = fast_div::make((uint32_t)b.n0);
        b.div1 = fast_div::make((uint32_t)b.n1);
        b.div2 = fast_div::make((uint32_t)b.n2);
        plan.boxes.push_back(b);
        plan.box_src_slot.push_back(src_slot);
        plan.box_dst_slot.push_back(dst_slot);
        owner_region r = reg;
        r.field = src_slot;
        box_owner.push_back(r);
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
            const int64_t sl = sp.gfirst[a] - sdom.first[a] + src.offsets[a];
            const int64_t sh = sp.glast[a] - sdom.first[a] + src.offsets[a];
            check_range(dst, a, dl, dh, "destination");
            check_range(src, a, sl, sh, "source");
            dof += dl * estride(dst, a);
            so += sl * estride(src, a);
            ax.push_back(axis{(int)(dh - dl + 1), estride(src, a), estride(dst, a), dst.layout[a]});
            reg.lo[a] = sl, reg.hi[a] = sh;
        }
        if (dst.ndim == D + 1)
        {
            ax.push_back(axis{dst.num_components, estride(src, D), estride(dst, D), dst.layout[D]});
            reg.lo[D] = 0, reg.hi[D] = dst.num_components - 1;
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
        if (!neg0 && !neg1)
        {
            auto ax2 = ax;
            ax2.push_back(axis{nc, sC, estride(dst, 3), dst.layout[3]});
            reg.hi[3] = nc - 1;
            emit_box(src, src_slot, dst, dst_slot, ax2, src_origin, dst_origin, 0, logical, reg);
            return;
        }
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

        // forward descriptor: 16-byte columns when every column is 16-byte aligned
        const bool cols = dst.level_stride == 1 && src.level_stride == 1;
        const bool vec16 = cols && (L * es) % 16 == 0 && (dst.index_stride * es) % 16 == 0 &&
                           (src.index_stride * es) % 16 == 0 &&
                           reinterpret_cast<uintptr_t>(dst.data) % 16 == 0 &&
                           reinterpret_cast<uintptr_t>(src.data) % 16 == 0;
        const int unit = vec16 ? 16 : es;
        const int64_t k = unit / es;
        list_desc l{};
        l.src = src.data;
        l.dst = dst.data;
        l.count = (int32_t)cnt;
        l.levels = (int32_t)(L / k);
        l.s_is = (int32_t)(src.index_stride / k);
        l.s_ls = (int32_t)(vec16 ? 1 : src.level_stride);
        l.d_is = (int32_t)(dst.index_stride / k);
        l.d_ls = (int32_t)(vec16 ? 1 : dst.level_stride);
        l.unit = (uint32_t)unit;
        l.level_fastest = dst.level_stride == 1 ? 1u : 0u;
        l.field = (uint32_t)logical;
        l.divq = fast_div::make((uint32_t)(l.level_fastest ? l.levels : l.count));
        const int64_t span_s = smax * (int64_t)l.s_is + (int64_t)(l.levels - 1) * l.s_ls;
        const int64_t span_d = dmax * (int64_t)l.d_is + (int64_t)(l.levels - 1) * l.d_ls;
        if (cnt * l.levels > k_i32max || span_s > k_i32max || span_d > k_i32max)
            throw error(GHEXB_ERR_RANGE, "an index-list descriptor spans more than 2^31 elements");
        plan.lists.push_back(l);
        plan.list_idx_off.push_back(idx0);
        plan.list_src_slot.push_back(src_slot);
        plan.list_dst_slot.push_back(dst_slot);
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
            list_desc a{};
            a.src = src.data;
            a.dst = dst.data;
            a.count = (int32_t)(e - b);
            a.levels = (int32_t)L;
            a.s_is = (int32_t)src.index_stride;
            a.s_ls = (int32_t)src.level_stride;
            a.d_is = (int32_t)dst.index_stride;
            a.d_ls = (int32_t)dst.level_stride;
            a.unit = (uint32_t)es;
            a.level_fastest = dst.level_stride == 1 ? 1u : 0u;
            a.field = (uint32_t)logical;
            a.divq = fast_div::make((uint32_t)(a.level_fastest ? a.levels : a.count));
            plan.adj_lists.push_back(a);
            plan.adj_idx_off.push_back(idx0 + b);
            plan.adj_didx_off.push_back(idx0 + cnt + b);
            plan.adj_src_slot.push_back(src_slot);
            plan.adj_dst_slot.push_back(dst_slot);
            list_src_field.push_back(src_slot);
            b = e;
        }
    }
};

void make_tiles(const std::vector<box_desc>& boxes, const std::vector<list_desc>& lists,
    const std::vector<int>& box_order, const std::vector<int>& list_order, int tile_elems,
    std::vector<tile>& out)
{
    auto emit = [&](int desc, int kind, int64_t n) {
        for (int64_t s = 0; s < n; s += tile_elems)
            out.push_back(tile{desc, kind, (uint32_t)s, (uint32_t)std::min<int64_t>(tile_elems, n - s)});
    };
    for (int i : box_order)
    {
        const auto& b = boxes[i];
        emit(i, 0, (int64_t)b.n0 * b.n1 * b.n2 * b.n3);
    }
    for (int i : list_order)
    {
        const auto& l = lists[i];
        emit(i, 1, (int64_t)l.count * l.levels);
    }
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
            if (P.kind == pattern_kind::unstructured)
            {
                for (const auto& re : P.domains[d].urecv)
                {
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
                        B.list_pair(dst, Fd[k], src, Fe[k], re.lids, se->lids, logical_of(pi, (int)k));
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

}

void upload_plan(ghexb_plan_s& plan)
{
    // upload index lists, patch device pointers, upload descriptor tables
    upload(plan.d_idx, plan.idx);
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
    upload(plan.d_boxes, plan.boxes);
    upload(plan.d_lists, plan.lists);
    upload(plan.d_adj_lists, plan.adj_lists);
    check_cuda(cudaStreamCreateWithFlags(&plan.cap_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    retile(plan);
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

int64_t check_tables(const ghexb_plan_s& plan)
{
    int64_t checked = 0;
    for (size_t i = 0; i < plan.boxes.size(); ++i)
    {
        const auto& b = plan.boxes[i];
        const auto& sf = plan.fields[plan.box_src_slot[i]];
        const auto& df = plan.fields[plan.box_dst_slot[i]];
        const int64_t ss = field_span(sf), ds = field_span(df);
        const uint32_t n = (uint32_t)((int64_t)b.n0 * b.n1 * b.n2 * b.n3);
        for (uint32_t f = 0; f < n; ++f)
        {
            // the decomposition of box_tile / box_adjoint_tile in kernels.cu
            const uint32_t q0 = b.div0.div(f);
            const int32_t i0 = (int32_t)(f - q0 * (uint32_t)b.n0);
            const uint32_t q1 = b.div1.div(q0);
            const int32_t i1 = (int32_t)(q0 - q1 * (uint32_t)b.n1);
            const uint32_t q2 = b.div2.div(q1);
            const int32_t i2 = (int32_t)(q1 - q2 * (uint32_t)b.n2);
            const int32_t i3 = (int32_t)q2;
            if (i3 >= b.n3) throw error(GHEXB_ERR_INTERNAL, "box decomposition out of range");
            check_offset(sf, b.src, (int64_t)i0 * b.s0 + (int64_t)i1 * b.s1 + (int64_t)i2 * b.s2 + (int64_t)i3 * b.s3, ss, "source");
            check_offset(df, b.dst, (int64_t)i0 * b.d0 + (int64_t)i1 * b.d1 + (int64_t)i2 * b.d2 + (int64_t)i3 * b.d3, ds, "destination");
        }
        checked += n;
    }
    auto check_list = [&](const list_desc& l, int64_t s_off, int64_t d_off, const ghexb_field_s& sf,
                          const ghexb_field_s& df) {
        const int64_t k = l.unit / sf.esize; // elements per unit
        const int64_t ss = field_span(sf), ds = field_span(df);
        const uint32_t n = (uint32_t)((int64_t)l.count * l.levels);
        for (uint32_t f = 0; f < n; ++f)
        {
            const uint32_t q = l.divq.div(f);
            int32_t col, lev;
            if (l.level_fastest) col = (int32_t)q, lev = (int32_t)(f - q * (uint32_t)l.levels);
            else
                lev = (int32_t)q, col = (int32_t)(f - q * (uint32_t)l.count);
            if (col >= l.count || lev >= l.levels) throw error(GHEXB_ERR_INTERNAL, "list decomposition out of range");
            const int64_t so = ((int64_t)plan.idx[s_off + col] * l.s_is + (int64_t)lev * l.s_ls) * k;
            const int64_t dof = ((int64_t)plan.idx[d_off + col] * l.d_is + (int64_t)lev * l.d_ls) * k;
            check_offset(sf, l.src, so, ss, "source");
            check_offset(sf, l.src, so + k - 1, ss, "source");
            check_offset(df, l.dst, dof, ds, "destination");
            check_offset(df, l.dst, dof + k - 1, ds, "destination");
        }
        return (int64_t)n;
    };
    for (size_t i = 0; i < plan.lists.size(); ++i)
        checked += check_list(plan.lists[i], plan.list_idx_off[i], plan.list_idx_off[i] + plan.lists[i].count,
            plan.fields[plan.list_src_slot[i]], plan.fields[plan.list_dst_slot[i]]);
    for (size_t i = 0; i < plan.adj_lists.size(); ++i)
        checked += check_list(plan.adj_lists[i], plan.adj_idx_off[i], plan.adj_didx_off[i],
            plan.fields[plan.adj_src_slot[i]], plan.fields[plan.adj_dst_slot[i]]);
    return checked;
}

void retile(ghexb_plan_s& plan)
{
    release_graph(plan);
    // forward: grouped by logical field
    plan.tiles.clear();
    plan.logical_range.assign(plan.n_logical, {0, 0});
    plan.desc_range.assign(plan.boxes.size() + plan.lists.size(), {0, 0});
    for (int lg = 0; lg < plan.n_logical; ++lg)
    {
        const int begin = (int)plan.tiles.size();
        for (int i = 0; i < (int)plan.boxes.size(); ++i)
        {
            if ((int)plan.boxes[i].field != lg) continue;
            const int b0 = (int)plan.tiles.size();
            make_tiles(plan.boxes, plan.lists, {i}, {}, plan.tile_elems, plan.tiles);
            plan.desc_range[i] = {b0, (int)plan.tiles.size() - b0};
        }
        for (int i = 0; i < (int)plan.lists.size(); ++i)
        {
            if ((int)plan.lists[i].field != lg) continue;
            const int b0 = (int)plan.tiles.size();
            make_tiles(plan.boxes, plan.lists, {}, {i}, plan.tile_elems, plan.tiles);
            plan.desc_range[plan.boxes.size() + i] = {b0, (int)plan.tiles.size() - b0};
        }
        plan.logical_range[lg] = {begin, (int)plan.tiles.size() - begin};
    }
    // adjoint: grouped by phase
    plan.adj_tiles.clear();
    plan.phase_range.clear();
    int nph = 0;
    for (int p : plan.box_phase) nph = std::max(nph, p + 1);
    for (int p : plan.list_phase) nph = std::max(nph, p + 1);
    for (int ph = 0; ph < nph; ++ph)
    {
        const int begin = (int)plan.adj_tiles.size();
        std::vector<int> bo, lo;
        for (int i = 0; i < (int)plan.boxes.size(); ++i)
            if (plan.box_phase[i] == ph) bo.push_back(i);
        for (int i = 0; i < (int)plan.adj_lists.size(); ++i)
            if (plan.list_phase[i] == ph) lo.push_back(i);
        make_tiles(plan.boxes, plan.adj_lists, bo, lo, plan.tile_elems, plan.adj_tiles);
        plan.phase_range.push_back({begin, (int)plan.adj_tiles.size() - begin});
    }
    upload(plan.d_tiles, plan.tiles);
    upload(plan.d_adj_tiles, plan.adj_tiles);
}

void release_graph(ghexb_plan_s& plan)
{
    if (plan.exec) cudaGraphExecDestroy(plan.exec), plan.exec = nullptr;
    if (plan.graph) cudaGraphDestroy(plan.graph), plan.graph = nullptr;
}

void launch_plan(ghexb_plan_s& plan, int form, cudaStream_t stream)
{
    auto run = [&](int begin, int count) {
        if (count <= 0) return;
        check_cuda(launch_exchange(plan.d_boxes, plan.d_lists, plan.d_tiles + begin, count,
                       plan.grid(count), plan.block, stream),
            "exchange kernel launch");
    };
    switch (form)
    {
        case GHEXB_FORM_BATCHED: run(0, (int)plan.tiles.size()); break;
        case GHEXB_FORM_PER_FIELD:
            for (const auto& r : plan.logical_range) run(r.first, r.second);
            break;
        case GHEXB_FORM_PER_BOX:
            for (const auto& r : plan.desc_range) run(r.first, r.second);
            break;
        default: throw error(GHEXB_ERR_INVALID, "unknown exchange form " + std::to_string(form));
    }
}

void graph_launch_plan(ghexb_plan_s& plan, cudaStream_t stream)
{
    if (!plan.exec)
    {
        check_cuda(cudaStreamBeginCapture(plan.cap_stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        cudaError_t le = launch_exchange(plan.d_boxes, plan.d_lists, plan.d_tiles, (int)plan.tiles.size(),
            plan.grid((int)plan.tiles.size()), plan.block, plan.cap_stream);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(plan.cap_stream, &g);
        check_cuda(le, "exchange kernel capture");
        check_cuda(ce, "cudaStreamEndCapture");
        plan.graph = g;
        check_cuda(cudaGraphInstantiate(&plan.exec, plan.graph, 0), "cudaGraphInstantiate");
    }
    check_cuda(cudaGraphLaunch(plan.exec, stream), "cudaGraphLaunch");
}

void adjoint_plan(ghexb_plan_s& plan, cudaStream_t stream)
{
    if (!plan.adjoint_ok) throw error(GHEXB_ERR_INVALID, plan.adjoint_reason);
    for (const auto& r : plan.phase_range)
    {
        if (r.second <= 0) continue;
        check_cuda(launch_adjoint(plan.d_boxes, plan.d_adj_lists, plan.d_adj_tiles + r.first, r.second,
                       plan.grid(r.second), plan.block, stream),
            "adjoint kernel launch");
    }
}

void autotune_plan(ghexb_plan_s& plan, cudaStream_t stream, int repeats)
{
    if (repeats < 1) repeats = 10;
    struct cand
    {
        int tile, block, cps;
    };
    std::vector<cand> cands;
    for (int tile : {2048, 4096, 8192, 16384, 32768})
        for (int block : {128, 256, 512})
            for (int cps : {2, 4, 8, 16})
                if (block * cps <= 2048 && block * cps >= 512) cands.push_back({tile, block, cps});

    // every timed launch starts with a cold L2: read a buffer of twice the L2 size first
    int l2 = 0;
    check_cuda(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, plan.ctx->device), "cudaDeviceGetAttribute");
    const size_t flush_bytes = std::max<size_t>(2 * (size_t)l2, 64u << 20);
    uint4* flush = nullptr;
    unsigned* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        if (flush) cudaFree(flush);
        if (sink) cudaFree(sink);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    float best = 1e30f;
    cand bestc{plan.tile_elems, plan.block, plan.ctas_per_sm};
    try
    {
        check_cuda(cudaMalloc(&flush, flush_bytes), "cudaMalloc(l2 flush)");
        check_cuda(cudaMemsetAsync(flush, 0, flush_bytes, stream), "cudaMemsetAsync(l2 flush)");
        check_cuda(cudaMalloc(&sink, sizeof(unsigned)), "cudaMalloc(l2 flush sink)");
        check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
        check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
        const int fgrid = (plan.ctx ? plan.ctx->num_sms : 148) * 8;
        for (const auto& c : cands)
        {
            plan.tile_elems = c.tile, plan.block = c.block, plan.ctas_per_sm = c.cps;
            retile(plan);
            launch_plan(plan, GHEXB_FORM_BATCHED, stream); // warm-up
            float total = 0.f;
            for (int r = 0; r < repeats; ++r)
            {
                check_cuda(launch_l2_flush(flush, flush_bytes / 16, sink, fgrid, stream), "l2 flush");
                check_cuda(cudaEventRecord(e0, stream), "cudaEventRecord");
                launch_plan(plan, GHEXB_FORM_BATCHED, stream);
                check_cuda(cudaEventRecord(e1, stream), "cudaEventRecord");
                check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
                float ms = 0.f;
                check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
                total += ms;
            }
            if (total < best) best = total, bestc = c;
        }
    }
    catch (...)
    {
        cleanup();
        throw;
    }
    cleanup();
    plan.tile_elems = bestc.tile, plan.block = bestc.block, plan.ctas_per_sm = bestc.cps;
    retile(plan);
}
} // namespace ghexb

ghexb_plan_s::~ghexb_plan_s()
{
    ghexb::release_graph(*this);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    for (void* p : {(void*)d_boxes, (void*)d_lists, (void*)d_adj_lists, (void*)d_idx, (void*)d_tiles, (void*)d_adj_tiles})
        if (p) cudaFree(p);
}

int ghexb_plan_s::grid(int ntiles) const
{
    const int sms = ctx ? ctx->num_sms : 148;
    const int g = sms * ctas_per_sm;
    return ntiles < g ? ntiles : g;
}

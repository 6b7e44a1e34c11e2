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
                list_src_field.push_back(src_slot);
            }
            b = e;
        }
    }
};

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
    // two scheduler counters per forward tile class and per adjoint kernel
    upload(plan.d_counters, std::vector<unsigned>(2 * (ghexb_plan_s::k_classes + 2), 0u));
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
        if (b.n0 < 1 || b.n0 > 256 || b.map.j * (1 << b.map.wlog) < b.n0 || b.map.p * b.map.j > 8)
            throw error(GHEXB_ERR_INTERNAL, "invalid row mapping");
        const uint32_t rows = (uint32_t)((int64_t)b.n1 * b.n2);
        for (uint32_t r = 0; r < rows; ++r)
        {
            // the row decomposition of box_issue / box_drain / box_adjoint_rows in kernels.cu
            const uint32_t q = b.div1.div(r);
            const int64_t i1 = (int64_t)(r - q * (uint32_t)b.n1), i2 = q;
            if (i1 >= b.n1 || i2 >= b.n2) throw error(GHEXB_ERR_INTERNAL, "box decomposition out of range");
            for (int i0 = 0; i0 < b.n0; ++i0)
            {
                check_offset(sf, b.src, i0 * (int64_t)b.s0 + i1 * b.s1 + i2 * b.s2, ss, "source");
                check_offset(df, b.dst, i0 * (int64_t)b.d0 + i1 * b.d1 + i2 * b.d2, ds, "destination");
            }
        }
        checked += (int64_t)rows * b.n0;
    }
    auto check_list = [&](const list_desc& l, int64_t s_off, int64_t d_off, const ghexb_field_s& sf,
                          const ghexb_field_s& df) {
        const int64_t k = l.unit / sf.esize; // elements per unit
        const int64_t ss = field_span(sf), ds = field_span(df);
        if (l.levels < 1 || l.levels > 256) throw error(GHEXB_ERR_INTERNAL, "invalid list descriptor");
        for (int32_t col = 0; col < l.count; ++col)
            for (int32_t lev = 0; lev < l.levels; ++lev)
            {
                const int64_t so = ((int64_t)plan.idx[s_off + col] * l.s_is + (int64_t)lev * l.s_ls) * k;
                const int64_t dof = ((int64_t)plan.idx[d_off + col] * l.d_is + (int64_t)lev * l.d_ls) * k;
                check_offset(sf, l.src, so, ss, "source");
                check_offset(sf, l.src, so + k - 1, ss, "source");
                check_offset(df, l.dst, dof, ds, "destination");
                check_offset(df, l.dst, dof + k - 1, ds, "destination");
            }
        return (int64_t)l.count * l.levels;
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
    build_tiles(plan);
    for (int c = 0; c < ghexb_plan_s::k_classes; ++c)
    {
        upload(plan.d_ftiles[c], plan.ftiles[c]);
        upload(plan.d_ptiles[c], plan.ptiles[c]);
    }
    upload(plan.d_adj_btiles, plan.adj_btiles);
    upload(plan.d_adj_ltiles, plan.adj_ltiles);
}

void build_tiles(ghexb_plan_s& plan)
{
    // Tiles are row ranges. A tile holds about tile_elems elements, fewer for short rows: a row of
    // n0 elements touches at least one 32-byte sector, so the cost per element grows as rows
    // shrink below 256 bytes.
    auto box_rows = [&](int i) { return (int64_t)plan.boxes[i].n1 * plan.boxes[i].n2; };
    auto box_len = [&](int i) {
        const auto& b = plan.boxes[i];
        const int64_t rb = std::min<int64_t>(std::max<int64_t>((int64_t)b.n0 * b.esize, 32), 256);
        const int64_t elems = std::max<int64_t>(256, plan.tile_elems * rb / 256);
        return std::max<int64_t>(1, elems / b.n0);
    };
    auto list_len = [&](const list_desc& l) { return std::max<int64_t>(1, plan.tile_elems / l.levels); };
    auto box_class = [&](int i) { return plan.boxes[i].esize >= 4 ? 0 : 1; };
    auto list_class = [&](int i) { return plan.lists[i].unit >= 8 ? 2 : 3; };
    auto split = [&](int desc, int kind, int64_t rows, int64_t len, std::vector<tile>& out) {
        for (int64_t st = 0; st < rows; st += len)
            out.push_back(tile{desc, kind, (uint32_t)st, (uint32_t)std::min<int64_t>(len, rows - st)});
    };
    // the batched table hands out the most expensive descriptors (shortest rows) first
    std::vector<int> box_order(plan.boxes.size());
    for (size_t i = 0; i < box_order.size(); ++i) box_order[i] = (int)i;
    std::stable_sort(box_order.begin(), box_order.end(), [&](int a, int b) {
        return (int64_t)plan.boxes[a].n0 * plan.boxes[a].esize < (int64_t)plan.boxes[b].n0 * plan.boxes[b].esize;
    });
    plan.box_range.assign(plan.boxes.size(), {0, 0});
    plan.list_range.assign(plan.lists.size(), {0, 0});
    for (int c = 0; c < ghexb_plan_s::k_classes; ++c)
    {
        auto& F = plan.ftiles[c];
        auto& P = plan.ptiles[c];
        F.clear();
        P.clear();
        plan.logical_range[c].assign(plan.n_logical, {0, 0});
        if (c < 2)
        {
            for (int i : box_order)
                if (box_class(i) == c) split(i, 0, box_rows(i), box_len(i), F);
        }
        else
            for (int i = 0; i < (int)plan.lists.size(); ++i)
                if (list_class(i) == c) split(i, 1, plan.lists[i].count, list_len(plan.lists[i]), F);
        for (int lg = 0; lg < plan.n_logical; ++lg)
        {
            const int begin = (int)P.size();
            if (c < 2)
                for (int i : box_order)
                {
                    if ((int)plan.boxes[i].field != lg || box_class(i) != c) continue;
                    const int b0 = (int)P.size();
                    split(i, 0, box_rows(i), box_len(i), P);
                    plan.box_range[i] = {b0, (int)P.size() - b0};
                }
            else
                for (int i = 0; i < (int)plan.lists.size(); ++i)
                {
                    if ((int)plan.lists[i].field != lg || list_class(i) != c) continue;
                    const int b0 = (int)P.size();
                    split(i, 1, plan.lists[i].count, list_len(plan.lists[i]), P);
                    plan.list_range[i] = {b0, (int)P.size() - b0};
                }
            plan.logical_range[c][lg] = {begin, (int)P.size() - begin};
        }
    }
    // adjoint: grouped by phase
    plan.adj_btiles.clear();
    plan.adj_ltiles.clear();
    plan.adj_bphase_range.clear();
    plan.adj_lphase_range.clear();
    int nph = 0;
    for (int p : plan.box_phase) nph = std::max(nph, p + 1);
    for (int p : plan.list_phase) nph = std::max(nph, p + 1);
    for (int ph = 0; ph < nph; ++ph)
    {
        int begin = (int)plan.adj_btiles.size();
        for (int i : box_order)
            if (plan.box_phase[i] == ph) split(i, 0, box_rows(i), box_len(i), plan.adj_btiles);
        plan.adj_bphase_range.push_back({begin, (int)plan.adj_btiles.size() - begin});
        begin = (int)plan.adj_ltiles.size();
        for (int i = 0; i < (int)plan.adj_lists.size(); ++i)
            if (plan.list_phase[i] == ph) split(i, 1, plan.adj_lists[i].count, list_len(plan.adj_lists[i]), plan.adj_ltiles);
        plan.adj_lphase_range.push_back({begin, (int)plan.adj_ltiles.size() - begin});
    }
}

void release_graph(ghexb_plan_s& plan)
{
    if (plan.exec) cudaGraphExecDestroy(plan.exec), plan.exec = nullptr;
    if (plan.graph) cudaGraphDestroy(plan.graph), plan.graph = nullptr;
}

void launch_plan(ghexb_plan_s& plan, int form, cudaStream_t stream)
{
    auto run = [&](int c, int begin, int count) {
        if (count <= 0) return;
        const tile* t = (form == GHEXB_FORM_BATCHED ? plan.d_ftiles[c] : plan.d_ptiles[c]) + begin;
        unsigned* ctr = plan.d_counters + 2 * c;
        const cudaError_t e = c < 2
            ? launch_box_exchange(plan.d_boxes, t, count, c == 0, ctr, plan.grid(count), plan.block, stream)
            : launch_list_exchange(plan.d_lists, t, count, c == 2, ctr, plan.grid(count), plan.block, stream);
        check_cuda(e, "exchange kernel launch");
    };
    switch (form)
    {
        case GHEXB_FORM_BATCHED:
            for (int c = 0; c < ghexb_plan_s::k_classes; ++c) run(c, 0, (int)plan.ftiles[c].size());
            break;
        case GHEXB_FORM_PER_FIELD:
            for (int lg = 0; lg < plan.n_logical; ++lg)
                for (int c = 0; c < ghexb_plan_s::k_classes; ++c)
                    run(c, plan.logical_range[c][lg].first, plan.logical_range[c][lg].second);
            break;
        case GHEXB_FORM_PER_BOX:
            for (size_t i = 0; i < plan.boxes.size(); ++i)
                run(plan.boxes[i].esize >= 4 ? 0 : 1, plan.box_range[i].first, plan.box_range[i].second);
            for (size_t i = 0; i < plan.lists.size(); ++i)
                run(plan.lists[i].unit >= 8 ? 2 : 3, plan.list_range[i].first, plan.list_range[i].second);
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

void adjoint_plan(ghexb_plan_s& plan, cudaStream_t stream)
{
    if (!plan.adjoint_ok) throw error(GHEXB_ERR_INVALID, plan.adjoint_reason);
    for (size_t ph = 0; ph < plan.adj_bphase_range.size(); ++ph)
    {
        const auto rb = plan.adj_bphase_range[ph];
        const auto rl = plan.adj_lphase_range[ph];
        if (rb.second > 0)
            check_cuda(launch_box_adjoint(plan.d_boxes, plan.d_adj_btiles + rb.first, rb.second,
                           plan.d_counters + 2 * ghexb_plan_s::k_classes, plan.grid(rb.second), plan.block, stream),
                "adjoint kernel launch");
        if (rl.second > 0)
            check_cuda(launch_list_adjoint(plan.d_adj_lists, plan.d_adj_ltiles + rl.first, rl.second,
                           plan.d_counters + 2 * ghexb_plan_s::k_classes + 2, plan.grid(rl.second), plan.block, stream),
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
    for (void* p : {(void*)d_boxes, (void*)d_lists, (void*)d_adj_lists, (void*)d_idx, (void*)d_ftiles[0],
             (void*)d_ftiles[1], (void*)d_ftiles[2], (void*)d_ftiles[3], (void*)d_ptiles[0], (void*)d_ptiles[1],
             (void*)d_ptiles[2], (void*)d_ptiles[3], (void*)d_adj_btiles, (void*)d_adj_ltiles, (void*)d_counters})
        if (p) cudaFree(p);
}

int ghexb_plan_s::grid(int ntiles) const
{
    const int sms = ctx ? ctx->num_sms : 148;
    const int g = sms * ctas_per_sm;
    return ntiles < g ? ntiles : g;
}

// Regular structured patterns: halo boxes of every domain, intersected with every domain.
//
// Behaviour follows GHEX 0.4.0:
//  * structured::regular::halo_generator::operator() (structured/regular/halo_generator.hpp:91-146):
//    per dimension a minus / middle / plus interval, the 3^D combinations with dimension 0
//    varying slowest (compute_spaces, :161-195), the centre and empty boxes dropped, then a
//    periodic wrap of the global coordinates with C++ '%' semantics;
//  * halo_generator::intersect (:148-158);
//  * make_pattern_impl<structured grid>::apply (structured/pattern.hpp:214-568): every halo box is
//    intersected with every domain in domain-list order; the pieces are appended to the receive
//    map under the source domain's id (std::map, ascending id), tags are a running counter over
//    all receive entries of the process (:329-365), and send spaces are the receive spaces
//    translated into the sender's local frame (:367-435).
//
// Staged patterns follow structured::regular::make_staged_pattern (structured/regular/
// make_pattern.hpp:47-256): one pattern per dimension, exchanged one after the other.
#include <algorithm>
#include <map>

#include "core.hpp"

namespace ghexb
{
namespace
{
struct box2
{
    coord4 lfirst{}, llast{}, gfirst{}, glast{};
};

// 3^D combinations of the minus/middle/plus intervals; dimension 0 varies slowest.
void combine(int d, int dim, const box2 (&iv)[3], box2& cur, std::vector<box2>& out)
{
    if (d == dim)
    {
        out.push_back(cur);
        return;
    }
    for (int s = 0; s < 3; ++s)
    {
        cur.lfirst[d] = iv[s].lfirst[d];
        cur.llast[d] = iv[s].llast[d];
        cur.gfirst[d] = iv[s].gfirst[d];
        cur.glast[d] = iv[s].glast[d];
        combine(d + 1, dim, iv, cur, out);
    }
}

bool all_le(const coord4& a, const coord4& b, int dim)
{
    for (int i = 0; i < dim; ++i)
        if (a[i] > b[i]) return false;
    return true;
}
} // namespace

namespace
{
// the domain list of a regular pattern, validated
void set_domains(ghexb_pattern_s& p, int dim, const int* halos, int n, const int64_t* ids, const int* first,
    const int* last)
{
    if (dim < 1 || dim > 3) throw error(GHEXB_ERR_INVALID, "regular patterns support 1 to 3 dimensions");
    if (n < 1) throw error(GHEXB_ERR_INVALID, "a pattern needs at least one domain");
    p.kind = pattern_kind::regular;
    p.dim = dim;
    p.domains.assign(n, domain_info{});
    for (int i = 0; i < n; ++i)
    {
        auto& d = p.domains[i];
        d.id = ids[i];
        for (int k = 0; k < dim; ++k)
        {
            d.first[k] = first[i * dim + k];
            d.last[k] = last[i * dim + k];
            if (d.last[k] < d.first[k])
                throw error(GHEXB_ERR_INVALID, "domain " + std::to_string(d.id) + " is empty");
        }
        for (int j = 0; j < i; ++j)
            if (p.domains[j].id == d.id)
                throw error(GHEXB_ERR_INVALID, "repeated domain id " + std::to_string(d.id));
    }
    for (int k = 0; k < 2 * dim; ++k)
        if (halos[k] < 0) throw error(GHEXB_ERR_INVALID, "halo widths must be non-negative");
}
} // namespace

void build_regular(ghexb_pattern_s& p, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n, const int64_t* ids, const int* first,
    const int* last)
{
    set_domains(p, dim, halos, n, ids, first, last);

    const int centre = (dim == 1 ? 3 : dim == 2 ? 9 : 27) / 2;

    // receive spaces, keyed by source domain id (std::map ordering of the reference)
    std::vector<std::map<int64_t, std::vector<space_pair>>> recv(n);
    for (int i = 0; i < n; ++i)
    {
        const auto& dom = p.domains[i];
        box2 iv[3];
        for (int k = 0; k < dim; ++k)
        {
            const int ext = dom.last[k] - dom.first[k];
            iv[0].lfirst[k] = -halos[2 * k];
            iv[0].llast[k] = -1;
            iv[0].gfirst[k] = iv[0].lfirst[k] + dom.first[k];
            iv[0].glast[k] = dom.first[k] - 1;
            iv[1].lfirst[k] = 0;
            iv[1].llast[k] = ext;
            iv[1].gfirst[k] = dom.first[k];
            iv[1].glast[k] = dom.last[k];
            iv[2].lfirst[k] = ext + 1;
            iv[2].llast[k] = ext + halos[2 * k + 1];
            iv[2].gfirst[k] = dom.last[k] + 1;
            iv[2].glast[k] = dom.last[k] + halos[2 * k + 1];
        }
        std::vector<box2> all, boxes;
        box2 cur;
        combine(0, dim, iv, cur, all);
        for (int j = 0; j < (int)all.size(); ++j)
        {
            if (j == centre) continue;
            if (all_le(all[j].lfirst, all[j].llast, dim)) boxes.push_back(all[j]);
        }
        for (auto& b : boxes)
            for (int k = 0; k < dim; ++k)
            {
                if (!periodic[k]) continue;
                const int ext_h = b.glast[k] - b.gfirst[k];
                const int ext = g_last[k] + 1 - g_first[k];
                const int off = b.gfirst[k] - g_first[k];
                b.gfirst[k] = (off + ext) % ext + g_first[k];
                b.glast[k] = b.gfirst[k] + ext_h;
            }
        for (const auto& b : boxes)
            for (int e = 0; e < n; ++e)
            {
                const auto& other = p.domains[e];
                space_pair s;
                for (int k = 0; k < dim; ++k)
                {
                    s.gfirst[k] = std::max(b.gfirst[k], other.first[k]);
                    s.glast[k] = std::min(b.glast[k], other.last[k]);
                    s.lfirst[k] = b.lfirst[k] + (s.gfirst[k] - b.gfirst[k]);
                    s.llast[k] = b.lfirst[k] + (s.glast[k] - b.gfirst[k]);
                }
                if (all_le(s.gfirst, s.glast, dim)) recv[i][other.id].push_back(s);
            }
    }

    // receive entries in map order, tags from a running counter (single process: one rank)
    int tag_counter = -1;
    p.max_tag = 0;
    for (int i = 0; i < n; ++i)
    {
        for (auto& kv : recv[i])
        {
            struct_entry e;
            e.neighbor = p.find_domain(kv.first);
            e.tag = ++tag_counter;
            p.max_tag = std::max(p.max_tag, e.tag);
            e.spaces = std::move(kv.second);
            p.domains[i].recv.push_back(std::move(e));
        }
    }

    // send spaces: receiver's spaces with local coordinates in the sender's frame, keyed by
    // (receiver id, tag)
    std::vector<std::map<std::pair<int64_t, int>, struct_entry>> send(n);
    for (int i = 0; i < n; ++i)
        for (const auto& e : p.domains[i].recv)
        {
            const auto& src = p.domains[e.neighbor];
            auto& s = send[e.neighbor][{p.domains[i].id, e.tag}];
            s.neighbor = i;
            s.tag = e.tag;
            for (auto sp : e.spaces)
            {
                for (int k = 0; k < dim; ++k)
                {
                    sp.lfirst[k] = sp.gfirst[k] - src.first[k];
                    sp.llast[k] = sp.glast[k] - src.first[k];
                }
                s.spaces.push_back(sp);
            }
        }
    for (int i = 0; i < n; ++i)
        for (auto& kv : send[i]) p.domains[i].send.push_back(std::move(kv.second));
}

void build_regular_staged(ghexb_pattern_s* const* stages, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n, const int64_t* ids, const int* first, const int* last,
    const int64_t* neighbor_ids)
{
    for (int i = 0; i < dim; ++i) set_domains(*stages[i], dim, halos, n, ids, first, last);
    const auto& doms = stages[0]->domains;
    if (dim < 1 || dim > 3) throw error(GHEXB_ERR_INVALID, "regular patterns support 1 to 3 dimensions");

    // per stage and domain: receive and send spaces keyed by neighbour id, in insertion order
    using space_map = std::map<int64_t, std::vector<space_pair>>;
    std::vector<std::vector<space_map>> recv(dim, std::vector<space_map>(n)), send(dim, std::vector<space_map>(n));
    for (int d = 0; d < n; ++d)
    {
        // the domain's box, grown by the halos of the dimensions already exchanged
        space_pair box;
        for (int k = 0; k < dim; ++k)
        {
            box.lfirst[k] = 0;
            box.llast[k] = doms[d].last[k] - doms[d].first[k];
            box.gfirst[k] = doms[d].first[k];
            box.glast[k] = doms[d].last[k];
        }
        for (int i = 0; i < dim; ++i)
        {
            const int hm = halos[2 * i], hp = halos[2 * i + 1];
            const bool has_left = hm > 0 && (periodic[i] || box.gfirst[i] - hm >= g_first[i]);
            const bool has_right = hp > 0 && (periodic[i] || box.glast[i] + hp <= g_last[i]);
            auto neighbor = [&](int side) {
                const int64_t id = neighbor_ids[((int64_t)d * dim + i) * 2 + side];
                if (stages[i]->find_domain(id) < 0)
                    throw error(GHEXB_ERR_INVALID, "staged pattern: the domain lookup of domain " +
                                                       std::to_string(doms[d].id) + " names unknown domain " +
                                                       std::to_string(id));
                return id;
            };
            // the four spaces in the reference's order: receive left, send right, receive right,
            // send left (a neighbour on both sides pairs the k-th receive with its k-th send)
            auto shifted = [&](int lo, int hi) {
                space_pair s = box;
                const int l0 = box.lfirst[i], g0 = box.gfirst[i];
                s.lfirst[i] = lo, s.llast[i] = hi;
                s.gfirst[i] = g0 + (lo - l0), s.glast[i] = g0 + (hi - l0);
                return s;
            };
            const int lf = box.lfirst[i], ll = box.llast[i];
            if (has_left) recv[i][d][neighbor(0)].push_back(shifted(lf - hm, lf - 1));
            if (has_right) send[i][d][neighbor(1)].push_back(shifted(ll + 1 - hm, ll));
            if (has_right) recv[i][d][neighbor(1)].push_back(shifted(ll + 1, ll + hp));
            if (has_left) send[i][d][neighbor(0)].push_back(shifted(lf, lf - 1 + hp));
            if (has_left) box.lfirst[i] -= hm, box.gfirst[i] -= hm;
            if (has_right) box.llast[i] += hp, box.glast[i] += hp;
        }
    }

    for (int i = 0; i < dim; ++i)
    {
        auto& P = *stages[i];
        // tags: a running counter over the receive entries of the stage (one process)
        int tag_counter = -1;
        P.max_tag = 0;
        for (int d = 0; d < n; ++d)
            for (auto& kv : recv[i][d])
            {
                struct_entry e;
                e.neighbor = P.find_domain(kv.first);
                e.tag = ++tag_counter;
                P.max_tag = std::max(P.max_tag, e.tag);
                e.spaces = kv.second;
                P.domains[d].recv.push_back(std::move(e));
            }
        // send entries take the tag of the receive entry they feed; the k-th receive space is
        // filled from the k-th non-empty send space of the neighbour's entry (a side with a zero
        // halo width sends an empty space, which carries nothing)
        for (int d = 0; d < n; ++d)
            for (auto& kv : send[i][d])
            {
                const int r = P.find_domain(kv.first);
                struct_entry* re = nullptr;
                for (auto& e : P.domains[r].recv)
                    if (e.neighbor == d) re = &e;
                std::vector<const space_pair*> full;
                for (const auto& sp : kv.second)
                    if (all_le(sp.lfirst, sp.llast, dim)) full.push_back(&sp);
                if ((!re && !full.empty()) || (re && re->spaces.size() != full.size()))
                    throw error(GHEXB_ERR_INVALID, "staged pattern: the spaces domain " + std::to_string(doms[d].id) +
                                                       " sends to domain " + std::to_string(kv.first) +
                                                       " do not match what that domain receives from it");
                struct_entry e;
                e.neighbor = r;
                e.tag = re ? re->tag : 0;
                e.spaces = kv.second;
                for (size_t k = 0; k < full.size(); ++k)
                {
                    auto& rs = re->spaces[k];
                    for (int a = 0; a < dim; ++a)
                        if (rs.llast[a] - rs.lfirst[a] != full[k]->llast[a] - full[k]->lfirst[a])
                            throw error(GHEXB_ERR_INVALID, "staged pattern: a receive space of domain " +
                                                               std::to_string(kv.first) + " and the send space of domain " +
                                                               std::to_string(doms[d].id) + " feeding it differ in shape");
                    rs.has_src = true;
                    rs.sfirst = full[k]->lfirst;
                }
                P.domains[d].send.push_back(std::move(e));
            }
        for (int d = 0; d < n; ++d)
            for (const auto& e : P.domains[d].recv)
                for (const auto& sp : e.spaces)
                    if (!sp.has_src)
                        throw error(GHEXB_ERR_INVALID, "staged pattern: domain " + std::to_string(doms[d].id) +
                                                           " receives from domain " +
                                                           std::to_string(doms[e.neighbor].id) + ", which sends nothing to it");
    }
}

} // namespace ghexb

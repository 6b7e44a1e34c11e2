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

void build_regular(ghexb_pattern_s& p, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n, const int64_t* ids, const int* first,
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

} // namespace ghexb

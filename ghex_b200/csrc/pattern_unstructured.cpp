// Unstructured patterns.
//
// Behaviour follows GHEX 0.4.0:
//  * unstructured::domain_descriptor (unstructured/user_concepts.hpp:37-175): gids in storage
//    order, outer (halo) local ids given explicitly, inner gids unique;
//  * domain_descriptor::make_outer_lids (:88-113): halo gids that are not outer are skipped, a gid
//    repeated in the halo takes the next of its local ids, and every outer lid of a listed gid
//    must be used. Repeated gids are assigned their local ids in ascending order (the reference
//    takes std::unordered_multimap::equal_range order); all local ids of one gid receive the value
//    of the same owner, so the exchanged values do not depend on this choice;
//  * halo_generator (:180-256): all outer gids, or an explicit gid list;
//  * make_pattern_impl<unstructured grid>::apply without receive-domain hints
//    (unstructured/pattern.hpp:187-370): for every domain and every neighbour domain, the
//    neighbour's halo gids that are inner to the domain become the send list (in the neighbour's
//    halo order) and, mapped through the neighbour's make_outer_lids, its receive list. Tags are
//    (sender index << num_bits(#domains)) | receiver id; maps are ordered by (rank, tag);
//  * make_pattern_impl<unstructured grid>::apply with a receive domain ids generator
//    (unstructured/pattern.hpp:371-588): the generator names, for every halo element in the halo
//    generator's order, its owner domain and its local index there; receive lists group the halo
//    elements by owner (ascending owner id), the owner's send list holds the named local indices in
//    the receiver's order, tags are (owner id << 7) + receiver id and the maximum tag is
//    (max id << 7) + max id. Unlike the reference, a named index must be an inner element of the
//    owner (a halo element would be read while it is being written).
#include <algorithm>
#include <map>
#include <unordered_map>
#include <unordered_set>

#include "core.hpp"

namespace ghexb
{
namespace
{
struct udomain
{
    int64_t id;
    std::vector<int64_t> gids;
    std::unordered_map<int64_t, int64_t> inner;             // gid -> lid
    std::unordered_map<int64_t, std::vector<int64_t>> outer; // gid -> lids (ascending)
    std::vector<int64_t> outer_gids;                         // in lid order

    std::vector<int64_t> make_outer_lids(const std::vector<int64_t>& halo) const
    {
        std::vector<int64_t> lids;
        lids.reserve(halo.size());
        std::unordered_map<int64_t, size_t> used;
        for (auto gid : halo)
        {
            auto it = outer.find(gid);
            if (it == outer.end()) continue;
            size_t& k = used[gid];
            if (k >= it->second.size())
                throw error(GHEXB_ERR_INVALID, "halo gid does not have an associated lid in the domain");
            lids.push_back(it->second[k]);
            ++k;
        }
        for (const auto& kv : used)
            if (kv.second != outer.at(kv.first).size())
                throw error(GHEXB_ERR_INVALID, "halo gid occurs not often enough");
        return lids;
    }
};

unsigned num_bits(unsigned n) { return n ? 1u + num_bits(n >> 1) : 1u; }
} // namespace

void build_unstructured(ghexb_pattern_s& p, int n, const int64_t* ids, const int64_t* gid_off,
    const int64_t* gids, const int64_t* outer_off, const int64_t* outer_lids,
    const int64_t* halo_off, const int64_t* halo_gids, const int64_t* hint_off, const int64_t* hint_ids,
    const int64_t* hint_remote)
{
    if (n < 1) throw error(GHEXB_ERR_INVALID, "a pattern needs at least one domain");
    p.kind = pattern_kind::unstructured;
    p.dim = 1;
    std::vector<udomain> dom(n);
    p.domains.assign(n, domain_info{});
    int64_t max_id = ids[0];
    for (int i = 0; i < n; ++i)
    {
        auto& d = dom[i];
        d.id = ids[i];
        if (d.id < 0) throw error(GHEXB_ERR_INVALID, "unstructured domain ids must be non-negative");
        max_id = std::max(max_id, d.id);
        for (int j = 0; j < i; ++j)
            if (dom[j].id == d.id) throw error(GHEXB_ERR_INVALID, "repeated domain id " + std::to_string(d.id));
        const int64_t g0 = gid_off[i], g1 = gid_off[i + 1];
        if (g1 < g0) throw error(GHEXB_ERR_INVALID, "gid offsets must be non-decreasing");
        d.gids.assign(gids + g0, gids + g1);
        std::unordered_set<int64_t> outer_set;
        for (int64_t k = outer_off[i]; k < outer_off[i + 1]; ++k)
        {
            const int64_t lid = outer_lids[k];
            if (lid < 0 || lid >= (int64_t)d.gids.size())
                throw error(GHEXB_ERR_INVALID, "outer local index out of range");
            if (!outer_set.insert(lid).second) throw error(GHEXB_ERR_INVALID, "repeated outer (local) index");
        }
        for (int64_t lid = 0; lid < (int64_t)d.gids.size(); ++lid)
        {
            const int64_t gid = d.gids[lid];
            if (outer_set.count(lid))
            {
                d.outer[gid].push_back(lid);
                d.outer_gids.push_back(gid);
            }
            else if (!d.inner.emplace(gid, lid).second)
                throw error(GHEXB_ERR_INVALID, "repeated inner (global) index");
        }
        p.domains[i].id = d.id;
        p.domains[i].size = (int64_t)d.gids.size();
        p.domains[i].outer.assign(outer_lids + outer_off[i], outer_lids + outer_off[i + 1]);
        std::sort(p.domains[i].outer.begin(), p.domains[i].outer.end());
    }
    if (max_id > (int64_t)0x7fffffff) throw error(GHEXB_ERR_INVALID, "domain ids must fit into int");

    // halos of every domain: local ids and their gids
    std::vector<std::vector<int64_t>> halo_gid_lists(n), halo_lid_lists(n);
    for (int i = 0; i < n; ++i)
    {
        std::vector<int64_t> lids;
        if (halo_off) lids = dom[i].make_outer_lids(std::vector<int64_t>(halo_gids + halo_off[i], halo_gids + halo_off[i + 1]));
        else
            lids = dom[i].make_outer_lids(dom[i].outer_gids);
        for (auto lid : lids) halo_gid_lists[i].push_back(dom[i].gids[lid]);
        halo_lid_lists[i] = std::move(lids);
    }

    if (hint_off)
    {
        auto hint_tag = [](int64_t sender, int64_t receiver) {
            return (int)(((uint32_t)sender << 7) + (uint32_t)receiver);
        };
        p.max_tag = hint_tag(max_id, max_id);
        std::vector<std::map<int64_t, list_entry>> recv(n), send(n); // keyed by neighbour id
        for (int i = 0; i < n; ++i)
        {
            const auto& lids = halo_lid_lists[i];
            if (hint_off[i + 1] - hint_off[i] != (int64_t)lids.size())
                throw error(GHEXB_ERR_INVALID, "the receive domain ids generator gives " +
                                                   std::to_string(hint_off[i + 1] - hint_off[i]) + " entries for the " +
                                                   std::to_string(lids.size()) + " halo elements of domain " +
                                                   std::to_string(dom[i].id));
            for (size_t k = 0; k < lids.size(); ++k)
            {
                const int64_t owner = hint_ids[hint_off[i] + (int64_t)k];
                const int64_t rem = hint_remote[hint_off[i] + (int64_t)k];
                const int o = p.find_domain(owner);
                if (o < 0)
                    throw error(GHEXB_ERR_INVALID, "the receive domain ids generator names unknown domain " +
                                                       std::to_string(owner));
                if (rem < 0 || rem >= (int64_t)dom[o].gids.size() ||
                    std::binary_search(p.domains[o].outer.begin(), p.domains[o].outer.end(), rem))
                    throw error(GHEXB_ERR_INVALID, "the receive domain ids generator names local index " +
                                                       std::to_string(rem) + " of domain " + std::to_string(owner) +
                                                       ", which is not an inner element");
                auto& r = recv[i][owner];
                r.neighbor = o;
                r.tag = hint_tag(owner, dom[i].id);
                r.lids.push_back(lids[k]);
                auto& sd = send[o][dom[i].id];
                sd.neighbor = i;
                sd.tag = r.tag;
                sd.lids.push_back(rem);
            }
        }
        for (int i = 0; i < n; ++i)
        {
            for (auto& kv : send[i]) p.domains[i].usend.push_back(std::move(kv.second));
            for (auto& kv : recv[i]) p.domains[i].urecv.push_back(std::move(kv.second));
        }
        return;
    }

    const unsigned shift = num_bits((unsigned)n);
    auto make_tag = [shift](unsigned src_index, int64_t tgt_id) { return (int)((src_index << shift) | (unsigned)tgt_id); };
    p.max_tag = make_tag((unsigned)n, max_id);

    // send lists (sender d, receiver o) and receive lists, keyed by tag
    std::vector<std::map<int, list_entry>> send(n), recv(n);
    for (int o = 0; o < n; ++o)         // neighbour whose halo is filled
        for (int i = 0; i < n; ++i)     // candidate owner
        {
            const int tag = make_tag((unsigned)i, dom[o].id);
            list_entry s;
            std::vector<int64_t> gid_list;
            for (auto gid : halo_gid_lists[o])
            {
                auto it = dom[i].inner.find(gid);
                if (it == dom[i].inner.end()) continue;
                s.lids.push_back(it->second);
                gid_list.push_back(gid);
            }
            if (s.lids.empty()) continue;
            s.neighbor = o;
            s.tag = tag;
            list_entry r;
            r.neighbor = i;
            r.tag = tag;
            r.lids = dom[o].make_outer_lids(gid_list);
            if (r.lids.size() != s.lids.size())
                throw error(GHEXB_ERR_INTERNAL, "receive and send lists differ in length");
            send[i].emplace(tag, std::move(s));
            recv[o].emplace(tag, std::move(r));
        }
    for (int i = 0; i < n; ++i)
    {
        for (auto& kv : send[i]) p.domains[i].usend.push_back(std::move(kv.second));
        for (auto& kv : recv[i]) p.domains[i].urecv.push_back(std::move(kv.second));
    }
}

} // namespace ghexb

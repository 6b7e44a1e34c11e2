// Cubed-sphere patterns.
//
// Behaviour follows GHEX 0.4.0:
//  * tile neighbour table and the affine tile-to-neighbour transforms
//    (structured/cubed_sphere/transform.hpp:41-128). These are data of the cube's coordinate
//    system: the values must equal the reference's for the exchanged halos to agree, so the
//    tables below hold the same numbers;
//  * cubed_sphere::halo_generator::operator() (structured/cubed_sphere/halo_generator.hpp:75-196):
//    four halo strips (bottom and top include the corners), each intersected with the domain's
//    own tile and with the four neighbour tiles, transformed into the neighbour's coordinates;
//  * halo_generator::intersect with the inverse transform (:225-284) and the generic structured
//    make_pattern (structured/pattern.hpp:214-568) for the receive map, tags and send spaces.
// Cube-corner diagonal regions intersect no tile and are never received.
#include <algorithm>
#include <map>
#include <tuple>

#include "core.hpp"

namespace ghexb
{
namespace
{
// neighbour tiles of each tile, order -x, +x, -y, +y
const int k_tile_nb[6][4] = {
    {4, 1, 5, 2}, {0, 3, 5, 2}, {0, 3, 1, 4}, {2, 5, 1, 4}, {2, 5, 3, 0}, {4, 1, 3, 0}};

// even tiles (0, 2, 4) share one set of four transforms, odd tiles (1, 3, 5) another
const cs_transform k_even[4] = {
    {{0, -1, 1, 0}, {1, 1}, {-1, 0}},
    {{1, 0, 0, 1}, {-1, 0}, {0, 0}},
    {{1, 0, 0, 1}, {0, 1}, {0, 0}},
    {{0, 1, -1, 0}, {-1, 1}, {0, -1}},
};
const cs_transform k_odd[4] = {
    {{1, 0, 0, 1}, {1, 0}, {0, 0}},
    {{0, -1, 1, 0}, {1, -1}, {-1, 0}},
    {{0, 1, -1, 0}, {1, 1}, {0, -1}},
    {{1, 0, 0, 1}, {0, -1}, {0, 0}},
};
const cs_transform k_identity = {{1, 0, 0, 1}, {0, 0}, {0, 0}};

// the inverse of tile t's transform towards neighbour n is the neighbour's transform back
// towards t: (neighbour tile, its direction index)
const int k_inv_src[6][4][2] = {
    {{4, 3}, {1, 0}, {5, 3}, {2, 0}},
    {{0, 1}, {3, 2}, {5, 1}, {2, 2}},
    {{0, 3}, {3, 0}, {1, 3}, {4, 0}},
    {{2, 1}, {5, 2}, {1, 1}, {4, 2}},
    {{2, 3}, {5, 0}, {3, 3}, {0, 0}},
    {{4, 1}, {1, 2}, {3, 1}, {0, 2}},
};

struct box
{
    coord4 f{}, l{};
};
struct box2
{
    box loc, glob;
};

box isect(const box& a, const box& b)
{
    box r;
    for (int i = 0; i < 4; ++i)
    {
        r.f[i] = std::max(a.f[i], b.f[i]);
        r.l[i] = std::min(a.l[i], b.l[i]);
    }
    return r;
}
box2 isect2(const box2& a, const box& b)
{
    box2 r;
    r.glob = isect(a.glob, b);
    for (int i = 0; i < 4; ++i)
    {
        r.loc.f[i] = a.loc.f[i] + (r.glob.f[i] - a.glob.f[i]);
        r.loc.l[i] = a.loc.l[i] + (r.glob.l[i] - a.glob.l[i]);
    }
    return r;
}
bool le4(const coord4& a, const coord4& b)
{
    for (int i = 0; i < 4; ++i)
        if (a[i] > b[i]) return false;
    return true;
}

// halo boxes of one domain (tile, x, y, z coordinates)
std::vector<box2> halo_boxes(const domain_info& d, int c, const int* h)
{
    const int t = d.tile;
    const box dom{d.first, d.last};
    const box dom_loc{{0, 0, 0, 0}, {0, d.last[1] - d.first[1], d.last[2] - d.first[2],
                                        d.last[3] - d.first[3]}};
    const box tile_box{{t, 0, 0, d.first[3]}, {t, c - 1, c - 1, d.last[3]}};
    box nb[4] = {tile_box, tile_box, tile_box, tile_box};
    nb[0].f[1] -= c, nb[0].l[1] -= c;
    nb[1].f[1] += c, nb[1].l[1] += c;
    nb[2].f[2] -= c, nb[2].l[2] -= c;
    nb[3].f[2] += c, nb[3].l[2] += c;

    auto mk = [&](const box& g) {
        box2 b;
        b.glob = g;
        for (int i = 0; i < 4; ++i)
        {
            b.loc.f[i] = dom_loc.f[i] + (g.f[i] - dom.f[i]);
            b.loc.l[i] = dom_loc.l[i] + (g.l[i] - dom.l[i]);
        }
        return b;
    };
    std::vector<box2> regions;
    {
        box g = dom; // bottom strip, with both corners
        g.f[1] -= h[0];
        g.f[2] -= h[2];
        g.l[1] = dom.l[1] + h[1];
        g.l[2] = dom.f[2] - 1;
        regions.push_back(mk(g));
    }
    {
        box g = dom; // left strip
        g.f[1] -= h[0];
        g.l[1] = dom.f[1] - 1;
        regions.push_back(mk(g));
    }
    {
        box g = dom; // right strip
        g.f[1] = dom.l[1] + 1;
        g.l[1] = dom.l[1] + h[1];
        regions.push_back(mk(g));
    }
    {
        box g = dom; // top strip, with both corners
        g.f[1] -= h[0];
        g.f[2] = dom.l[2] + 1;
        g.l[1] = dom.l[1] + h[1];
        g.l[2] = dom.l[2] + h[3];
        regions.push_back(mk(g));
    }

    std::vector<box2> out;
    for (const auto& r : regions)
    {
        const box2 own = isect2(r, tile_box);
        if (own.glob.f[1] <= own.glob.l[1] && own.glob.f[2] <= own.glob.l[2]) out.push_back(own);
        for (int n = 0; n < 4; ++n)
        {
            box2 hn = isect2(r, nb[n]);
            if (!(hn.glob.f[1] <= hn.glob.l[1] && hn.glob.f[2] <= hn.glob.l[2])) continue;
            const cs_transform& tr = cs_forward(t, n);
            const auto f = tr.apply(hn.glob.f[1], hn.glob.f[2], c);
            const auto l = tr.apply(hn.glob.l[1], hn.glob.l[2], c);
            hn.glob.f[0] = hn.glob.l[0] = k_tile_nb[t][n];
            if (tr.reversed_x()) hn.glob.f[1] = l[0], hn.glob.l[1] = f[0];
            else
                hn.glob.f[1] = f[0], hn.glob.l[1] = l[0];
            if (tr.reversed_y()) hn.glob.f[2] = l[1], hn.glob.l[2] = f[1];
            else
                hn.glob.f[2] = f[1], hn.glob.l[2] = l[1];
            out.push_back(hn);
        }
    }
    return out;
}

// Intersection of halo box a (of domain d) with domain b's global box, in d's local frame.
// Returns false when the two lie on different tiles or do not overlap.
bool intersect_domain(const domain_info& d, const box2& a, const domain_info& b, int c,
    space_pair& out)
{
    const int tile = a.glob.f[0];
    if (tile != b.first[0]) return false;
    const box bg{b.first, b.last};
    if (tile != d.tile)
    {
        const box x = isect(a.glob, bg);
        if (!le4(x.f, x.l)) return false;
        int n = 0;
        while (n < 4 && cs_neighbor_tile(d.tile, n) != tile) ++n;
        if (n == 4) return false;
        const cs_transform& t = cs_inverse(d.tile, n);
        auto f = t.apply(x.f[1], x.f[2], c);
        auto l = t.apply(x.l[1], x.l[2], c);
        f[0] -= d.first[1];
        f[1] -= d.first[2];
        l[0] -= d.first[1];
        l[1] -= d.first[2];
        coord4 lf = a.loc.f, ll = a.loc.l;
        lf[3] += x.f[3] - a.glob.f[3];
        ll[3] += x.l[3] - a.glob.l[3];
        if (t.reversed_x()) lf[1] = l[0], ll[1] = f[0];
        else
            lf[1] = f[0], ll[1] = l[0];
        if (t.reversed_y()) lf[2] = l[1], ll[2] = f[1];
        else
            lf[2] = f[1], ll[2] = l[1];
        out.lfirst = lf;
        out.llast = ll;
        out.gfirst = x.f;
        out.glast = x.l;
        return true;
    }
    const box2 r = isect2(a, bg);
    if (!le4(r.glob.f, r.glob.l)) return false;
    out.lfirst = r.loc.f;
    out.llast = r.loc.l;
    out.gfirst = r.glob.f;
    out.glast = r.glob.l;
    return true;
}
} // namespace

int cs_neighbor_tile(int tile, int n) { return k_tile_nb[tile][n]; }
const cs_transform& cs_forward(int tile, int n) { return (tile % 2 == 0) ? k_even[n] : k_odd[n]; }
const cs_transform& cs_inverse(int tile, int n)
{
    return cs_forward(k_inv_src[tile][n][0], k_inv_src[tile][n][1]);
}
const cs_transform& cs_identity() { return k_identity; }

void build_cubed_sphere(ghexb_pattern_s& p, int edge, int levels, const int* halos, int n,
    const int* tiles, const int* x_first, const int* x_last, const int* y_first,
    const int* y_last)
{
    if (edge < 1 || levels < 1) throw error(GHEXB_ERR_INVALID, "cube edge size and levels must be positive");
    if (n < 1) throw error(GHEXB_ERR_INVALID, "a pattern needs at least one domain");
    for (int k = 0; k < 4; ++k)
        if (halos[k] < 0) throw error(GHEXB_ERR_INVALID, "halo widths must be non-negative");
    p.kind = pattern_kind::cubed_sphere;
    p.dim = 4;
    p.edge_size = edge;
    p.levels = levels;
    p.domains.assign(n, domain_info{});
    for (int i = 0; i < n; ++i)
    {
        auto& d = p.domains[i];
        if (tiles[i] < 0 || tiles[i] > 5) throw error(GHEXB_ERR_INVALID, "tile ids are 0..5");
        if (x_first[i] < 0 || x_last[i] >= edge || y_first[i] < 0 || y_last[i] >= edge ||
            x_last[i] < x_first[i] || y_last[i] < y_first[i])
            throw error(GHEXB_ERR_INVALID, "domain " + std::to_string(i) + " is not inside its tile");
        d.id = i;
        d.tile = tiles[i];
        d.first = {tiles[i], x_first[i], y_first[i], 0};
        d.last = {tiles[i], x_last[i], y_last[i], levels - 1};
        for (int j = 0; j < i; ++j)
            if (p.domains[j].first == d.first)
                throw error(GHEXB_ERR_INVALID, "repeated cubed-sphere domain id");
    }
    // receive map key: domain_id_type ordering (tile, then y_first, then x_first)
    auto key = [&](int i) {
        const auto& d = p.domains[i];
        return std::make_tuple(d.first[0], d.first[2], d.first[1]);
    };
    std::vector<std::map<std::tuple<int, int, int>, std::pair<int, std::vector<space_pair>>>> recv(n);
    for (int i = 0; i < n; ++i)
    {
        const auto& d = p.domains[i];
        for (const auto& h : halo_boxes(d, edge, halos))
        {
            if (!le4(h.loc.f, h.loc.l)) continue;
            for (int e = 0; e < n; ++e)
            {
                space_pair s;
                if (intersect_domain(d, h, p.domains[e], edge, s))
                {
                    auto& slot = recv[i][key(e)];
                    slot.first = e;
                    slot.second.push_back(s);
                }
            }
        }
    }
    int tag_counter = -1;
    p.max_tag = 0;
    for (int i = 0; i < n; ++i)
        for (auto& kv : recv[i])
        {
            struct_entry e;
            e.neighbor = kv.second.first;
            e.tag = ++tag_counter;
            p.max_tag = std::max(p.max_tag, e.tag);
            e.spaces = std::move(kv.second.second);
            p.domains[i].recv.push_back(std::move(e));
        }
    // send spaces keyed by (receiver key, tag)
    std::vector<std::map<std::tuple<int, int, int, int>, struct_entry>> send(n);
    for (int i = 0; i < n; ++i)
        for (const auto& e : p.domains[i].recv)
        {
            const auto& src = p.domains[e.neighbor];
            const auto ki = key(i);
            auto& s = send[e.neighbor][std::make_tuple(std::get<0>(ki), std::get<1>(ki), std::get<2>(ki), e.tag)];
            s.neighbor = i;
            s.tag = e.tag;
            for (auto sp : e.spaces)
            {
                for (int k = 0; k < 4; ++k)
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

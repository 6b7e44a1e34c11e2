// C entry points that run GHEX 0.4.0's own CPU exchange — test infrastructure, built into
// oracle/_ref/libghex_ref.so by oracle/ref/build.py from the reference's headers and
// src/context.cpp, with the stand-ins of oracle/ref/shim for its absent dependencies (MPI, oomph,
// gridtools, hwmalloc). One process holds every domain; messages go through the loopback
// transport (one copy per message, as an MPI self-send).
//
// Used as the oracle for golden outputs and as the timed CPU baseline of the reference.
#include <ghex/config.hpp>
#include <ghex/context.hpp>
#include <ghex/communication_object.hpp>
#include <ghex/structured/cubed_sphere/field_descriptor.hpp>
#include <ghex/structured/cubed_sphere/halo_generator.hpp>
#include <ghex/structured/pattern.hpp>
#include <ghex/structured/regular/domain_descriptor.hpp>
#include <ghex/structured/regular/field_descriptor.hpp>
#include <ghex/structured/regular/halo_generator.hpp>
#include <ghex/structured/regular/make_pattern.hpp>
#include <ghex/unstructured/communication_object_ipr.hpp>
#include <ghex/unstructured/pattern.hpp>
#include <ghex/unstructured/user_concepts.hpp>

#include <algorithm>
#include <chrono>
#include <memory>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace
{
thread_local std::string g_err;

int fail(const std::string& m)
{
    g_err = m;
    return 1;
}

enum dtype_code
{
    F32 = 0,
    F64 = 1,
    I32 = 2,
    I64 = 3
};

// runs `exchange` once untimed and then `iters` times timed; returns seconds per exchange
template<typename F>
double timed(int iters, F&& exchange)
{
    exchange();
    if (iters <= 0) return 0.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < iters; ++i) exchange();
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count() / iters;
}

// Exchanges all buffer_info vectors of a tuple of vectors in one call of the communication object.
template<typename CO, typename V0>
void exchange_all(CO& co, V0& v0)
{
    if (!v0.empty()) co.exchange(v0.begin(), v0.end()).wait();
}
template<typename CO, typename V0, typename V1>
void exchange_all(CO& co, V0& v0, V1& v1)
{
    if (v0.empty()) return exchange_all(co, v1);
    if (v1.empty()) return exchange_all(co, v0);
    co.exchange(v0.begin(), v0.end(), v1.begin(), v1.end()).wait();
}

// ---- regular -------------------------------------------------------------------------------
template<int D>
int regular(const int* g_first, const int* g_last, int n_dom, const int* ids, const int* firsts, const int* lasts,
    int n_groups, const int* halos, const int* periodic, int n_fields, const int* field_group, const int* dtype,
    void** data, const int* offsets, const int* extents, int iters, double* seconds)
{
    using dom_t = ghex::structured::regular::domain_descriptor<int, std::integral_constant<int, D>>;
    using hg_t = ghex::structured::regular::halo_generator<int, std::integral_constant<int, D>>;
    using layout = std::conditional_t<D == 3, gridtools::layout_map<2, 1, 0>,
        std::conditional_t<D == 2, gridtools::layout_map<1, 0>, gridtools::layout_map<0>>>;
    using arr = std::array<int, D>;
    ghex::context ctxt(MPI_COMM_WORLD, true);
    std::vector<dom_t> doms;
    for (int i = 0; i < n_dom; ++i)
    {
        arr f, l;
        for (int k = 0; k < D; ++k) f[k] = firsts[i * D + k], l[k] = lasts[i * D + k];
        doms.emplace_back(ids[i], f, l);
    }
    arr gf, gl;
    for (int k = 0; k < D; ++k) gf[k] = g_first[k], gl[k] = g_last[k];
    using pattern_t = decltype(ghex::make_pattern<ghex::structured::grid>(
        ctxt, std::declval<hg_t&>(), doms));
    std::vector<pattern_t> pats;
    pats.reserve(n_groups);
    for (int g = 0; g < n_groups; ++g)
    {
        std::array<int, 2 * D> h;
        std::array<bool, D> p;
        for (int k = 0; k < 2 * D; ++k) h[k] = halos[g * 2 * D + k];
        for (int k = 0; k < D; ++k) p[k] = periodic[g * D + k] != 0;
        hg_t hg(gf, gl, h, p);
        pats.push_back(ghex::make_pattern<ghex::structured::grid>(ctxt, hg, doms));
    }
    using fd_d = ghex::structured::regular::field_descriptor<double, ghex::cpu, dom_t, layout>;
    using fd_f = ghex::structured::regular::field_descriptor<float, ghex::cpu, dom_t, layout>;
    using fd_i = ghex::structured::regular::field_descriptor<int32_t, ghex::cpu, dom_t, layout>;
    using fd_l = ghex::structured::regular::field_descriptor<int64_t, ghex::cpu, dom_t, layout>;
    std::vector<fd_d> fdd;
    std::vector<fd_f> fdf;
    std::vector<fd_i> fdi;
    std::vector<fd_l> fdl;
    fdd.reserve(n_fields * n_dom), fdf.reserve(n_fields * n_dom), fdi.reserve(n_fields * n_dom), fdl.reserve(n_fields * n_dom);
    std::vector<decltype(pats[0](std::declval<fd_d&>()))> bd;
    std::vector<decltype(pats[0](std::declval<fd_f&>()))> bf;
    std::vector<decltype(pats[0](std::declval<fd_i&>()))> bi;
    std::vector<decltype(pats[0](std::declval<fd_l&>()))> bl;
    for (int fi = 0; fi < n_fields; ++fi)
        for (int d = 0; d < n_dom; ++d)
        {
            arr off, ext;
            for (int k = 0; k < D; ++k) off[k] = offsets[fi * D + k], ext[k] = extents[(fi * n_dom + d) * D + k];
            void* p = data[fi * n_dom + d];
            auto& pat = pats[field_group[fi]];
            switch (dtype[fi])
            {
                case F64:
                    fdd.push_back(ghex::wrap_field<ghex::cpu, layout>(doms[d], (double*)p, off, ext));
                    bd.push_back(pat(fdd.back()));
                    break;
                case F32:
                    fdf.push_back(ghex::wrap_field<ghex::cpu, layout>(doms[d], (float*)p, off, ext));
                    bf.push_back(pat(fdf.back()));
                    break;
                case I32:
                    fdi.push_back(ghex::wrap_field<ghex::cpu, layout>(doms[d], (int32_t*)p, off, ext));
                    bi.push_back(pat(fdi.back()));
                    break;
                default:
                    fdl.push_back(ghex::wrap_field<ghex::cpu, layout>(doms[d], (int64_t*)p, off, ext));
                    bl.push_back(pat(fdl.back()));
                    break;
            }
        }
    if (!bi.empty() || !bl.empty())
    {
        if (!bd.empty() || !bf.empty()) return fail("integer fields cannot be mixed with float fields here");
        auto co = ghex::make_communication_object<pattern_t>(ctxt);
        *seconds = timed(iters, [&] { exchange_all(co, bi, bl); });
        return 0;
    }
    auto co = ghex::make_communication_object<pattern_t>(ctxt);
    *seconds = timed(iters, [&] { exchange_all(co, bd, bf); });
    return 0;
}

// ---- staged regular pattern ----------------------------------------------------------------
// make_staged_pattern with a domain lookup read from a table: nbr[(d*D + i)*2 + s] is the
// neighbour of domain d along dimension i at offset -1 (s = 0) or +1 (s = 1).
template<int D>
struct table_lookup
{
    struct neighbor
    {
        int m_id;
        int rank() const noexcept { return 0; }
        int id() const noexcept { return m_id; }
    };
    std::vector<int> ids;
    const int64_t* nbr;
    neighbor operator()(int id, std::array<int, D> const& offset) const
    {
        const int d = (int)(std::find(ids.begin(), ids.end(), id) - ids.begin());
        for (int i = 0; i < D; ++i)
            if (offset[i] != 0) return {(int)nbr[((int64_t)d * D + i) * 2 + (offset[i] > 0 ? 1 : 0)]};
        return {id};
    }
};

// One field (one dtype) exchanged stage after stage with one communication object, as GHEX's
// test_simple_regular_domain does.
template<int D, typename T>
int regular_staged(const int* g_first, const int* g_last, int n_dom, const int* ids, const int* firsts,
    const int* lasts, const int* halos, const int* periodic, const int64_t* nbr, void** data, const int* offsets,
    const int* extents, int iters, double* seconds)
{
    using dom_t = ghex::structured::regular::domain_descriptor<int, std::integral_constant<int, D>>;
    using layout = std::conditional_t<D == 3, gridtools::layout_map<2, 1, 0>,
        std::conditional_t<D == 2, gridtools::layout_map<1, 0>, gridtools::layout_map<0>>>;
    using arr = std::array<int, D>;
    ghex::context ctxt(MPI_COMM_WORLD, true);
    std::vector<dom_t> doms;
    for (int i = 0; i < n_dom; ++i)
    {
        arr f, l;
        for (int k = 0; k < D; ++k) f[k] = firsts[i * D + k], l[k] = lasts[i * D + k];
        doms.emplace_back(ids[i], f, l);
    }
    arr gf, gl;
    std::array<int, 2 * D> h;
    std::array<bool, D> p;
    for (int k = 0; k < D; ++k) gf[k] = g_first[k], gl[k] = g_last[k], p[k] = periodic[k] != 0;
    for (int k = 0; k < 2 * D; ++k) h[k] = halos[k];
    table_lookup<D> lu{std::vector<int>(ids, ids + n_dom), nbr};
    auto stages = ghex::structured::regular::make_staged_pattern(ctxt, doms, lu, gf, gl, h, p);
    using fd_t = ghex::structured::regular::field_descriptor<T, ghex::cpu, dom_t, layout>;
    std::vector<fd_t> fds;
    fds.reserve(n_dom);
    for (int d = 0; d < n_dom; ++d)
    {
        arr off, ext;
        for (int k = 0; k < D; ++k) off[k] = offsets[k], ext[k] = extents[d * D + k];
        fds.push_back(ghex::wrap_field<ghex::cpu, layout>(doms[d], (T*)data[d], off, ext));
    }
    using pattern_t = std::remove_reference_t<decltype(*stages[0])>;
    using bi_t = decltype((*stages[0])(fds[0]));
    auto co = ghex::make_communication_object<pattern_t>(ctxt);
    *seconds = timed(iters, [&] {
        for (int i = 0; i < D; ++i)
        {
            std::vector<bi_t> bis;
            for (auto& f : fds) bis.push_back((*stages[i])(f));
            co.exchange(bis.begin(), bis.end()).wait();
        }
    });
    return 0;
}

template<int D>
int regular_staged_dispatch(int dtype, const int* g_first, const int* g_last, int n_dom, const int* ids,
    const int* firsts, const int* lasts, const int* halos, const int* periodic, const int64_t* nbr, void** data,
    const int* offsets, const int* extents, int iters, double* seconds)
{
    switch (dtype)
    {
        case F64:
            return regular_staged<D, double>(g_first, g_last, n_dom, ids, firsts, lasts, halos, periodic, nbr, data,
                offsets, extents, iters, seconds);
        case F32:
            return regular_staged<D, float>(g_first, g_last, n_dom, ids, firsts, lasts, halos, periodic, nbr, data,
                offsets, extents, iters, seconds);
        case I32:
            return regular_staged<D, int32_t>(g_first, g_last, n_dom, ids, firsts, lasts, halos, periodic, nbr, data,
                offsets, extents, iters, seconds);
        default:
            return regular_staged<D, int64_t>(g_first, g_last, n_dom, ids, firsts, lasts, halos, periodic, nbr, data,
                offsets, extents, iters, seconds);
    }
}

// ---- cubed sphere -------------------------------------------------------------------------
template<typename T>
int cubed(int edge, int levels, const int* halos, int n_dom, const int* tiles, const int* xf, const int* xl,
    const int* yf, const int* yl, int n_fields, const int* ncomp, const int* is_vector, void** data,
    const int* offsets, const int* extents, int iters, double* seconds)
{
    using namespace ghex::structured::cubed_sphere;
    ghex::context ctxt(MPI_COMM_WORLD, true);
    cube c{edge, levels};
    std::vector<domain_descriptor> doms;
    for (int i = 0; i < n_dom; ++i) doms.emplace_back(c, tiles[i], xf[i], xl[i], yf[i], yl[i]);
    halo_generator hg(std::array<int, 4>{halos[0], halos[1], halos[2], halos[3]});
    auto pat = ghex::make_pattern<ghex::structured::grid>(ctxt, hg, doms);
    using fd_t = field_descriptor<T, ghex::cpu>;
    std::vector<fd_t> fds;
    fds.reserve(n_fields * n_dom);
    std::vector<decltype(pat(std::declval<fd_t&>()))> bis;
    for (int fi = 0; fi < n_fields; ++fi)
        for (int d = 0; d < n_dom; ++d)
        {
            std::array<int, 3> off{offsets[fi * 3], offsets[fi * 3 + 1], offsets[fi * 3 + 2]};
            const int* e = extents + (fi * n_dom + d) * 3;
            std::array<int, 3> ext{e[0], e[1], e[2]};
            fds.emplace_back(doms[d], (T*)data[fi * n_dom + d], off, ext, (unsigned)ncomp[fi], is_vector[fi] != 0);
            bis.push_back(pat(fds.back()));
        }
    auto co = ghex::make_communication_object<decltype(pat)>(ctxt);
    *seconds = timed(iters, [&] { co.exchange(bis.begin(), bis.end()).wait(); });
    return 0;
}

// ---- unstructured --------------------------------------------------------------------------
int unstructured(int n_dom, const int* ids, const int64_t* gid_off, const int* gids, const int64_t* outer_off,
    const int64_t* outer_lids, int n_fields, const int* dtype, const int* levels, const int* levels_first,
    void** data, int iters, double* seconds)
{
    using dom_t = ghex::unstructured::domain_descriptor<int, int>;
    using hg_t = ghex::unstructured::halo_generator<int, int>;
    ghex::context ctxt(MPI_COMM_WORLD, true);
    std::vector<dom_t> doms;
    for (int i = 0; i < n_dom; ++i)
    {
        std::vector<int> g(gids + gid_off[i], gids + gid_off[i + 1]);
        std::vector<std::size_t> o(outer_lids + outer_off[i], outer_lids + outer_off[i + 1]);
        doms.emplace_back(ids[i], g.begin(), g.end(), o.begin(), o.end());
    }
    hg_t hg;
    auto pat = ghex::make_pattern<ghex::unstructured::grid>(ctxt, hg, doms);
    using dd_d = ghex::unstructured::data_descriptor<ghex::cpu, int, int, double>;
    using dd_f = ghex::unstructured::data_descriptor<ghex::cpu, int, int, float>;
    std::vector<dd_d> fdd;
    std::vector<dd_f> fdf;
    fdd.reserve(n_fields * n_dom), fdf.reserve(n_fields * n_dom);
    std::vector<decltype(pat(std::declval<dd_d&>()))> bd;
    std::vector<decltype(pat(std::declval<dd_f&>()))> bf;
    for (int fi = 0; fi < n_fields; ++fi)
        for (int d = 0; d < n_dom; ++d)
        {
            void* p = data[fi * n_dom + d];
            if (dtype[fi] == F64)
            {
                fdd.emplace_back(doms[d], (double*)p, (std::size_t)levels[fi], levels_first[fi] != 0);
                bd.push_back(pat(fdd.back()));
            }
            else
            {
                fdf.emplace_back(doms[d], (float*)p, (std::size_t)levels[fi], levels_first[fi] != 0);
                bf.push_back(pat(fdf.back()));
            }
        }
    auto co = ghex::make_communication_object<decltype(pat)>(ctxt);
    *seconds = timed(iters, [&] { exchange_all(co, bd, bf); });
    return 0;
}
// make_pattern(ctx, halo_gen, recv_domain_ids_gen, domains) (unstructured/pattern.hpp:371-588):
// the receive domain ids generator is read from tables, one (owner id, remote index) per halo
// element of every domain in the halo generator's order; the halo generator takes the gid list.
template<typename T>
int unstructured_hinted(int n_dom, const int* ids, const int64_t* gid_off, const int* gids, const int64_t* outer_off,
    const int64_t* outer_lids, const int* halo_gids, int n_halo_gids, const int64_t* hint_off, const int* hint_ids,
    const int* hint_remote, int levels, void** data, int iters, double* seconds)
{
    using dom_t = ghex::unstructured::domain_descriptor<int, int>;
    using hg_t = ghex::unstructured::halo_generator<int, int>;
    struct hints
    {
        struct halo
        {
            std::vector<int> m_ids, m_ranks;
            std::vector<int> m_remote;
            const std::vector<int>& domain_ids() const noexcept { return m_ids; }
            const std::vector<int>& remote_indices() const noexcept { return m_remote; }
            const std::vector<int>& ranks() const noexcept { return m_ranks; }
        };
        std::vector<int> ids;
        const int64_t* off;
        const int* hid;
        const int* hrem;
        halo operator()(const dom_t& d) const
        {
            const int k = (int)(std::find(ids.begin(), ids.end(), d.domain_id()) - ids.begin());
            halo h;
            h.m_ids.assign(hid + off[k], hid + off[k + 1]);
            h.m_remote.assign(hrem + off[k], hrem + off[k + 1]);
            h.m_ranks.assign(h.m_ids.size(), 0);
            return h;
        }
    };
    ghex::context ctxt(MPI_COMM_WORLD, true);
    std::vector<dom_t> doms;
    for (int i = 0; i < n_dom; ++i)
    {
        std::vector<int> g(gids + gid_off[i], gids + gid_off[i + 1]);
        std::vector<std::size_t> o(outer_lids + outer_off[i], outer_lids + outer_off[i + 1]);
        doms.emplace_back(ids[i], g.begin(), g.end(), o.begin(), o.end());
    }
    hg_t hg = n_halo_gids < 0 ? hg_t{} : hg_t{std::vector<int>(halo_gids, halo_gids + n_halo_gids)};
    hints rdig{std::vector<int>(ids, ids + n_dom), hint_off, hint_ids, hint_remote};
    auto pat = ghex::make_pattern<ghex::unstructured::grid>(ctxt, hg, rdig, doms);
    using dd_t = ghex::unstructured::data_descriptor<ghex::cpu, int, int, T>;
    std::vector<dd_t> dds;
    dds.reserve(n_dom);
    for (int d = 0; d < n_dom; ++d) dds.emplace_back(doms[d], (T*)data[d], (std::size_t)levels, true);
    std::vector<decltype(pat(dds[0]))> bis;
    for (auto& dd : dds) bis.push_back(pat(dd));
    auto co = ghex::make_communication_object<decltype(pat)>(ctxt);
    *seconds = timed(iters, [&] { co.exchange(bis.begin(), bis.end()).wait(); });
    return 0;
}

// One in-place receive communication object per domain (communication_object_ipr.hpp), as in
// GHEX's test_in_place_receive: every object posts its receives into the field's halo and sends
// its packed values, then every handle is waited on.
template<typename T>
int unstructured_ipr(int n_dom, const int* ids, const int64_t* gid_off, const int* gids, const int64_t* outer_off,
    const int64_t* outer_lids, const int* halo_gids, int n_halo_gids, int levels, void** data, int iters,
    double* seconds)
{
    using dom_t = ghex::unstructured::domain_descriptor<int, int>;
    using hg_t = ghex::unstructured::halo_generator<int, int>;
    ghex::context ctxt(MPI_COMM_WORLD, true);
    std::vector<dom_t> doms;
    for (int i = 0; i < n_dom; ++i)
    {
        std::vector<int> g(gids + gid_off[i], gids + gid_off[i + 1]);
        std::vector<std::size_t> o(outer_lids + outer_off[i], outer_lids + outer_off[i + 1]);
        doms.emplace_back(ids[i], g.begin(), g.end(), o.begin(), o.end());
    }
    hg_t hg = n_halo_gids < 0 ? hg_t{} : hg_t{std::vector<int>(halo_gids, halo_gids + n_halo_gids)};
    auto pat = ghex::make_pattern<ghex::unstructured::grid>(ctxt, hg, doms);
    using dd_t = ghex::unstructured::data_descriptor<ghex::cpu, int, int, T>;
    std::vector<dd_t> dds;
    dds.reserve(n_dom);
    for (int d = 0; d < n_dom; ++d) dds.emplace_back(doms[d], (T*)data[d], (std::size_t)levels, true);
    using co_t = decltype(ghex::unstructured::make_communication_object_ipr(ctxt, pat(dds[0])));
    std::vector<std::unique_ptr<co_t>> cos;
    for (int d = 0; d < n_dom; ++d) cos.emplace_back(new co_t(ctxt, pat(dds[d])));
    *seconds = timed(iters, [&] {
        std::vector<typename co_t::handle> hs;
        for (auto& co : cos) hs.push_back(co->exchange());
        for (auto& h : hs) h.wait();
    });
    return 0;
}
} // namespace

extern "C" {

int ghexref_last_error(char* buf, size_t len)
{
    std::snprintf(buf, len, "%s", g_err.c_str());
    return 0;
}

int ghexref_regular_staged_exchange(int dim, const int* g_first, const int* g_last, int n_dom, const int* ids,
    const int* firsts, const int* lasts, const int* halos, const int* periodic, const int64_t* neighbor_ids,
    int dtype, void** data, const int* offsets, const int* extents, int iters, double* seconds)
{
    try
    {
        switch (dim)
        {
            case 2:
                return regular_staged_dispatch<2>(dtype, g_first, g_last, n_dom, ids, firsts, lasts, halos, periodic,
                    neighbor_ids, data, offsets, extents, iters, seconds);
            case 3:
                return regular_staged_dispatch<3>(dtype, g_first, g_last, n_dom, ids, firsts, lasts, halos, periodic,
                    neighbor_ids, data, offsets, extents, iters, seconds);
            default: return fail("dim must be 2 or 3");
        }
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

int ghexref_regular_exchange(int dim, const int* g_first, const int* g_last, int n_dom, const int* ids,
    const int* firsts, const int* lasts, int n_groups, const int* halos, const int* periodic, int n_fields,
    const int* field_group, const int* dtype, void** data, const int* offsets, const int* extents, int iters,
    double* seconds)
{
    try
    {
        switch (dim)
        {
            case 2:
                return regular<2>(g_first, g_last, n_dom, ids, firsts, lasts, n_groups, halos, periodic, n_fields,
                    field_group, dtype, data, offsets, extents, iters, seconds);
            case 3:
                return regular<3>(g_first, g_last, n_dom, ids, firsts, lasts, n_groups, halos, periodic, n_fields,
                    field_group, dtype, data, offsets, extents, iters, seconds);
            default: return fail("dim must be 2 or 3");
        }
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

int ghexref_cubed_exchange(int dtype, int edge, int levels, const int* halos, int n_dom, const int* tiles,
    const int* xf, const int* xl, const int* yf, const int* yl, int n_fields, const int* ncomp, const int* is_vector,
    void** data, const int* offsets, const int* extents, int iters, double* seconds)
{
    try
    {
        if (dtype == F64)
            return cubed<double>(edge, levels, halos, n_dom, tiles, xf, xl, yf, yl, n_fields, ncomp, is_vector, data,
                offsets, extents, iters, seconds);
        return cubed<float>(edge, levels, halos, n_dom, tiles, xf, xl, yf, yl, n_fields, ncomp, is_vector, data,
            offsets, extents, iters, seconds);
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

int ghexref_unstructured_exchange(int n_dom, const int* ids, const int64_t* gid_off, const int* gids,
    const int64_t* outer_off, const int64_t* outer_lids, int n_fields, const int* dtype, const int* levels,
    const int* levels_first, void** data, int iters, double* seconds)
{
    try
    {
        return unstructured(n_dom, ids, gid_off, gids, outer_off, outer_lids, n_fields, dtype, levels, levels_first,
            data, iters, seconds);
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// hint_off[k] .. hint_off[k+1]: domain k's (owner id, remote index) per halo element
int ghexref_unstructured_exchange_hinted(int n_dom, const int* ids, const int64_t* gid_off, const int* gids,
    const int64_t* outer_off, const int64_t* outer_lids, const int* halo_gids, int n_halo_gids,
    const int64_t* hint_off, const int* hint_ids, const int* hint_remote, int dtype, int levels, void** data,
    int iters, double* seconds)
{
    try
    {
        if (dtype == F64)
            return unstructured_hinted<double>(n_dom, ids, gid_off, gids, outer_off, outer_lids, halo_gids,
                n_halo_gids, hint_off, hint_ids, hint_remote, levels, data, iters, seconds);
        if (dtype == I32)
            return unstructured_hinted<int>(n_dom, ids, gid_off, gids, outer_off, outer_lids, halo_gids,
                n_halo_gids, hint_off, hint_ids, hint_remote, levels, data, iters, seconds);
        return fail("dtype must be f64 or i32");
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// halo_gids: the gid list of the halo generator, or n_halo_gids < 0 for all outer gids
int ghexref_unstructured_exchange_ipr(int n_dom, const int* ids, const int64_t* gid_off, const int* gids,
    const int64_t* outer_off, const int64_t* outer_lids, const int* halo_gids, int n_halo_gids, int dtype, int levels,
    void** data, int iters, double* seconds)
{
    try
    {
        switch (dtype)
        {
            case F64:
                return unstructured_ipr<double>(n_dom, ids, gid_off, gids, outer_off, outer_lids, halo_gids,
                    n_halo_gids, levels, data, iters, seconds);
            case F32:
                return unstructured_ipr<float>(n_dom, ids, gid_off, gids, outer_off, outer_lids, halo_gids,
                    n_halo_gids, levels, data, iters, seconds);
            case I32:
                return unstructured_ipr<int>(n_dom, ids, gid_off, gids, outer_off, outer_lids, halo_gids,
                    n_halo_gids, levels, data, iters, seconds);
            default: return fail("dtype must be f32, f64 or i32");
        }
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

} // extern "C"

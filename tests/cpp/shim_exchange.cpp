// Exchange through the C++ front end (include/ghex_b200.hpp), written as GHEX's own regular-grid
// tests are: 64^3 cells split 2x2x2 into domains of 32^3, halo 1 on every side, periodic in x, y
// and z, float64, x fastest. Every halo cell must equal the interior value of its periodic owner,
// which is known in closed form (value = global linear index + 0.5); the interior must stay as it
// was. Run once with device fields (ghexb::gpu) and once with fields in ordinary host memory
// (ghexb::cpu). Also checks GHEX's error behaviour: a second exchange before wait() and a field of
// a domain outside the pattern. Then unstructured column data (run_unstructured) the same two ways.
// Prints "shim: ok" and returns 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "ghex_b200.hpp"

namespace
{
constexpr int N = 64, P = 32, H = 1, E = P + 2 * H;
using dim3_t = std::integral_constant<int, 3>;
using domain = ghexb::structured::regular::domain_descriptor<int, dim3_t>;
using halo_gen = ghexb::structured::regular::halo_generator<int, dim3_t>;
using layout = ghexb::layout_map<2, 1, 0>; // x fastest

double owner_value(int gx, int gy, int gz)
{
    gx = (gx + N) % N, gy = (gy + N) % N, gz = (gz + N) % N;
    return (double)(gx + N * (gy + N * gz)) + 0.5;
}

std::vector<double> initial(const domain& d)
{
    std::vector<double> a((size_t)E * E * E, std::nan(""));
    for (int z = 0; z < P; ++z)
        for (int y = 0; y < P; ++y)
            for (int x = 0; x < P; ++x)
                a[(x + H) + E * ((y + H) + E * (z + H))] = owner_value(d.first()[0] + x, d.first()[1] + y, d.first()[2] + z);
    return a;
}

int check(const domain& d, const std::vector<double>& a)
{
    int bad = 0;
    for (int z = 0; z < E; ++z)
        for (int y = 0; y < E; ++y)
            for (int x = 0; x < E; ++x)
            {
                const double want = owner_value(d.first()[0] + x - H, d.first()[1] + y - H, d.first()[2] + z - H);
                const double got = a[x + E * (y + E * z)];
                if (std::memcmp(&want, &got, sizeof got)) ++bad;
            }
    return bad;
}

template<typename Arch>
int run(ghexb::context& ctxt, bool device)
{
    std::vector<domain> doms;
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 2; ++i)
                doms.push_back(domain(i + 2 * (j + 2 * k), {i * P, j * P, k * P}, {i * P + P - 1, j * P + P - 1, k * P + P - 1}));
    halo_gen hg({0, 0, 0}, {N - 1, N - 1, N - 1}, {H, H, H, H, H, H}, {true, true, true});
    auto pattern = ghexb::make_pattern<ghexb::structured::grid>(ctxt, hg, doms);
    auto co = ghexb::make_communication_object<decltype(pattern)>(ctxt);

    std::vector<std::vector<double>> host;
    std::vector<double*> data;
    for (const auto& d : doms)
    {
        host.push_back(initial(d));
        if (device)
        {
            double* p = nullptr;
            if (cudaMalloc(&p, host.back().size() * sizeof(double)) != cudaSuccess) return 100;
            cudaMemcpy(p, host.back().data(), host.back().size() * sizeof(double), cudaMemcpyHostToDevice);
            data.push_back(p);
        }
        else
            data.push_back(host.back().data());
    }
    std::vector<ghexb::buffer_info> bis;
    for (size_t i = 0; i < doms.size(); ++i)
        bis.push_back(pattern(ghexb::wrap_field<Arch, layout>(doms[i], data[i], {H, H, H}, {E, E, E})));

    auto h = co.exchange(bis.begin(), bis.end());
    int errors = 0;
    // a second exchange before wait(): "earlier exchange operation was not finished"
    try
    {
        auto h2 = co.exchange(bis[0], bis[1]);
        h2.wait();
        std::printf("shim: a second exchange before wait() was accepted\n");
        ++errors;
    }
    catch (const ghexb::error& e)
    {
        if (e.code() != GHEXB_ERR_BUSY) ++errors, std::printf("shim: busy error code %d\n", e.code());
    }
    h.wait();
    for (size_t i = 0; i < doms.size(); ++i)
    {
        if (device)
            cudaMemcpy(host[i].data(), data[i], host[i].size() * sizeof(double), cudaMemcpyDeviceToHost);
        const int bad = check(doms[i], host[i]);
        if (bad) std::printf("shim: domain %zu has %d wrong cells (%s fields)\n", i, bad, device ? "device" : "host");
        errors += bad;
    }
    // a field of a domain the pattern does not have
    try
    {
        domain stranger(99, {0, 0, 0}, {P - 1, P - 1, P - 1});
        auto bi = pattern(ghexb::wrap_field<Arch, layout>(stranger, data[0], {H, H, H}, {E, E, E}));
        std::printf("shim: a field of an unknown domain was accepted\n");
        ++errors;
    }
    catch (const ghexb::error& e)
    {
        if (e.code() != GHEXB_ERR_INCOMPATIBLE || !std::strstr(e.what(), "incompatible"))
            ++errors, std::printf("shim: unknown domain gave %d: %s\n", e.code(), e.what());
    }
    bis.clear();
    if (device)
        for (double* p : data) cudaFree(p);
    return errors;
}

// Unstructured column data as GHEX's unstructured tests write it: a ring of NV vertices in four
// domains of consecutive global ids, each storing its inner vertices and then its two neighbours
// (the outer, halo, elements), LV levels per vertex, levels first. After the exchange a halo
// column holds its owner's values (value = gid * 10 + level + 0.25).
constexpr int NV = 64, ND = 4, LV = 3;
using udomain = ghexb::unstructured::domain_descriptor<int, int>;
using uhalo_gen = ghexb::unstructured::halo_generator<int, int>;

double column_value(int gid, int lev) { return gid * 10.0 + lev + 0.25; }

template<typename Arch>
int run_unstructured(ghexb::context& ctxt, bool device)
{
    const int per = NV / ND;
    std::vector<udomain> doms;
    std::vector<std::vector<int>> gids(ND);
    for (int d = 0; d < ND; ++d)
    {
        for (int k = 0; k < per; ++k) gids[d].push_back(d * per + k);
        gids[d].push_back((d * per + NV - 1) % NV); // left neighbour
        gids[d].push_back(((d + 1) * per) % NV);    // right neighbour
        const std::vector<int> outer{per, per + 1};
        doms.emplace_back(d, gids[d].begin(), gids[d].end(), outer.begin(), outer.end());
    }
    auto pattern = ghexb::make_pattern<ghexb::unstructured::grid>(ctxt, uhalo_gen(), doms);
    auto co = ghexb::make_communication_object<decltype(pattern)>(ctxt);
    std::vector<std::vector<double>> host(ND);
    std::vector<double*> data;
    for (int d = 0; d < ND; ++d)
    {
        host[d].assign((size_t)(per + 2) * LV, std::nan(""));
        for (int k = 0; k < per; ++k)
            for (int l = 0; l < LV; ++l) host[d][(size_t)k * LV + l] = column_value(gids[d][k], l);
        if (device)
        {
            double* p = nullptr;
            if (cudaMalloc(&p, host[d].size() * sizeof(double)) != cudaSuccess) return 100;
            cudaMemcpy(p, host[d].data(), host[d].size() * sizeof(double), cudaMemcpyHostToDevice);
            data.push_back(p);
        }
        else
            data.push_back(host[d].data());
    }
    std::vector<ghexb::buffer_info> bis;
    for (int d = 0; d < ND; ++d)
        bis.push_back(pattern(ghexb::unstructured::data_descriptor<Arch, int, int, double>(doms[d], data[d], LV, true)));
    co.exchange(bis.begin(), bis.end()).wait();
    int errors = 0;
    for (int d = 0; d < ND; ++d)
    {
        if (device) cudaMemcpy(host[d].data(), data[d], host[d].size() * sizeof(double), cudaMemcpyDeviceToHost);
        for (int k = 0; k < per + 2; ++k)
            for (int l = 0; l < LV; ++l)
            {
                const double want = column_value(gids[d][k], l), got = host[d][(size_t)k * LV + l];
                if (std::memcmp(&want, &got, sizeof got)) ++errors;
            }
    }
    if (errors) std::printf("shim: %d wrong unstructured values (%s fields)\n", errors, device ? "device" : "host");
    bis.clear();
    if (device)
        for (double* p : data) cudaFree(p);
    return errors;
}
} // namespace

int main()
{
    try
    {
        ghexb::context ctxt(0);
        const int dev_errors = run<ghexb::gpu>(ctxt, true) + run_unstructured<ghexb::gpu>(ctxt, true);
        const int host_errors = run<ghexb::cpu>(ctxt, false) + run_unstructured<ghexb::cpu>(ctxt, false);
        if (dev_errors || host_errors)
        {
            std::printf("shim: %d device and %d host errors\n", dev_errors, host_errors);
            return 1;
        }
        std::printf("shim: ok\n");
        return 0;
    }
    catch (const std::exception& e)
    {
        std::printf("shim: exception %s\n", e.what());
        return 2;
    }
}

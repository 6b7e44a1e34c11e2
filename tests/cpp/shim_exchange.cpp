// Exchange through the C++ front end (include/ghex_b200.hpp), written as GHEX's own regular-grid
// tests are: 64^3 cells split 2x2x2 into domains of 32^3, halo 1 on every side, periodic in x, y
// and z, float64, x fastest. Every halo cell must equal the interior value of its periodic owner,
// which is known in closed form (value = global linear index + 0.5); the interior must stay as it
// was. Run once with device fields (ghexb::gpu) and once with fields in ordinary host memory
// (ghexb::cpu). Also checks GHEX's error behaviour: a second exchange before wait() and a field of
// a domain outside the pattern. Prints "shim: ok" and returns 0 when every check passes.
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
} // namespace

int main()
{
    try
    {
        ghexb::context ctxt(0);
        const int dev_errors = run<ghexb::gpu>(ctxt, true);
        const int host_errors = run<ghexb::cpu>(ctxt, false);
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

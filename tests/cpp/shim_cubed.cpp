// Cubed-sphere exchange through the C++ front end (include/ghex_b200.hpp), as GHEX's cubed-sphere
// test writes it: make_pattern<structured::grid> over cubed_sphere::domain_descriptor, a
// cubed_sphere::halo_generator and cubed_sphere::field_descriptor<float, Arch>.
//
//   shim_cubed <input> <output> <gpu|cpu> <is_vector 0|1>
//
// The input file holds int32 edge, levels, halo, memory halo, domain edge, components and domain
// count, then per domain int32 (tile, x_first, x_last, y_first, y_last), then per domain its field
// as float32 (x, y, z, component), x fastest. The output file receives the fields after one
// exchange, in the same order. Prints "shim_cubed: ok" and returns 0 when the exchange ran.
#include <cstdio>
#include <vector>

#include <cuda_runtime.h>

#include "ghex_b200.hpp"

namespace cs = ghexb::structured::cubed_sphere;

template<typename Arch>
int run(const char* in_path, const char* out_path, bool device, bool is_vector)
{
    std::FILE* in = std::fopen(in_path, "rb");
    if (!in) return 10;
    int head[7];
    if (std::fread(head, sizeof(int), 7, in) != 7) return 11;
    const int edge = head[0], levels = head[1], halo = head[2], mem = head[3], n = head[4], ncomp = head[5], nd = head[6];
    const int ext = n + 2 * mem;
    const size_t count = (size_t)ext * ext * levels * ncomp;
    std::vector<std::array<int, 5>> boxes(nd);
    for (auto& b : boxes)
        if (std::fread(b.data(), sizeof(int), 5, in) != 5) return 12;
    std::vector<std::vector<float>> host(nd, std::vector<float>(count));
    for (auto& h : host)
        if (std::fread(h.data(), sizeof(float), count, in) != count) return 13;
    std::fclose(in);

    ghexb::context ctxt(0);
    const cs::cube c{edge, levels};
    std::vector<cs::domain_descriptor> doms;
    for (const auto& b : boxes) doms.emplace_back(c, b[0], b[1], b[2], b[3], b[4]);
    auto pattern = ghexb::make_pattern<ghexb::structured::grid>(ctxt, cs::halo_generator(halo), doms);
    auto co = ghexb::make_communication_object<decltype(pattern)>(ctxt);
    std::vector<float*> data;
    for (auto& h : host)
    {
        if (device)
        {
            float* p = nullptr;
            if (cudaMalloc(&p, count * sizeof(float)) != cudaSuccess) return 14;
            cudaMemcpy(p, h.data(), count * sizeof(float), cudaMemcpyHostToDevice);
            data.push_back(p);
        }
        else
            data.push_back(h.data());
    }
    std::vector<ghexb::buffer_info> bis;
    for (int d = 0; d < nd; ++d)
        bis.push_back(pattern(cs::field_descriptor<float, Arch>(doms[d], data[d], {mem, mem, 0}, {ext, ext, levels},
            (unsigned)ncomp, is_vector)));
    co.exchange(bis.begin(), bis.end()).wait();
    bis.clear();
    std::FILE* out = std::fopen(out_path, "wb");
    if (!out) return 15;
    for (int d = 0; d < nd; ++d)
    {
        if (device)
        {
            cudaMemcpy(host[d].data(), data[d], count * sizeof(float), cudaMemcpyDeviceToHost);
            cudaFree(data[d]);
        }
        std::fwrite(host[d].data(), sizeof(float), count, out);
    }
    std::fclose(out);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 5)
    {
        std::printf("usage: shim_cubed <input> <output> <gpu|cpu> <is_vector>\n");
        return 2;
    }
    try
    {
        const bool device = std::string(argv[3]) == "gpu", is_vector = std::string(argv[4]) == "1";
        const int rc = device ? run<ghexb::gpu>(argv[1], argv[2], true, is_vector) : run<ghexb::cpu>(argv[1], argv[2], false, is_vector);
        if (rc) std::printf("shim_cubed: failed (%d)\n", rc);
        else
            std::printf("shim_cubed: ok\n");
        return rc;
    }
    catch (const std::exception& e)
    {
        std::printf("shim_cubed: exception %s\n", e.what());
        return 3;
    }
}

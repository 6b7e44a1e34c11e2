// The known answers of GHEX's cubed-sphere exchange test, callable on any data — test
// infrastructure. The reference's test source (test/structured/cubed_sphere/
// test_cubed_sphere_exchange.cpp) is compiled as it is, against the gtest stand-in of
// oracle/ref/shim that counts failed expectations; its per-domain checking functions
// (check_even_0 .. check_odd_3 through check_field, :110-843) then run on a view of the caller's
// field memory. Its TEST_F bodies are compiled but never run.
#include <gtest/gtest.h>

#include <test/structured/cubed_sphere/test_cubed_sphere_exchange.cpp>

namespace
{
// The accessors check_field uses, over memory laid out x fastest, then y, z, component.
struct field_view
{
    using value_type = float;
    const float* m_data;
    ghex::structured::cubed_sphere::domain_id_type m_id;
    std::array<int, 4> m_offsets;
    std::array<int, 4> m_extents;
    std::array<int, 4> m_strides; // bytes
    int m_ncomp;
    bool m_vector;

    const float* data() const { return m_data; }
    const std::array<int, 4>& offsets() const { return m_offsets; }
    const std::array<int, 4>& extents() const { return m_extents; }
    const std::array<int, 4>& byte_strides() const { return m_strides; }
    int num_components() const { return m_ncomp; }
    bool is_vector_field() const { return m_vector; }
    const ghex::structured::cubed_sphere::domain_id_type& domain_id() const { return m_id; }
};
} // namespace

extern "C" int ghexref_cs_check_field(const float* data, int tile, int x_first, int y_first, int mem_halo, int n,
    int levels, int ncomp, int is_vector, int halo)
{
    const int ext = n + 2 * mem_halo;
    field_view f{data, ghex::structured::cubed_sphere::domain_id_type{tile, {x_first, y_first}},
        {mem_halo, mem_halo, 0, 0}, {ext, ext, levels, ncomp},
        {4, 4 * ext, 4 * ext * ext, 4 * ext * ext * levels}, ncomp, is_vector != 0};
    ghexref_failures() = 0;
    check_field(f, halo, n);
    return ghexref_failures();
}

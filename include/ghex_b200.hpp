/*
 * ghex_b200.hpp — C++ front end over the C ABI of ghex_b200.h, with the names and call shapes of
 * GHEX's own C++ interface for the regular structured grid, the cubed sphere and unstructured column
 * data, so
 * that GHEX code of the form
 *
 *     auto ctxt    = ghexb::context(device);
 *     auto pattern = ghexb::make_pattern<ghexb::structured::grid>(ctxt, halo_gen, local_domains);
 *     auto co      = ghexb::make_communication_object<decltype(pattern)>(ctxt);
 *     auto field   = ghexb::wrap_field<ghexb::gpu, ghexb::layout_map<2, 1, 0>>(dom, ptr, offsets, extents);
 *     co.exchange(pattern(field)).wait();
 *
 * runs on the B200 kernels. It replaces (paths relative to the GHEX 0.4.0 source tree):
 *   ghex::context                         context.hpp:20-35
 *   structured::regular::domain_descriptor structured/regular/domain_descriptor.hpp:248-254
 *   structured::regular::halo_generator    structured/regular/halo_generator.hpp:68-78
 *   make_pattern<structured::grid>         pattern_container.hpp:112-120
 *   pattern(field) -> buffer_info          pattern_container.hpp:88-95
 *   wrap_field<Arch, Layout>               structured/regular/field_descriptor.hpp:167-194
 *   make_communication_object<Pattern>     communication_object.hpp:653-660
 *   communication_object::exchange         communication_object.hpp:233-274
 *   communication_handle::wait/is_ready    communication_object.hpp:627-648
 *   unstructured::domain_descriptor        unstructured/user_concepts.hpp:37-174
 *   unstructured::halo_generator           unstructured/user_concepts.hpp:181-256
 *   unstructured::data_descriptor          unstructured/user_concepts.hpp:264-581
 *   make_pattern<unstructured::grid>       pattern_container.hpp:112-120, unstructured/pattern.hpp:187-370
 *   structured::cubed_sphere::cube, domain_descriptor, halo_generator, field_descriptor
 *                                          structured/cubed_sphere/domain_descriptor.hpp:26-104,
 *                                          halo_generator.hpp:59-71, field_descriptor.hpp:26-121
 *
 * Header only; link with libghex_b200.so. Every failing C call throws ghexb::error (a
 * std::runtime_error carrying the status code and the library's message), as GHEX throws
 * std::runtime_error. Differences from GHEX: one process owns every domain (the context takes a
 * CUDA device, not an MPI communicator); ghexb::cpu fields are exchanged by the GPU kernels in
 * place in host memory, which the field's buffer_info page-locks for as long as it lives.
 */
#ifndef GHEX_B200_HPP
#define GHEX_B200_HPP

#include <array>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_set>
#include <utility>
#include <vector>

#include "ghex_b200.h"

namespace ghexb
{
// ---- errors -------------------------------------------------------------------------------------
class error : public std::runtime_error
{
  public:
    error(int code, const std::string& what)
    : std::runtime_error(what)
    , m_code(code)
    {
    }
    int code() const noexcept { return m_code; }

  private:
    int m_code;
};

inline void check(int status)
{
    if (status != GHEXB_OK)
    {
        char msg[1024] = {0};
        ghexb_last_error(msg, sizeof msg);
        throw error(status, msg);
    }
}

// ---- architecture tags and layouts (ghex::cpu / ghex::gpu, gridtools::layout_map) ---------------
struct cpu
{
};
struct gpu
{
};

// gridtools convention: the dimension with the largest value has stride 1
template<int... L>
struct layout_map
{
    static constexpr int size = sizeof...(L);
    static std::array<int, sizeof...(L)> values() { return {{L...}}; }
};

namespace detail
{
template<typename T> struct dtype_of;
template<> struct dtype_of<float> : std::integral_constant<int, GHEXB_F32> {};
template<> struct dtype_of<double> : std::integral_constant<int, GHEXB_F64> {};
template<> struct dtype_of<std::int32_t> : std::integral_constant<int, GHEXB_I32> {};
template<> struct dtype_of<std::int64_t> : std::integral_constant<int, GHEXB_I64> {};
template<> struct dtype_of<std::uint8_t> : std::integral_constant<int, GHEXB_U8> {};
template<> struct dtype_of<std::uint16_t> : std::integral_constant<int, GHEXB_U16> {};

template<typename H, int (*Destroy)(H)>
struct handle_deleter
{
    void operator()(H h) const noexcept
    {
        if (h) Destroy(h);
    }
};
template<typename S, int (*Destroy)(S*)>
using owned = std::unique_ptr<S, handle_deleter<S*, Destroy>>;
} // namespace detail

// ---- context --------------------------------------------------------------------------------------
class context
{
  public:
    explicit context(int device = 0)
    {
        ghexb_context h = nullptr;
        check(ghexb_context_create(device, &h));
        m_h.reset(h);
    }
    ghexb_context get() const noexcept { return m_h.get(); }
    int rank() const noexcept { return 0; } // one process owns every domain
    int size() const noexcept { return 1; }

  private:
    detail::owned<ghexb_context_s, ghexb_context_destroy> m_h;
};

namespace structured
{
struct grid
{
};

namespace regular
{
// domain_descriptor<DomainId, Dimension>(id, first, last): inclusive global coordinates
template<typename DomainId, typename Dimension>
class domain_descriptor
{
  public:
    static constexpr int dim = Dimension::value;
    using domain_id_type = DomainId;
    using coordinate_type = std::array<int, dim>;

    domain_descriptor(DomainId id, const coordinate_type& first, const coordinate_type& last)
    : m_id(id)
    , m_first(first)
    , m_last(last)
    {
    }
    DomainId domain_id() const noexcept { return m_id; }
    const coordinate_type& first() const noexcept { return m_first; }
    const coordinate_type& last() const noexcept { return m_last; }

  private:
    DomainId m_id;
    coordinate_type m_first, m_last;
};

// halo_generator<DomainId, Dimension>(g_first, g_last, halos, periodic); halos holds 2*dim values
// (dim0-, dim0+, dim1-, ...)
template<typename DomainId, typename Dimension>
class halo_generator
{
  public:
    static constexpr int dim = Dimension::value;
    using coordinate_type = std::array<int, dim>;

    halo_generator(const coordinate_type& g_first, const coordinate_type& g_last, const std::array<int, 2 * dim>& halos,
        const std::array<bool, dim>& periodic)
    : m_first(g_first)
    , m_last(g_last)
    , m_halos(halos)
    , m_periodic(periodic)
    {
    }
    const coordinate_type& global_first() const noexcept { return m_first; }
    const coordinate_type& global_last() const noexcept { return m_last; }
    const std::array<int, 2 * dim>& halos() const noexcept { return m_halos; }
    const std::array<bool, dim>& periodic() const noexcept { return m_periodic; }

  private:
    coordinate_type m_first, m_last;
    std::array<int, 2 * dim> m_halos;
    std::array<bool, dim> m_periodic;
};

// field_descriptor<T, Arch, DomainDescriptor, Layout>: borrows the user's memory
template<typename T, typename Arch, typename DomainDescriptor, typename Layout>
class field_descriptor
{
  public:
    static constexpr int dim = DomainDescriptor::dim;
    using value_type = T;
    using arch_type = Arch;
    using domain_descriptor_type = DomainDescriptor;
    static_assert(Layout::size == dim, "the layout map must have one entry per dimension");

    field_descriptor(const DomainDescriptor& dom, T* data, const std::array<int, dim>& offsets,
        const std::array<int, dim>& extents, const std::vector<std::int64_t>& byte_strides = {})
    : m_dom(dom)
    , m_data(data)
    , m_offsets(offsets)
    , m_extents(extents)
    , m_byte_strides(byte_strides)
    {
        if (!byte_strides.empty() && (int)byte_strides.size() != dim)
            throw error(GHEXB_ERR_INVALID, "wrap_field: one byte stride per dimension");
    }
    const DomainDescriptor& domain() const noexcept { return m_dom; }
    typename DomainDescriptor::domain_id_type domain_id() const noexcept { return m_dom.domain_id(); }
    T* data() const noexcept { return m_data; }
    const std::array<int, dim>& offsets() const noexcept { return m_offsets; }
    const std::array<int, dim>& extents() const noexcept { return m_extents; }
    const std::vector<std::int64_t>& byte_strides() const noexcept { return m_byte_strides; }

    // bytes from data() to one past the last element
    std::size_t span_bytes() const
    {
        std::array<std::int64_t, dim> st{};
        if (!m_byte_strides.empty())
            for (int a = 0; a < dim; ++a) st[a] = m_byte_strides[a];
        else
        {
            // strides from the layout map: the largest value is contiguous
            const auto lm = Layout::values();
            std::int64_t s = sizeof(T);
            for (int v = dim - 1; v >= 0; --v)
                for (int a = 0; a < dim; ++a)
                    if (lm[a] == v) st[a] = s, s *= m_extents[a];
        }
        std::int64_t end = 0;
        for (int a = 0; a < dim; ++a) end += (std::int64_t)(m_extents[a] - 1) * st[a];
        return (std::size_t)end + sizeof(T);
    }

  private:
    DomainDescriptor m_dom;
    T* m_data;
    std::array<int, dim> m_offsets, m_extents;
    std::vector<std::int64_t> m_byte_strides;
};
} // namespace regular

namespace cubed_sphere
{
// cubed_sphere::cube{edge_size, levels}
struct cube
{
    int edge_size;
    int levels;
};

// cubed_sphere::domain_descriptor(cube, tile, x_first, x_last, y_first, y_last); its id is
// (tile, x_first, y_first)
class domain_descriptor
{
  public:
    struct domain_id_type
    {
        int tile, x, y;
        bool operator==(const domain_id_type& o) const noexcept { return tile == o.tile && x == o.x && y == o.y; }
    };
    domain_descriptor(const cube& c, int tile, int x_first, int x_last, int y_first, int y_last)
    : m_cube(c)
    , m_tile(tile)
    , m_x{x_first, x_last}
    , m_y{y_first, y_last}
    {
    }
    domain_id_type domain_id() const noexcept { return {m_tile, m_x[0], m_y[0]}; }
    int edge_size() const noexcept { return m_cube.edge_size; }
    int levels() const noexcept { return m_cube.levels; }
    int tile() const noexcept { return m_tile; }
    const std::array<int, 2>& x() const noexcept { return m_x; }
    const std::array<int, 2>& y() const noexcept { return m_y; }

  private:
    cube m_cube;
    int m_tile;
    std::array<int, 2> m_x, m_y;
};

// cubed_sphere::halo_generator(halo) or (halos: -x, +x, -y, +y)
class halo_generator
{
  public:
    explicit halo_generator(int halo) noexcept
    : m_halos{halo, halo, halo, halo}
    {
    }
    explicit halo_generator(const std::array<int, 4>& halos) noexcept
    : m_halos(halos)
    {
    }
    const std::array<int, 4>& halos() const noexcept { return m_halos; }

  private:
    std::array<int, 4> m_halos;
};

// cubed_sphere::field_descriptor<T, Arch, Layout>(dom, data, offsets, extents, num_components,
// is_vector_field) on (x, y, z, component), x fastest by default; a vector field's components
// 0 and 1 are negated where a tile edge's rotation turns them
template<typename T, typename Arch, typename Layout = layout_map<3, 2, 1, 0>>
class field_descriptor
{
  public:
    using value_type = T;
    using arch_type = Arch;
    field_descriptor(const domain_descriptor& dom, T* data, const std::array<int, 3>& offsets, const std::array<int, 3>& extents,
        unsigned num_components = 1u, bool is_vector_field = false)
    : m_dom(dom)
    , m_data(data)
    , m_offsets{offsets[0], offsets[1], offsets[2], 0}
    , m_extents{extents[0], extents[1], extents[2], (int)num_components}
    , m_is_vector(is_vector_field)
    {
    }
    const domain_descriptor& domain() const noexcept { return m_dom; }
    T* data() const noexcept { return m_data; }
    const std::array<int, 4>& offsets() const noexcept { return m_offsets; }
    const std::array<int, 4>& extents() const noexcept { return m_extents; }
    int num_components() const noexcept { return m_extents[3]; }
    bool is_vector_field() const noexcept { return m_is_vector; }
    std::size_t span_bytes() const noexcept
    {
        std::size_t n = sizeof(T);
        for (int e : m_extents) n *= (std::size_t)e;
        return n;
    }

  private:
    domain_descriptor m_dom;
    T* m_data;
    std::array<int, 4> m_offsets, m_extents;
    bool m_is_vector;
};
} // namespace cubed_sphere
} // namespace structured

namespace unstructured
{
struct grid
{
};

// unstructured::domain_descriptor<DomainId, Idx>(id, gids first, last, outer lids first, last):
// the domain's global ids in storage order and the local ids of its outer (halo) elements
template<typename DomainId, typename Idx>
class domain_descriptor
{
  public:
    using domain_id_type = DomainId;
    using global_index_type = Idx;
    using local_index_type = std::size_t;

    template<typename GidIt, typename LidIt>
    domain_descriptor(domain_id_type id, GidIt first, GidIt last, LidIt outer_first, LidIt outer_last)
    : m_id(id)
    , m_gids(first, last)
    {
        std::unordered_set<local_index_type> seen;
        for (auto it = outer_first; it != outer_last; ++it)
        {
            const local_index_type lid = (local_index_type)*it;
            if (!seen.insert(lid).second) throw std::runtime_error("repeated outer (local) index");
            if (lid >= m_gids.size()) throw std::runtime_error("outer local index out of range");
            m_outer.push_back(lid);
        }
    }

    domain_id_type domain_id() const noexcept { return m_id; }
    std::size_t size() const noexcept { return m_gids.size(); }
    std::size_t inner_size() const noexcept { return m_gids.size() - m_outer.size(); }
    const std::vector<global_index_type>& gids() const noexcept { return m_gids; }
    const std::vector<local_index_type>& outer_lids() const noexcept { return m_outer; }

  private:
    domain_id_type m_id;
    std::vector<global_index_type> m_gids;
    std::vector<local_index_type> m_outer;
};

// halo_generator(): every outer element is a halo element; halo_generator(gids): the halo of a
// domain is its outer elements with these global ids, in this order
template<typename DomainId, typename Idx>
class halo_generator
{
  public:
    halo_generator() = default;
    explicit halo_generator(std::vector<Idx> gids)
    : m_all(false)
    , m_gids(std::move(gids))
    {
    }
    bool all() const noexcept { return m_all; }
    const std::vector<Idx>& gids() const noexcept { return m_gids; }

  private:
    bool m_all = true;
    std::vector<Idx> m_gids;
};

// data_descriptor<Arch, DomainId, Idx, T>(domain, data, levels, levels_first, outer_stride): a
// column field of `levels` values per element; levels_first: the levels of an element are
// adjacent; outer_stride: elements between consecutive outer indices (0: no padding)
template<typename Arch, typename DomainId, typename Idx, typename T>
class data_descriptor
{
  public:
    using arch_type = Arch;
    using value_type = T;
    using domain_descriptor_type = domain_descriptor<DomainId, Idx>;

    data_descriptor(const domain_descriptor_type& domain, T* field, std::size_t levels = 1u, bool levels_first = true,
        std::size_t outer_stride = 0u)
    : m_domain_id(domain.domain_id())
    , m_size(domain.size())
    , m_levels(levels)
    , m_levels_first(levels_first)
    , m_outer_stride(outer_stride)
    , m_data(field)
    {
    }

    DomainId domain_id() const noexcept { return m_domain_id; }
    T* data() const noexcept { return m_data; }
    std::size_t levels() const noexcept { return m_levels; }
    bool levels_first() const noexcept { return m_levels_first; }
    std::size_t outer_stride() const noexcept { return m_outer_stride; }
    // bytes from the first element to one past the last one the field may address
    std::size_t span_bytes() const noexcept
    {
        const std::size_t index_stride = m_levels_first ? (m_outer_stride ? m_outer_stride : m_levels) : 1u;
        const std::size_t level_stride = m_levels_first ? 1u : (m_outer_stride ? m_outer_stride : m_size);
        return ((m_size - 1) * index_stride + (m_levels - 1) * level_stride + 1) * sizeof(T);
    }

  private:
    DomainId m_domain_id;
    std::size_t m_size, m_levels;
    bool m_levels_first;
    std::size_t m_outer_stride;
    T* m_data;
};
} // namespace unstructured

// wrap_field<Arch, Layout>(dom, data, offsets, extents[, byte_strides])
template<typename Arch, typename Layout, typename DomainDescriptor, typename T>
structured::regular::field_descriptor<T, Arch, DomainDescriptor, Layout> wrap_field(const DomainDescriptor& dom, T* data,
    const std::array<int, DomainDescriptor::dim>& offsets, const std::array<int, DomainDescriptor::dim>& extents,
    const std::vector<std::int64_t>& byte_strides = {})
{
    return {dom, data, offsets, extents, byte_strides};
}

// A field bound to a pattern (GHEX's buffer_info): owns the library's field handle, and for cpu
// fields the page-locking of their memory.
class buffer_info
{
  public:
    ghexb_field get() const noexcept { return m_state->field.get(); }

  private:
    struct state
    {
        detail::owned<ghexb_field_s, ghexb_field_destroy> field;
        void* registered = nullptr;
        ~state()
        {
            if (registered) ghexb_host_unregister(registered);
        }
    };
    std::shared_ptr<state> m_state = std::make_shared<state>();
    template<typename, typename> friend class pattern_container;
};

// The pattern of a set of domains (pattern_container<grid, domain_id>)
template<typename Grid, typename DomainDescriptor>
class pattern_container
{
  public:
    using domain_descriptor_type = DomainDescriptor;
    using grid_type = Grid;

    ghexb_pattern get() const noexcept { return m_h.get(); }
    int size() const
    {
        int n = 0;
        check(ghexb_pattern_num_domains(get(), &n));
        return n;
    }
    int max_tag() const
    {
        int t = 0;
        check(ghexb_pattern_max_tag(get(), &t));
        return t;
    }

    // pattern(field) -> buffer_info; throws "field incompatible with available domains!" for a
    // field of a domain that is not part of the pattern
    template<typename T, typename Arch, typename Layout>
    buffer_info operator()(const structured::regular::field_descriptor<T, Arch, DomainDescriptor, Layout>& f) const
    {
        constexpr int dim = DomainDescriptor::dim;
        const auto lm = Layout::values();
        buffer_info bi;
        if (std::is_same<Arch, cpu>::value)
        {
            int owned = 0;
            check(ghexb_host_register(f.data(), f.span_bytes(), &owned));
            if (owned) bi.m_state->registered = f.data();
        }
        ghexb_field h = nullptr;
        check(ghexb_field_wrap(get(), (std::int64_t)f.domain_id(), detail::dtype_of<T>::value, f.data(), dim,
            f.offsets().data(), f.extents().data(), lm.data(), f.byte_strides().empty() ? nullptr : f.byte_strides().data(),
            1, 0, &h));
        bi.m_state->field.reset(h);
        return bi;
    }

    // pattern(field_descriptor) -> buffer_info for cubed-sphere fields (addressed by the domain's
    // place in the pattern's list)
    template<typename T, typename Arch, typename Layout>
    buffer_info operator()(const structured::cubed_sphere::field_descriptor<T, Arch, Layout>& f) const
    {
        const auto id = f.domain().domain_id();
        int index = -1;
        for (size_t k = 0; k < m_cubed_ids.size() && index < 0; ++k)
            if (m_cubed_ids[k] == id) index = (int)k;
        if (index < 0) throw error(GHEXB_ERR_INCOMPATIBLE, "field incompatible with available domains!");
        const auto lm = Layout::values();
        buffer_info bi;
        if (std::is_same<Arch, cpu>::value)
        {
            int owned = 0;
            check(ghexb_host_register(f.data(), f.span_bytes(), &owned));
            if (owned) bi.m_state->registered = f.data();
        }
        ghexb_field h = nullptr;
        check(ghexb_field_wrap(get(), index, detail::dtype_of<T>::value, f.data(), 4, f.offsets().data(), f.extents().data(),
            lm.data(), nullptr, f.num_components(), f.is_vector_field() ? 1 : 0, &h));
        bi.m_state->field.reset(h);
        return bi;
    }

    // pattern(data_descriptor) -> buffer_info for unstructured column fields
    template<typename Arch, typename DomainId, typename Idx, typename T>
    buffer_info operator()(const unstructured::data_descriptor<Arch, DomainId, Idx, T>& f) const
    {
        buffer_info bi;
        if (std::is_same<Arch, cpu>::value)
        {
            int owned = 0;
            check(ghexb_host_register(f.data(), f.span_bytes(), &owned));
            if (owned) bi.m_state->registered = f.data();
        }
        ghexb_field h = nullptr;
        check(ghexb_field_wrap_unstructured(get(), (std::int64_t)f.domain_id(), detail::dtype_of<T>::value, f.data(),
            (std::int64_t)f.levels(), f.levels_first() ? 1 : 0, (std::int64_t)f.outer_stride(), &h));
        bi.m_state->field.reset(h);
        return bi;
    }

  private:
    std::shared_ptr<ghexb_pattern_s> m_h;
    std::vector<structured::cubed_sphere::domain_descriptor::domain_id_type> m_cubed_ids; // cubed-sphere patterns
    explicit pattern_container(ghexb_pattern h)
    : m_h(h, [](ghexb_pattern p) { if (p) ghexb_pattern_destroy(p); })
    {
    }
    template<typename G, typename H, typename R>
    friend auto make_pattern(context&, const H&, const R&);
};

// make_pattern<structured::grid>(ctxt, halo_gen, domain_range) and
// make_pattern<unstructured::grid>(ctxt, halo_gen, domain_range)
template<typename Grid, typename HaloGenerator, typename DomainRange>
auto make_pattern(context& ctxt, const HaloGenerator& hg, const DomainRange& domains)
{
    static_assert(std::is_same<Grid, structured::grid>::value || std::is_same<Grid, unstructured::grid>::value,
        "this front end covers the regular structured grid and unstructured column data");
    using dom_type = typename std::decay<decltype(*std::begin(domains))>::type;
    if constexpr (std::is_same<dom_type, structured::cubed_sphere::domain_descriptor>::value)
    {
        // make_pattern<structured::grid> over cubed-sphere domains (GHEX dispatches on the domain type)
        std::vector<int> tiles, x0, x1, y0, y1;
        int edge = 0, levels = 0;
        std::vector<structured::cubed_sphere::domain_descriptor::domain_id_type> ids;
        for (const auto& d : domains)
        {
            tiles.push_back(d.tile()), x0.push_back(d.x()[0]), x1.push_back(d.x()[1]);
            y0.push_back(d.y()[0]), y1.push_back(d.y()[1]);
            edge = d.edge_size(), levels = d.levels();
            ids.push_back(d.domain_id());
        }
        ghexb_pattern h = nullptr;
        check(ghexb_pattern_create_cubed_sphere(ctxt.get(), edge, levels, hg.halos().data(), (int)tiles.size(), tiles.data(),
            x0.data(), x1.data(), y0.data(), y1.data(), &h));
        pattern_container<Grid, dom_type> pc(h);
        pc.m_cubed_ids = std::move(ids);
        return pc;
    }
    else if constexpr (std::is_same<Grid, unstructured::grid>::value)
    {
        std::vector<std::int64_t> ids, gid_off{0}, gids, outer_off{0}, outer, halo_off{0}, halo;
        for (const auto& d : domains)
        {
            ids.push_back((std::int64_t)d.domain_id());
            for (auto g : d.gids()) gids.push_back((std::int64_t)g);
            for (auto l : d.outer_lids()) outer.push_back((std::int64_t)l);
            gid_off.push_back((std::int64_t)gids.size());
            outer_off.push_back((std::int64_t)outer.size());
            if (!hg.all())
            {
                for (auto g : hg.gids()) halo.push_back((std::int64_t)g);
                halo_off.push_back((std::int64_t)halo.size());
            }
        }
        ghexb_pattern h = nullptr;
        check(ghexb_pattern_create_unstructured(ctxt.get(), (int)ids.size(), ids.data(), gid_off.data(), gids.data(),
            outer_off.data(), outer.data(), hg.all() ? nullptr : halo_off.data(), hg.all() ? nullptr : halo.data(), &h));
        return pattern_container<Grid, dom_type>(h);
    }
    else
    {
        constexpr int dim = dom_type::dim;
        std::vector<std::int64_t> ids;
        std::vector<int> firsts, lasts;
        for (const auto& d : domains)
        {
            ids.push_back((std::int64_t)d.domain_id());
            firsts.insert(firsts.end(), d.first().begin(), d.first().end());
            lasts.insert(lasts.end(), d.last().begin(), d.last().end());
        }
        std::array<int, dim> periodic{};
        for (int a = 0; a < dim; ++a) periodic[a] = hg.periodic()[a] ? 1 : 0;
        ghexb_pattern h = nullptr;
        check(ghexb_pattern_create_regular(ctxt.get(), dim, hg.global_first().data(), hg.global_last().data(), hg.halos().data(),
            periodic.data(), (int)ids.size(), ids.data(), firsts.data(), lasts.data(), &h));
        return pattern_container<Grid, dom_type>(h);
    }
}

// The handle of one exchange: wait() blocks until the halos are written (communication_handle)
class [[nodiscard]] communication_handle
{
  public:
    void wait()
    {
        if (!m_h) return;
        check(ghexb_handle_wait(m_h.get()));
        m_h.reset();
        m_keep.clear();
    }
    bool is_ready()
    {
        if (!m_h) return true;
        int ready = 0;
        check(ghexb_handle_is_ready(m_h.get(), &ready));
        return ready != 0;
    }
    void progress() {} // nothing to progress: the exchange is a stream-ordered kernel

  private:
    detail::owned<ghexb_handle_s, ghexb_handle_destroy> m_h;
    std::vector<buffer_info> m_keep; // the fields stay bound until the exchange completed
    template<typename> friend class communication_object;
};

template<typename Pattern>
class communication_object
{
  public:
    explicit communication_object(context& ctxt)
    {
        ghexb_co h = nullptr;
        check(ghexb_co_create(ctxt.get(), &h));
        m_h.reset(h);
    }

    // exchange(pattern(f1), pattern(f2), ...); throws "earlier exchange operation was not
    // finished" when the previous exchange has not been waited for
    template<typename... BufferInfos>
    communication_handle exchange(const buffer_info& first, const BufferInfos&... rest)
    {
        std::vector<buffer_info> bis{first, rest...};
        return exchange(bis.begin(), bis.end());
    }

    // exchange(first, last) over a range of buffer_infos
    template<typename Iterator,
        typename = typename std::enable_if<!std::is_same<typename std::decay<Iterator>::type, buffer_info>::value>::type>
    communication_handle exchange(Iterator first, Iterator last)
    {
        communication_handle hd;
        std::vector<ghexb_field> fields;
        for (auto it = first; it != last; ++it)
        {
            fields.push_back(it->get());
            hd.m_keep.push_back(*it);
        }
        ghexb_handle h = nullptr;
        check(ghexb_co_exchange(m_h.get(), fields.data(), (int)fields.size(), nullptr, &h));
        hd.m_h.reset(h);
        return hd;
    }

  private:
    detail::owned<ghexb_co_s, ghexb_co_destroy> m_h;
};

// make_communication_object<Pattern>(ctxt)
template<typename Pattern>
communication_object<Pattern> make_communication_object(context& ctxt)
{
    return communication_object<Pattern>(ctxt);
}
} // namespace ghexb

#endif /* GHEX_B200_HPP */

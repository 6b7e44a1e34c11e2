// Host-side core types of ghex_b200: patterns, pattern-bound fields and the work-descriptor
// tables that the kernels walk. Everything here is plain C++ (no CUDA types) except the
// descriptor structs shared with the device code in descriptors.hpp.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ghex_b200.h"
#include "descriptors.hpp"

namespace ghexb
{

// Exception carrying a C-ABI status code; every extern "C" entry point catches it and turns it
// into (code, thread-local message).
struct error : std::runtime_error
{
    int code;
    error(int c, const std::string& msg)
    : std::runtime_error(msg)
    , code(c)
    {
    }
};

inline int dtype_size(int dt)
{
    switch (dt)
    {
        case GHEXB_F32: return 4;
        case GHEXB_F64: return 8;
        case GHEXB_I32: return 4;
        case GHEXB_I64: return 8;
        case GHEXB_U8: return 1;
        case GHEXB_U16: return 2;
        default: throw error(GHEXB_ERR_INVALID, "unknown dtype code " + std::to_string(dt));
    }
}
inline bool dtype_is_float(int dt) { return dt == GHEXB_F32 || dt == GHEXB_F64; }

using coord4 = std::array<int, 4>;

// A pair of iteration spaces: the same box in the owning domain's local coordinates and in
// global coordinates (structured/pattern.hpp:95-120). Coordinates are inclusive.
struct space_pair
{
    coord4 lfirst{}, llast{}, gfirst{}, glast{};
    // staged patterns: the receive space's data comes from the matching send space of the
    // neighbour, whose first cell is sfirst in the neighbour's local coordinates (the global
    // coordinates of a staged receive space are not wrapped and do not locate the source)
    bool has_src = false;
    coord4 sfirst{};
};

// The iteration spaces one domain receives from (or sends to) one neighbour domain: one entry
// of pattern::recv_halos()/send_halos() (structured/pattern.hpp:150-152).
struct struct_entry
{
    int neighbor = -1; // index of the neighbour in the pattern's domain list
    int tag = 0;
    std::vector<space_pair> spaces;
};

// One entry of an unstructured pattern's halo maps (unstructured/pattern.hpp:93-124): local
// indices in the receiver's halo order.
struct list_entry
{
    int neighbor = -1;
    int tag = 0;
    std::vector<int64_t> lids;
};

enum class pattern_kind
{
    regular,
    cubed_sphere,
    unstructured
};

struct domain_info
{
    int64_t id = 0;   // user id (regular / unstructured), list index (cubed sphere)
    coord4 first{};   // regular: x,y,z ; cubed sphere: tile,x,y,z
    coord4 last{};
    int tile = 0;     // cubed sphere
    int64_t size = 0; // unstructured: number of local ids
    std::vector<int64_t> outer; // unstructured: outer (halo) local ids, ascending
    std::vector<struct_entry> recv, send;
    std::vector<list_entry> urecv, usend;
};

struct context_s
{
    int device = 0;
    int num_sms = 148;
};

} // namespace ghexb

struct ghexb_context_s : ghexb::context_s
{
};

struct ghexb_pattern_s
{
    ghexb_context_s* ctx = nullptr;
    ghexb::pattern_kind kind = ghexb::pattern_kind::regular;
    int dim = 3;        // regular: domain dimension; cubed sphere: 4 (tile,x,y,z)
    int edge_size = 0;  // cubed sphere
    int levels = 0;     // cubed sphere
    int max_tag = 0;
    std::vector<ghexb::domain_info> domains;
    int find_domain(int64_t id) const
    {
        for (size_t i = 0; i < domains.size(); ++i)
            if (domains[i].id == id) return (int)i;
        return -1;
    }
};

struct ghexb_field_s
{
    ghexb_pattern_s* pattern = nullptr;
    int domain_index = -1;
    int dtype = GHEXB_F64;
    int esize = 8;
    char* data = nullptr;
    // structured
    int ndim = 0;
    std::array<int, 4> offsets{};
    std::array<int, 4> extents{};
    std::array<int, 4> layout{};
    std::array<int64_t, 4> byte_strides{};
    int num_components = 1;
    bool is_vector = false;
    // unstructured
    int64_t levels = 1;
    bool levels_first = true;
    int64_t index_stride = 1; // elements
    int64_t level_stride = 1; // elements
};

namespace ghexb
{
// pattern builders (pattern_regular.cpp, pattern_cubed_sphere.cpp, pattern_unstructured.cpp)
void build_regular_staged(ghexb_pattern_s* const* stages, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n, const int64_t* ids, const int* first, const int* last,
    const int64_t* neighbor_ids);
void build_regular(ghexb_pattern_s& p, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n, const int64_t* ids, const int* first,
    const int* last);
void build_cubed_sphere(ghexb_pattern_s& p, int edge, int levels, const int* halos, int n,
    const int* tiles, const int* x_first, const int* x_last, const int* y_first,
    const int* y_last);
// hint_off == nullptr: no receive domain ids generator
void build_unstructured(ghexb_pattern_s& p, int n, const int64_t* ids, const int64_t* gid_off,
    const int64_t* gids, const int64_t* outer_off, const int64_t* outer_lids,
    const int64_t* halo_off, const int64_t* halo_gids, const int64_t* hint_off = nullptr,
    const int64_t* hint_ids = nullptr, const int64_t* hint_remote = nullptr);

// cubed-sphere coordinate transforms (pattern_cubed_sphere.cpp)
struct cs_transform
{
    std::array<int, 4> rot;
    std::array<int, 2> trans;
    std::array<int, 2> off;
    bool switched_xy() const { return rot[0] == 0; }
    bool reversed_x() const { return switched_xy() ? rot[1] == -1 : rot[0] == -1; }
    bool reversed_y() const { return switched_xy() ? rot[2] == -1 : rot[3] == -1; }
    std::array<int, 2> apply(int x, int y, int c) const
    {
        return {rot[0] * x + rot[1] * y + trans[0] * c + off[0],
            rot[2] * x + rot[3] * y + trans[1] * c + off[1]};
    }
};
int cs_neighbor_tile(int tile, int n);
const cs_transform& cs_forward(int tile, int n);
const cs_transform& cs_inverse(int tile, int n);
const cs_transform& cs_identity();
} // namespace ghexb

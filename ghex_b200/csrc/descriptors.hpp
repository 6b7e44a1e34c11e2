// Work descriptors shared by the host plan builder and the device kernels.
//
// A halo exchange is lowered, once per field set, into a flat table of descriptors:
//  * box_desc  — a strided (up to 4-D) box copied from a source field into a destination field.
//                The source strides are signed and given per destination dimension, so the
//                cubed-sphere edge transforms (reversal, x/y switch) are just other strides.
//  * list_desc — an index-list gather/scatter of unstructured column data.
// Kernels never see patterns, fields or domains: only these tables plus tile lists.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define GHEXB_HD __host__ __device__ __forceinline__
#else
#define GHEXB_HD inline
#endif

namespace ghexb
{

// Unsigned division by an invariant divisor d >= 1 through a multiply-high and a shift
// (Granlund & Montgomery, "Division by invariant integers using multiplication", PLDI 1994,
// round-up variant): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (umulhi(n, m) + n) >> l for all n < 2^31.
struct fast_div
{
    uint32_t d;
    uint32_t m;
    uint32_t l;

    static fast_div make(uint32_t divisor)
    {
        fast_div f{divisor, 1u, 0u};
        uint32_t l = 0;
        while ((1ull << l) < divisor) ++l;
        f.l = l;
        f.m = (uint32_t)(((1ull << 32) * ((1ull << l) - divisor)) / divisor + 1ull);
        return f;
    }

    GHEXB_HD uint32_t div(uint32_t n) const
    {
#if defined(__CUDA_ARCH__)
        return (__umulhi(n, m) + n) >> l;
#else
        return (uint32_t)((((uint64_t)n * m) >> 32) + n) >> l;
#endif
    }
};

// How the lanes of a warp cover rows of n elements: W = 2^wlog lanes share a row (W is the next
// power of two of n, at most 32), each taking j = ceil(n / W) elements, and a thread takes p rows
// per pipeline chunk, so that p * j <= 8 elements per thread and chunk.
struct row_map
{
    uint8_t wlog;
    uint8_t j;
    uint8_t p;
    uint8_t pad;

    static row_map make(int n)
    {
        row_map m{0, 1, 8, 0};
        while ((1 << m.wlog) < n && m.wlog < 5) ++m.wlog;
        m.j = (uint8_t)((n + (1 << m.wlog) - 1) >> m.wlog);
        m.p = (uint8_t)(m.j > 8 ? 1 : 8 / m.j);
        return m;
    }
};

// Strided box copy, organised in rows: for every row r < n1 * n2 with (i1, i2) = (r mod n1, r / n1)
// and every i0 < n0
//   dst[i0*d0 + i1*d1 + i2*d2] = src[i0*s0 + i1*s1 + i2*s2] ^ xor_mask
// in units of `esize` bytes. Dimension 0 is the destination's contiguous dimension and n0 <= 256
// (longer rows are split into several descriptors). All offsets fit int32.
struct alignas(16) box_desc
{
    const char* src;
    char* dst;
    int32_t n0, n1, n2;
    int32_t s0, s1, s2;
    int32_t d0, d1, d2;
    uint32_t esize;     // bytes per element: 1, 2, 4 or 8
    uint32_t field;     // logical field the descriptor belongs to
    row_map map;
    uint64_t xor_mask;  // sign-bit mask for negated vector components, else 0
    fast_div div1;      // divides a row index by n1
};

// Index-list copy of column data, organised in rows (columns): for k < count, l < levels
//   dst[didx[k]*d_is + l*d_ls] = src[sidx[k]*s_is + l*s_ls]
// in units of `unit` bytes (16 when every column is 16-byte aligned, else the element size);
// levels <= 256 units per descriptor.
struct alignas(16) list_desc
{
    const char* src;
    char* dst;
    const int32_t* sidx;
    const int32_t* didx;
    int32_t count;
    int32_t levels; // in units
    int32_t s_is, s_ls, d_is, d_ls; // in units
    uint32_t unit;
    uint32_t field;
    row_map map;
};

// A forward work item: the elements [e0, e0 + count) of one box or list descriptor, or of a
// pair of x-face boxes, with all the kernel needs to address them, so that a CTA reads one
// 112-byte record and nothing else before its data loads.
//  * box:  element e -> i0 = e mod n0, r = e / n0, i1 = r mod n1, i2 = r / n1;
//          dst[i0*d0 + i1*d1 + i2*d2] = src[i0*s0 + i1*s1 + i2*s2]  (sign bit flipped if neg)
//  * list: element e -> k = e / n0 (column), l = e mod n0 (level);
//          dst[didx[k]*d0 + l*d1] = src[sidx[k]*s0 + l*s1]
//  * pair: two boxes A and B of short rows in one destination field whose rows interleave in
//          memory: row r of A ends where row r + 1 of B begins (the high-x halo of a row and the
//          low-x halo of the next). Element e -> segment q = e / n0 (n0 = na + nb elements),
//          c = e mod n0, plane i2 = q / n1, s = q mod n1 (n1 = rows + 1); the segment is
//          contiguous in the destination: dst[c + (s - 1)*d1 + i2*d2]. Its first na elements
//          come from A row s - 1 (s >= 1): src[c*s0 + (s-1)*s1 + i2*s2], the others from B row
//          s (s < rows): src2[(c-na)*u0 + s*u1 + i2*u2]. Writing both halos of a row boundary
//          in one coalesced store turns partial-sector writes into whole-sector ones.
// Offsets are in units of `unit` bytes (the element size; 16 for aligned list columns).
struct alignas(16) xtile
{
    const char* src;
    char* dst;
    const int32_t* sidx;
    const int32_t* didx;
    const char* src2; // pair: source of box B
    uint32_t e0, count;
    int32_t s0, s1, s2;
    int32_t d0, d1, d2;
    int32_t u0, u1, u2; // pair: source strides of box B
    uint32_t n0, m0;    // first extent and its fast-division magic
    uint32_t n1, m1;    // second extent (boxes, pairs)
    uint32_t na;        // pair: row length of box A
    uint8_t l0, l1;     // fast-division shifts
    uint8_t unit;       // bytes per element: 1, 2, 4, 8 or 16
    uint8_t kind;       // 0 box, 1 list, 2 pair
    uint8_t neg;        // 1: flip the sign bit (negated cubed-sphere vector components); pair: of A
    uint8_t neg2;       // pair: of B
    uint8_t cls;        // element class (exchange.hpp): kind, unit and neg in one value
    uint8_t pad[1];
};
static_assert(sizeof(xtile) == 112, "xtile is seven 16-byte words");
constexpr int k_xtile_words = 7;

// Adjoint of the boxes in gather form. The owner elements read by the forward boxes of one
// source field are cut into disjoint cells (boxes in the owner's coordinates); every element of
// a cell was copied to the same ordered list of halo images. For an owner element o:
//   acc = own[o]; for each image i in order: acc = acc (+|-) img_i[o]; img_i[o] = 0; own[o] = acc
// which is the explicit transpose in receive order, with no two threads touching one element.
// Unstructured columns take the same form: a group of owner columns with the same number of
// images; the column table holds, per owner, the address of its column and of each image's
// column (nimg + 1 addresses), and element e of the group is level e mod n0 of owner e / n0.
constexpr int k_max_images = 8;

struct gimage
{
    char* ptr;            // image of the cell's element (0,0,0)
    int32_t t0, t1, t2;   // element strides of the image per cell axis
    uint32_t neg;         // 1: the forward negated this image
};

struct alignas(16) gtile
{
    char* own;            // box: owner element (0,0,0) of the cell
    uint32_t e0, count;   // elements [e0, e0 + count) of the cell (list: of the owner group)
    int32_t o0, o1, o2;   // owner element strides per cell axis (axis 0 fastest); list: o0 = level stride
    uint32_t n0, m0, n1, m1;
    uint8_t l0, l1;
    uint8_t esize;        // 4 or 8 (float or double)
    uint8_t nimg;         // 1..k_max_images
    gimage img[k_max_images]; // list: img[0].t0 = level stride of the images
    uint8_t cls;          // element class (exchange.hpp): kind, esize and nimg in one value
    uint8_t kind;         // 0 box cell, 1 group of unstructured owner columns
    uint8_t pad0[2];
    uint32_t col0;        // list: first entry of the group in the column table
    uint8_t pad[8];
};
static_assert(sizeof(gtile) == 256, "gtile is sixteen 16-byte words");

// Host form of a gather cell, relative to field slots so that it survives a rebind.
struct gcell
{
    int own_slot;
    int64_t own_off;        // owner element (0,0,0), elements from the field's data
    int32_t n[3];           // extents along the cell axes (axis 0 fastest in the owner)
    int32_t o[3];           // owner element strides
    int nimg;
    struct
    {
        int slot;
        int64_t off;        // image of element (0,0,0), elements from the field's data
        int32_t t[3];
        uint32_t neg;
    } img[k_max_images];
    int esize;
};

// A contiguous range [start, start+count) of one descriptor's rows.
struct alignas(16) tile
{
    int32_t desc;
    int32_t kind; // 0: box, 1: list
    uint32_t start;
    uint32_t count;
};

} // namespace ghexb

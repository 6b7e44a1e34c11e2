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

// A contiguous range [start, start+count) of one descriptor's rows.
struct alignas(16) tile
{
    int32_t desc;
    int32_t kind; // 0: box, 1: list
    uint32_t start;
    uint32_t count;
};

} // namespace ghexb

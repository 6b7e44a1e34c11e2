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

// Strided box copy: for every (i0,i1,i2,i3) < (n0,n1,n2,n3)
//   dst[i0*d0 + i1*d1 + i2*d2 + i3*d3] = src[i0*s0 + i1*s1 + i2*s2 + i3*s3] ^ xor_mask
// in units of `esize` bytes. i0 runs fastest and is the destination's contiguous dimension.
// All offsets fit int32 (checked when the table is built).
struct alignas(16) box_desc
{
    const char* src;
    char* dst;
    int32_t n0, n1, n2, n3;
    int32_t s0, s1, s2, s3;
    int32_t d0, d1, d2, d3;
    uint32_t esize;     // bytes per element: 1, 2, 4 or 8
    uint32_t field;     // logical field the descriptor belongs to
    uint64_t xor_mask;  // sign-bit mask for negated vector components, else 0
    fast_div div0, div1, div2;
    uint32_t pad;
};

// Index-list copy of column data: for k < count, l < levels
//   dst[didx[k]*d_is + l*d_ls] = src[sidx[k]*s_is + l*s_ls]
// in units of `unit` bytes (16 when every column is 16-byte aligned, else the element size).
// If level_fastest, consecutive threads walk l, else k.
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
    uint32_t level_fastest;
    uint32_t field;
    fast_div divq; // divides by levels (level_fastest) or by count
};

// A contiguous range [start, start+count) of one descriptor's flattened index space.
struct alignas(16) tile
{
    int32_t desc;
    int32_t kind; // 0: box, 1: list
    uint32_t start;
    uint32_t count;
};

} // namespace ghexb

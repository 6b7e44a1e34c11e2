// Staged exchange of box descriptors through the tensor memory accelerator (sm_100a).
//
// The source region of a halo box is loaded by cp.async.bulk.tensor into a ring of shared-memory
// stages (one producer thread per CTA, completion counted on mbarriers) and written to the halo
// by the CTA's other warps with ordinary stores. A tensor map needs 16-byte aligned strides, so
// the source rows of a box are split into classes: rows i1 = a (mod p) and planes i2 = b (mod q)
// with p = 16 / gcd(row stride in bytes, 16) and q alike for planes, each class one 3-D map whose
// strides are p and q times the field's. Every map covers exactly its class's part of the source
// region (an x extent of the region plus the few elements before it down to a 16-byte boundary):
// a load box that reaches past the region is filled by the hardware without touching memory, so
// no byte outside the region is fetched. Boxes whose source rows are not contiguous along either
// destination axis stay on the element kernel (exchange.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ghexb
{
// One load and the writes of its elements. The elements of an item are enumerated as
// (u, v, z) with u fastest: u < nu, v < nv, z < nz (z counts the class planes of the load box);
// element (u, v, z) is at shared-memory element sbase + u*su + v*sv + z*sz of the stage and goes
// to dst + u*du + v*dv + z*dz (elements of es bytes). u runs along the destination's contiguous
// axis, so consecutive threads store consecutive addresses.
struct alignas(16) sitem
{
    char* dst;
    int32_t du, dv, dz;
    uint32_t map;            // index of the tensor map in the plan's map table
    int32_t c1, c2;          // load coordinates along the class rows and planes (x starts at 0)
    uint32_t bytes;          // bytes the load writes to shared memory (the whole box)
    uint32_t su, sv, sz;     // shared-memory element strides
    uint32_t sbase;          // shared-memory element of (0, 0, 0)
    uint32_t nu, mu;         // u extent and its fast-division magic
    uint32_t nv, mv;         // v extent and its magic
    uint32_t count;          // nu * nv * nz
    uint8_t lu, lv;          // fast-division shifts
    uint8_t es;              // element size in bytes: 1, 2, 4 or 8
    uint8_t neg;             // 1: flip the sign bit (negated cubed-sphere vector components)
    uint32_t pad;
};
static_assert(sizeof(sitem) == 80, "sitem is five 16-byte words");

struct staged_launch
{
    const sitem* items;
    const CUtensorMap* maps;
    unsigned* status;        // bit 0: a producer wait gave up, bit 1: a consumer wait gave up
    int nitems;
    int stages;              // shared-memory stages per CTA
    int stage_bytes;         // bytes per stage (a multiple of 128)
    int consumers;           // consumer warps per CTA
    int grid;                // CTAs (persistent: item i runs on CTA i mod grid)
};

// Launches the staged kernel; the caller has set the kernel's dynamic shared memory limit with
// staged_prepare(stages * stage_bytes + 128) (128 bytes to align the stages).
cudaError_t launch_staged(const staged_launch& a, cudaStream_t stream);
cudaError_t staged_prepare(int smem_bytes);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
CUresult encode_tensor_map(CUtensorMap* map, CUtensorMapDataType type, cuuint32_t rank, void* base,
    const cuuint64_t* dims, const cuuint64_t* strides, const cuuint32_t* box, CUtensorMapL2promotion promo);
} // namespace ghexb

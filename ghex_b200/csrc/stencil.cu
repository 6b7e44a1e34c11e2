// The 7-point update of the differentiable-exchange workload and its adjoint.
//
// GHEX has no stencil: this is the compute step of the program whose gradient the exchange's
// adjoint is checked in (exchange, then x <- x + alpha * L(x) on the interior, repeated). It is a
// plain memory-bound sweep; its arithmetic is spelled out with round-to-nearest intrinsics in a
// fixed order (no contraction into fused multiply-adds), so that an elementwise CPU restatement
// reproduces it bit for bit:
//
//   forward, interior p:   s  = ((((x[p-ex] + x[p+ex]) + x[p-ey]) + x[p+ey]) + x[p-ez]) + x[p+ez]
//                          y[p] = x[p] + alpha * (s - 6 * x[p])
//   forward, halo p:       y[p] = 0
//   adjoint, every p:      G(q) = gy[q] on the interior, 0 elsewhere (and outside the array)
//                          t  = ((((G(p-ex) + G(p+ex)) + G(p-ey)) + G(p+ey)) + G(p-ez)) + G(p+ez)
//                          gx[p] = G(p) + alpha * (t - 6 * G(p))
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "async_copy.hpp"
#include "stencil.hpp"

namespace ghexb
{
namespace
{
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <typename T> __device__ __forceinline__ T sub_rn(T a, T b);
template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

struct domain_args
{
    stencil_domain d[k_stencil_batch];
};

// A block of 32 x 8 threads computes a patch of 32 x (8 x rows) (i, j) columns of one domain
// (blockIdx.z) over a slab of planes, each thread the rows ty, ty + 8, ... of its column i. The
// planes it reads (the patch and a ring of one column around it) pass through shared memory:
// asynchronous element copies (cp.async, which zero-fill what the update treats as zero) keep
// k_ahead planes in flight ahead of the plane being computed, in a ring of k_stages plane
// buffers, and every neighbour is then a shared-memory read at a fixed offset. Element offsets
// advance by the plane stride from plane to plane (I: 32-bit when every offset of the launch
// fits, else 64-bit), so the work per element is a few copies, seven shared-memory reads, the
// arithmetic and one store.
constexpr int k_tx = 32, k_ty = 8, k_px = k_tx + 2;
constexpr int k_stages = 8, k_ahead = k_stages - 1;
constexpr int k_threads = k_tx * k_ty;

// Rows per thread: two for float (a 32 x 16 patch), one for double (32 x 8), the faster choice
// for each type on the 130 x 130 x 66 domains of the 256x256x128 program (forward, float: 33 us
// with two rows against 37 us with one; double: 44 us with one row against 50 us with two).
template <typename T> struct patch
{
    static constexpr int rows = sizeof(T) == 8 ? 1 : 2;
    static constexpr int plane = k_px * (k_ty * rows + 2);          // the patch and its ring
    static constexpr int slots = (plane + k_threads - 1) / k_threads; // copies per thread and plane
};
static_assert((k_stages & (k_stages - 1)) == 0, "a ring of a power of two");

template <typename T>
__device__ __forceinline__ void copy_element(uint32_t dst, const T* src, bool valid)
{
    // src-size 0 writes zeros and reads nothing
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"((int)sizeof(T)),
                 "r"(valid ? (int)sizeof(T) : 0)
                 : "memory");
}
__device__ __forceinline__ void copy_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void copy_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Buffer element (a, b) of a plane holds (i0 - 1 + a, j0 - 1 + b). Forward: every element in the
// array (an interior element reads only those); adjoint: G, the gradient on interior elements and
// zero elsewhere.
template <typename T, bool ADJOINT, typename I>
__global__ void __launch_bounds__(k_threads) stencil7_kernel(const __grid_constant__ domain_args args, T alpha,
    unsigned nslabs, unsigned nblocks_y, int slab)
{
    constexpr int k_rows = patch<T>::rows, k_plane = patch<T>::plane, k_slots = patch<T>::slots;
    __shared__ __align__(16) T buf[k_stages][k_plane];
    const stencil_domain& d = args.d[blockIdx.z];
    const T* __restrict__ in = static_cast<const T*>(d.in);
    T* __restrict__ out = static_cast<T*>(d.out);
    const int h = d.halo, ex = d.ex, ey = d.ey, ez = d.ez;
    const I sx = (I)d.sx, sy = (I)d.sy, sz = (I)d.sz;
    const auto within = [](int v, int lo, int hi) { return v >= lo && v < hi; };
    const int tid = threadIdx.y * k_tx + threadIdx.x;
    const int i0 = blockIdx.x * k_tx, i = i0 + threadIdx.x;
    // copied planes: forward [0, ez), adjoint [h, ez - h)
    const int klo = ADJOINT ? h : 0, khi = ADJOINT ? ez - h : ez;
    const uint32_t base = smem_u32(&buf[0][0]);
    for (unsigned b = blockIdx.y; b < nblocks_y; b += gridDim.y)
    {
        const unsigned ytile = b / nslabs;
        const int j0 = (int)ytile * (k_ty * k_rows);
        const int k0 = (int)(b - ytile * nslabs) * slab;
        if (i0 >= ex || j0 >= ey || k0 >= ez) continue; // uniform in the block
        const int nout = min(slab, ez - k0), nplanes = nout + 2;
        // this thread's elements of every plane buffer: offsets at plane k0 - 1 (advanced per plane)
        I src[k_slots];
        bool col[k_slots];
        uint32_t dst[k_slots];
#pragma unroll
        for (int r = 0; r < k_slots; ++r)
        {
            const int e = tid + r * k_threads;
            const int gi = i0 - 1 + e % k_px, gj = j0 - 1 + e / k_px;
            col[r] = e < k_plane && (ADJOINT ? within(gi, h, ex - h) && within(gj, h, ey - h) : within(gi, 0, ex) && within(gj, 0, ey));
            src[r] = col[r] ? (I)gi * sx + (I)gj * sy + (I)(k0 - 1) * sz : I(0);
            dst[r] = base + (uint32_t)(min(e, k_plane - 1) * sizeof(T));
        }
        int next = 0; // the next plane to copy
        const auto issue = [&]() {
            if (next < nplanes)
            {
                const int k = k0 - 1 + next;
                const bool kin = k >= klo && k < khi;
                const uint32_t so = (uint32_t)((next & (k_stages - 1)) * (k_plane * (int)sizeof(T)));
#pragma unroll
                for (int r = 0; r < k_slots; ++r)
                {
                    const bool ok = col[r] && kin;
                    if ((r + 1) * k_threads <= k_plane || tid + r * k_threads < k_plane)
                        copy_element(dst[r] + so, in + (ok ? src[r] : I(0)), ok);
                    src[r] += sz;
                }
            }
            ++next;
            copy_commit(); // an empty group past the last plane keeps the count of groups uniform
        };
#pragma unroll
        for (int L = 0; L < k_ahead; ++L) issue();
        int c[k_rows];
        bool mine[k_rows], col_in[k_rows];
        I o[k_rows];
#pragma unroll
        for (int q = 0; q < k_rows; ++q)
        {
            const int ty = threadIdx.y + q * k_ty, j = j0 + ty;
            c[q] = (ty + 1) * k_px + threadIdx.x + 1;
            mine[q] = i < ex && j < ey;
            col_in[q] = within(i, h, ex - h) && within(j, h, ey - h);
            o[q] = mine[q] ? (I)i * sx + (I)j * sy + (I)k0 * sz : I(0);
        }
        for (int m = 0; m < nout; ++m)
        {
            // planes m, m + 1 and m + 2 have landed (groups through m + k_ahead - 1 were committed)
            copy_wait<k_ahead - 3>();
            __syncthreads();
            issue(); // plane m + k_ahead, into the buffer of plane m - 1, which every thread has read
            const T* zm = buf[m & (k_stages - 1)];
            const T* pk = buf[(m + 1) & (k_stages - 1)];
            const T* zp = buf[(m + 2) & (k_stages - 1)];
            const bool kin = within(k0 + m, h, ez - h);
#pragma unroll
            for (int q = 0; q < k_rows; ++q)
            {
                const int cq = c[q];
                T y;
                if constexpr (!ADJOINT)
                {
                    y = T(0);
                    if (col_in[q] && kin)
                    {
                        const T x = pk[cq];
                        T s = add_rn(pk[cq - 1], pk[cq + 1]);
                        s = add_rn(s, pk[cq - k_px]);
                        s = add_rn(s, pk[cq + k_px]);
                        s = add_rn(s, zm[cq]);
                        s = add_rn(s, zp[cq]);
                        y = add_rn(x, mul_rn(alpha, sub_rn(s, mul_rn(T(6), x))));
                    }
                }
                else
                {
                    const T g = pk[cq];
                    T t = add_rn(pk[cq - 1], pk[cq + 1]);
                    t = add_rn(t, pk[cq - k_px]);
                    t = add_rn(t, pk[cq + k_px]);
                    t = add_rn(t, zm[cq]);
                    t = add_rn(t, zp[cq]);
                    y = add_rn(g, mul_rn(alpha, sub_rn(t, mul_rn(T(6), g))));
                }
                if (mine[q]) out[o[q]] = y;
                o[q] += sz;
            }
        }
        // the next slab's copies reuse the buffers: all copies landed, all reads done
        copy_wait<0>();
        __syncthreads();
    }
}

template <typename T, typename I>
void launch_kernel(bool adjoint, dim3 grid, const domain_args& args, T alpha, unsigned nslabs, unsigned ny, int slab,
    cudaStream_t stream)
{
    const dim3 block(k_tx, k_ty);
    if (adjoint)
        stencil7_kernel<T, true, I><<<grid, block, 0, stream>>>(args, alpha, nslabs, ny, slab);
    else
        stencil7_kernel<T, false, I><<<grid, block, 0, stream>>>(args, alpha, nslabs, ny, slab);
}

template <typename T>
cudaError_t launch_t(const stencil_domain* doms, int n, double alpha, bool adjoint, cudaStream_t stream)
{
    for (int b = 0; b < n; b += k_stencil_batch)
    {
        domain_args args{};
        const int m = n - b < k_stencil_batch ? n - b : k_stencil_batch;
        int mx = 0, my = 0, mz = 0;
        bool narrow = true; // every element offset, and the offsets advanced two planes past the end, below 2^31
        for (int i = 0; i < m; ++i)
        {
            const stencil_domain& d = doms[b + i];
            args.d[i] = d;
            mx = std::max(mx, d.ex), my = std::max(my, d.ey), mz = std::max(mz, d.ez);
            const int64_t span = (int64_t)(d.ex - 1) * d.sx + (int64_t)(d.ey - 1) * d.sy + (int64_t)(d.ez + 2) * d.sz;
            narrow = narrow && span < ((int64_t)1 << 31) - 1;
        }
        if (mx <= 0 || my <= 0 || mz <= 0) continue;
        // slabs of about 16 planes, of equal depth
        const int nsl = (mz + 15) / 16, slab = (mz + nsl - 1) / nsl;
        const unsigned xtiles = (unsigned)((mx + k_tx - 1) / k_tx);
        const unsigned nslabs = (unsigned)((mz + slab - 1) / slab);
        constexpr int rows = k_ty * patch<T>::rows;
        const uint64_t ny = (uint64_t)((my + rows - 1) / rows) * nslabs;
        if (ny > 0xffffffffull) return cudaErrorInvalidValue;
        const dim3 grid(xtiles, (unsigned)std::min<uint64_t>(ny, 65535), (unsigned)m);
        if (narrow)
            launch_kernel<T, int32_t>(adjoint, grid, args, (T)alpha, nslabs, (unsigned)ny, slab, stream);
        else
            launch_kernel<T, int64_t>(adjoint, grid, args, (T)alpha, nslabs, (unsigned)ny, slab, stream);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
} // namespace

cudaError_t launch_stencil7(bool f64, const stencil_domain* doms, int n, double alpha, bool adjoint, cudaStream_t stream)
{
    return f64 ? launch_t<double>(doms, n, alpha, adjoint, stream) : launch_t<float>(doms, n, alpha, adjoint, stream);
}
} // namespace ghexb

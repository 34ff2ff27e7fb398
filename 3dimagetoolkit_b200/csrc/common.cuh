// common.cuh -- shared definitions of the sm_100a kernels of the RSFE Split-Bregman path.
//
// Volume layout is the reference's image3d layout (header/image3d_imp.hxx:142-153):
// (i, j, k) at (i*ny + j)*nz + k, k contiguous.
//
// Colour-packed layout (Gauss-Seidel only): the points with even (i+j+k) ("red") and
// odd (i+j+k) ("black") are stored in two arrays of nx*ny*hz elements, hz = (nz+1)/2,
// point (i, j, k) at (i*ny + j)*hz + (k >> 1) of the array of its colour. Every
// neighbour of a point has the other colour, and its packed index is found with the
// same formula, so a half-sweep reads one colour and writes the other with unit
// stride along the packed axis.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace im3d {

struct Dims {
    int nx, ny, nz;
    // boundary of the Gaussian convolution passes: 0 = zero outside the volume
    // (acyclic_fftw_convolution), 1 = periodic (cyclic_fftw_convolution)
    int cyc = 0;
    // a halo index along an axis of length n: false when outside and the boundary is
    // zero, else the index (wrapped into [0, n) for the periodic boundary)
    __host__ __device__ bool halo(int a, int n, int& out) const
    {
        if (a >= 0 && a < n) {
            out = a;
            return true;
        }
        if (!cyc) return false;
        int r = a % n;
        if (r < 0) r += n;
        out = r;
        return true;
    }
    __host__ __device__ long long n() const { return (long long)nx * ny * nz; }
    // packed row pitch: (nz+1)/2 points of one colour, padded to a multiple of 4 so that
    // every packed row starts 16-byte aligned (padding slots hold no point: k >= nz)
    __host__ __device__ int hz() const { return (((nz + 1) >> 1) + 3) & ~3; }
    __host__ __device__ long long npk() const { return (long long)nx * ny * hz(); }
    __host__ __device__ long long idx(int i, int j, int k) const
    {
        return ((long long)i * ny + j) * nz + k;
    }
    __host__ __device__ long long pidx(int i, int j, int k) const
    {
        return ((long long)i * ny + j) * hz() + (k >> 1);
    }
};

template <typename T, int N>
struct alignas(sizeof(T) * N <= 16 ? sizeof(T) * N : 16) Vec {
    T v[N];
};

// 16-byte vector of T: 4 floats or 2 doubles
template <typename T>
struct V16;
template <>
struct V16<float> {
    static constexpr int W = 4;
    typedef float4 type;
    __device__ static float get(const float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
    __device__ static void set(float4& v, int c, float x)
    {
        if (c == 0) v.x = x;
        else if (c == 1) v.y = x;
        else if (c == 2) v.z = x;
        else v.w = x;
    }
};
template <>
struct V16<double> {
    static constexpr int W = 2;
    typedef double2 type;
    __device__ static double get(const double2& v, int c) { return c == 0 ? v.x : v.y; }
    __device__ static void set(double2& v, int c, double x)
    {
        if (c == 0) v.x = x;
        else v.y = x;
    }
};

template <typename T, int N>
__device__ __forceinline__ Vec<T, N> vzero()
{
    Vec<T, N> r;
#pragma unroll
    for (int q = 0; q < N; ++q) r.v[q] = T(0);
    return r;
}

// Device-side control block: FP64 accumulators of the global reductions, written
// with atomics by the kernels and read back by the host between launches.
struct Ctrl {
    double sum[8];
    unsigned long long umax[4];
    int flag[8];
};

enum CtrlSlot {
    SUM_DPHI2 = 0,  // sum (phi - phiold)^2
    SUM_PHIOLD2 = 1,  // sum phiold^2
    SUM_RES2 = 2,   // sum residual^2 of the Poisson solve
    SUM_BEFF2 = 3,  // sum (b + u_in/dt)^2
    SUM_A = 4,      // scratch
    SUM_B = 5,
};

template <typename T>
__device__ __forceinline__ T ld_g(const T* p)
{
    return __ldg(p);
}

// Warp + block reduction of a double, one atomicAdd per block.
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Linear index and count of the blocks of a grid. The kernel bodies take their block
// index and grid as arguments (a work-list launch over several volumes passes each
// block's index within its own volume's grid), so these take them too.
__device__ __forceinline__ long long block_linear_id(const uint3 b, const dim3 g)
{
    return b.x + (long long)g.x * (b.y + (long long)g.y * b.z);
}

__device__ __forceinline__ long long grid_blocks(const dim3 g)
{
    return (long long)g.x * g.y * g.z;
}

// Block sums of one or two doubles, written by thread 0 to block bid's slot of `part`
// (part[bid] and, for the second value, part[nblocks + bid]). No atomics: a one-block
// finalize kernel adds the slots in a fixed order, so the totals do not depend on
// block scheduling.
template <int NWARPS_MAX = 32>
__device__ __forceinline__ void block_sum_store(double v, double* part, long long bid)
{
    __shared__ double red_sm[NWARPS_MAX];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    v = warp_sum(v);
    if ((tid & 31) == 0) red_sm[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
        double w = (tid < ((nthreads + 31) >> 5)) ? red_sm[tid] : 0.0;
        w = warp_sum(w);
        if (tid == 0) part[bid] = w;
    }
}

template <int NWARPS_MAX = 32>
__device__ __forceinline__ void block_sum2_store(double a, double b, double* part, long long bid,
                                                 long long nblocks)
{
    __shared__ double red_a[NWARPS_MAX], red_b[NWARPS_MAX];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    a = warp_sum(a);
    b = warp_sum(b);
    if ((tid & 31) == 0) {
        red_a[tid >> 5] = a;
        red_b[tid >> 5] = b;
    }
    __syncthreads();
    if (tid < 32) {
        const bool live = tid < ((nthreads + 31) >> 5);
        double wa = live ? red_a[tid] : 0.0;
        double wb = live ? red_b[tid] : 0.0;
        wa = warp_sum(wa);
        wb = warp_sum(wb);
        if (tid == 0) {
            part[bid] = wa;
            part[nblocks + bid] = wb;
        }
    }
}

// sums[slot + v] = sum over b of part[v * nblocks + b], v < nvals, in a fixed order.
// One block of kFinThreads threads: thread t adds the slots b = t + m * kFinThreads in
// four interleaved accumulators (m mod 4), so that four loads are in flight, then the
// block adds the accumulators and the threads' sums in a fixed tree.
constexpr int kFinThreads = 1024;
__device__ __forceinline__ void finalize_sums_body(const double* __restrict__ part, long long nblocks,
                                                   int nvals, double* sums, int slot)
{
    __shared__ double sm[kFinThreads];
    for (int v = 0; v < nvals; ++v) {
        const double* pv = part + v * nblocks;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        long long b = threadIdx.x;
        for (; b + 3 * kFinThreads < nblocks; b += 4 * kFinThreads) {
            a0 += pv[b];
            a1 += pv[b + kFinThreads];
            a2 += pv[b + 2 * kFinThreads];
            a3 += pv[b + 3 * kFinThreads];
        }
        if (b < nblocks) a0 += pv[b];
        if (b + kFinThreads < nblocks) a1 += pv[b + kFinThreads];
        if (b + 2 * kFinThreads < nblocks) a2 += pv[b + 2 * kFinThreads];
        sm[threadIdx.x] = (a0 + a1) + (a2 + a3);
        __syncthreads();
        for (int w = kFinThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) sums[slot + v] = sm[0];
        __syncthreads();
    }
}

static __global__ void __launch_bounds__(kFinThreads) finalize_sums_kernel(const double* __restrict__ part,
                                                                    long long nblocks, int nvals,
                                                                    double* sums, int slot)
{
    finalize_sums_body(part, nblocks, nvals, sums, slot);
}

}  // namespace im3d

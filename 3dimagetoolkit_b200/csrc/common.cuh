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
    __host__ __device__ long long n() const { return (long long)nx * ny * nz; }
    __host__ __device__ int hz() const { return (nz + 1) >> 1; }
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

template <int NWARPS_MAX = 32>
__device__ __forceinline__ void block_sum_atomic(double v, double* target)
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
        if (tid == 0 && w != 0.0) atomicAdd(target, w);
    }
}

// Two sums at once (halves the barrier count of the tolerance reductions).
template <int NWARPS_MAX = 32>
__device__ __forceinline__ void block_sum2_atomic(double a, double b, double* ta, double* tb)
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
            if (wa != 0.0) atomicAdd(ta, wa);
            if (wb != 0.0) atomicAdd(tb, wb);
        }
    }
}

}  // namespace im3d

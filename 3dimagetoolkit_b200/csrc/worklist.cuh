// Work-list launches: one grid over the blocks of several volumes.
//
// A batch of volumes that advance their outer iterations together runs each stage of
// the loop as ONE launch instead of one per volume. The launch's flat grid is the
// concatenation of the volumes' own grids: entry e of the WorkList covers the flat
// blocks [first[e], first[e+1]) and names the volume (an index into a table of jobs in
// device memory, one per volume, holding that volume's arguments and grid). Each block
// finds its entry by a binary search over `first`, turns its offset into the block
// index of the volume's own grid and runs the stage's kernel body with it. A body sees
// exactly the block index, grid and arguments of the single-volume launch, so every
// voxel is computed by the same operations, and the per-block partial sums of the
// reductions land in the same slots of the volume's own partials: results are
// bit-identical to volume-at-a-time runs.
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace im3d {

constexpr int kMaxListVols = 64;

struct WorkList {
    int n;                                // entries (volumes) of this launch
    int vol[kMaxListVols];                // each entry's index into the job table
    int flag[kMaxListVols];               // a per-volume flag handed to the job
    unsigned first[kMaxListVols + 1];     // first flat block of each entry; first[n] = total (< 2^31)
};

template <class Job>
struct JobSlot {
    Job job;
    dim3 grid;  // the volume's own grid for this stage
};

__device__ __forceinline__ int worklist_entry(const WorkList& wl, unsigned b)
{
    int lo = 0, hi = wl.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (wl.first[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class Job, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    worklist_kernel(const JobSlot<Job>* __restrict__ slots, const __grid_constant__ WorkList wl)
{
    // 32-bit index arithmetic only: a 64-bit division is a long software sequence, which
    // every thread of the block would run
    const unsigned b = blockIdx.x;
    const int e = worklist_entry(wl, b);
    const JobSlot<Job>* s = slots + wl.vol[e];
    const dim3 g = s->grid;
    const unsigned r = b - wl.first[e];
    const unsigned q = r / g.x;
    const uint3 bi = make_uint3(r - q * g.x, q % g.y, q / g.y);
    s->job(bi, g, wl.flag[e]);
}

// ------------------------------------------------------------------ stage jobs
// Each holds one volume's arguments of a kernel of kernels.cuh and runs its body.

template <typename T, int N, int S, int TKT, int RKR, class Ld, class St, int RG>
struct ConvKWinJob {
    Ld ld;
    St st;
    Dims d;
    const T* taps;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        conv_k_win_body<T, N, S, TKT, RKR, Ld, St, RG>(b, g, ld, st, d, taps);
    }
};

template <typename T, int N, int AXIS, int S, int TW, int TY, int R, class Ld, class St>
struct ConvSWinJob {
    Ld ld;
    St st;
    Dims d;
    const T* taps;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        conv_s_win_body<T, N, AXIS, S, TW, TY, R, Ld, St>(b, g, ld, st, d, taps);
    }
};

template <int S, int JB, int D, int U, int MINB>
struct FitMarchJob {
    const float4* in;
    float2* out;
    float* f1;
    float* f2;
    Dims d;
    TapPairs<S> tp;
    float l1, l2;
    int chunk;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        conv_i_fit_march_body<S, JB, D, U, MINB>(b, g, in, out, f1, f2, d, tp, l1, l2, chunk);
    }
};

template <typename T, int S, int TW, int TY, int TA>
struct FitWinJob {
    const Vec<T, 4>* in;
    Vec<T, 2>* out;
    T* f1;
    T* f2;
    Dims d;
    const T* taps;
    T l1, l2;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        conv_i_fit_win_body<T, S, TW, TY, TA>(b, g, in, out, f1, f2, d, taps, l1, l2);
    }
};

// A half-sweep of the residual solve (no own value, omega 1).
template <typename T, int NI, bool NEU, int MINB>
struct RbHalfJob {
    T* U;
    const T* B;
    Dims d;
    GsCoef<T> c;
    int color, reverse;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        rb_half_vec_body<T, NI, false, NEU, MINB>(b, g, U, B, d, c, color, 0, T(1), reverse);
    }
};

// flag: this check also sums b_eff^2 (the first check of a solve)
template <typename T, int NI>
struct RbResidualJob {
    const T* U;
    const T* B;
    Dims d;
    GsCoef<T> c;
    double* part;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int flag) const
    {
        rb_residual_vec_body<T, NI>(b, g, U, B, d, c, part, flag);
    }
};

template <typename T, int NI, bool VEC>
struct ClampTolJob {
    const T* u;
    T* phi;
    T* u_out;
    Dims d;
    T a0, b0;
    double* part;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        if constexpr (VEC) clamp_tol_vec_body<T, true, NI>(b, g, u, phi, u_out, d, a0, b0, part);
        else clamp_tol_body<T, true, NI>(b, g, u, phi, u_out, d, a0, b0, part);
    }
};

template <typename T, int NI, bool VEC>
struct BregmanJob {
    const T* phi;
    T* b3;
    T* dmb;
    const T* g3;
    Dims d;
    double hx, hy, hz;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        if constexpr (VEC) bregman_vec_body<T, NI>(b, g, phi, b3, dmb, g3, d, hx, hy, hz);
        else bregman_body<T, NI>(b, g, phi, b3, dmb, g3, d, hx, hy, hz);
    }
};

template <typename T, int NI, bool VEC>
struct DivJob {
    const T* v;
    T* out;
    Dims d;
    double hx, hy, hz;
    __device__ __forceinline__ void operator()(uint3 b, dim3 g, int) const
    {
        if constexpr (VEC) div_vec_body<T, NI>(b, g, v, out, d, hx, hy, hz);
        else div_body<T>(b, g, v, out, d, hx, hy, hz);
    }
};

// The fold of one volume's partials into its control block (finalize_sums_kernel per
// volume, in the same order): block e of the launch serves entry e.
struct FinalizeJob {
    const double* part;
    long long nblocks;
    double* sums;
};

static __global__ void __launch_bounds__(kFinThreads)
    finalize_worklist_kernel(const FinalizeJob* __restrict__ jobs, const __grid_constant__ WorkList wl,
                             int nvals, int slot)
{
    const FinalizeJob j = jobs[wl.vol[blockIdx.x]];
    finalize_sums_body(j.part, j.nblocks, nvals + wl.flag[blockIdx.x], j.sums, slot);
}

}  // namespace im3d

// conv_tma.cuh -- the first pass of the fitting stage for FP32 volumes on sm_100a, with
// its rows moved by the Tensor Memory Accelerator: the Heaviside of phi
// (rsfe_splitbregman_imp.hxx:174-192) and the Gaussian along k of the four fields
// H*u0, H, (1-H)*u0, 1-H (the k factor of the separable filter that replaces
// acyclic_fftw_convolution, convolution_imp.hxx:535-653). Rows of up to 256 cells (one
// TMA box); longer rows take conv_k_win_kernel.
//
// Each block is persistent and takes row blocks of RB rows (one warp per row) in turn:
//   * one thread loads the rows of phi and u0 with 2-D TMA boxes into a two-stage ring,
//     two row blocks ahead, each stage completing on its own mbarrier (bounded waits);
//   * every warp turns its row into the four fields, with the halo of the filter (zero or
//     periodic), in two rows of shared memory that hold the fields in pairs,
//     (H*u0, H) and ((1-H)*u0, 1-H);
//   * every lane convolves 8 consecutive cells of both pairs with the paired FP32
//     instructions of sm_100 (__fadd2_rn, __ffma2_rn, __fmul2_rn: per component the same
//     operations as window_conv of conv_k_win_kernel, so the sums are bit-identical at
//     half the instructions) and writes them into an output tile laid out in the
//     128-byte swizzle of the TMA;
//   * one thread stores the tile with a 3-D TMA box while the next row block is cooked.
// Shared-memory reads are free of bank conflicts: the pair rows hold a pad chunk after
// every 4, so that the lanes' windows (4 chunks apart) start 5 chunks apart, and the
// output tile's swizzle spreads the lanes' cells the same way.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_sm100.cuh"

namespace im3d {

struct HeavTmaArgs {
    Dims d;
    const float* taps;  // S + 1 taps, centre last (load_taps)
    float center, inv_eps;
    int KB;             // cells of the box along k: nz rounded up to a multiple of 16, <= 256
    long long nrb;      // row blocks of RB rows
    int* err;           // set to 1 when a wait for a load timed out
};

template <int RB, int S>
struct HeavTmaLayout {
    static constexpr int SP = (S + 3) & ~3;  // halo rounded up to whole 16-byte chunks
    // positions of one cooked row: halo, row, halo, rounded up to 32
    __host__ __device__ static int cw(int KB) { return (KB + 2 * SP + 31) & ~31; }
    // float2 of one pair row: cw positions, one pad chunk per 4 (pair_slot)
    __host__ __device__ static int pair_row(int KB) { return cw(KB) / 4 * 5; }
    __host__ __device__ static size_t out_bytes(int KB) { return (size_t)RB * KB * 16; }
    __host__ __device__ static size_t raw_bytes(int KB) { return (size_t)4 * RB * KB * 4; }  // 2 stages x 2 fields
    __host__ __device__ static size_t cooked_bytes(int KB) { return (size_t)2 * RB * pair_row(KB) * 8; }
    // + 1024 for aligning the dynamic buffer, + 2 mbarriers
    __host__ __device__ static size_t total(int KB)
    {
        return 1024 + out_bytes(KB) + raw_bytes(KB) + cooked_bytes(KB) + 16;
    }
};

// Where logical chunk c (two positions of a field pair) of a cooked pair row lives: one
// pad chunk after every 4, so that lanes 4 chunks apart land 5 chunks apart, on distinct
// banks, and every chunk of a lane's window is at a constant offset from the lane's first.
__host__ __device__ __forceinline__ int pair_slot(int c)
{
    return c + (c >> 2);
}

template <int RB, int S>
__global__ void __launch_bounds__(RB * 32, 2)
    conv_k_heav_tma_kernel(const __grid_constant__ CUtensorMap mphi, const __grid_constant__ CUtensorMap mu0,
                           const __grid_constant__ CUtensorMap mout, const HeavTmaArgs a)
{
    constexpr int R = 8;  // cells per lane: one 128-byte row of the output tile
    typedef HeavTmaLayout<RB, S> L;
    constexpr int SP = L::SP;
    constexpr int XW = R + 2 * SP;  // positions of one lane's window, whole chunks
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int KB = a.KB, nz = a.d.nz;
    const int PR = L::pair_row(KB);
    const int box_f = RB * KB;  // floats of one input box
    unsigned char* outs = base;
    float* raw = reinterpret_cast<float*>(base + L::out_bytes(KB));
    float2* ck = reinterpret_cast<float2*>(raw + 4 * box_f);
    uint64_t* bars = reinterpret_cast<uint64_t*>(ck + 2 * RB * PR);
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t stage_bytes = 2u * (uint32_t)box_f * 4u;
    if (tid == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        tc::fence_mbar_init();
        s_fail = 0;
    }
    __syncthreads();
    // input box of stage st, field f (0 phi, 1 u0)
    auto in_box = [&](int st, int f) { return raw + (st * 2 + f) * box_f; };
    const long long G = gridDim.x;
    // thread 0's record, one bit per stage: loads in flight, and the parity they complete
    uint32_t inflight = 0u, ph = 0u;
    auto issue = [&](long long rb, int st) {
        tc::mbar_arrive_expect_tx(&bars[st], stage_bytes);
        const int y = (int)(rb * RB);
        tc::tma_load_2d(in_box(st, 0), &mphi, &bars[st], 0, y);
        tc::tma_load_2d(in_box(st, 1), &mu0, &bars[st], 0, y);
        inflight |= 1u << st;
    };
    long long rb = blockIdx.x;
    if (tid == 0) {
        if (rb < a.nrb) issue(rb, 0);
        if (rb + G < a.nrb) issue(rb + G, 1);
    }
    float w[S + 1];
    load_taps<float, S>(a.taps, w);
    float2 w2[S + 1];
#pragma unroll
    for (int t = 0; t <= S; ++t) w2[t] = make_float2(w[t], w[t]);
    // this warp's two cooked rows: (H*u0, H) and ((1-H)*u0, 1-H) per position
    float2* myck[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) myck[q] = ck + (q * RB + warp) * PR;
    const int lim = nz + 2 * SP;

    for (int it = 0; rb < a.nrb; rb += G, ++it) {
        const int st = it & 1;
        if (tc::mbar_wait(&bars[st], (uint32_t)((it >> 1) & 1))) {
            if (tid == 0) {
                inflight &= ~(1u << st);
                ph ^= 1u << st;
            }
        } else {
            s_fail = 1;
        }
        // the four fields of this warp's row, halo included (positions p = k + SP), CU
        // positions per lane at a time: their reads first, then the arithmetic
        {
            constexpr int CU = 4;
            const float* rp = in_box(st, 0) + warp * KB;
            const float* ru = in_box(st, 1) + warp * KB;
            for (int p0 = lane; p0 < lim; p0 += 32 * CU) {
                float ph_[CU], u_[CU];
                bool in_[CU];
#pragma unroll
                for (int e = 0; e < CU; ++e) {
                    const int p = p0 + 32 * e;
                    int kk = 0;
                    in_[e] = p < lim && a.d.halo(p - SP, nz, kk);
                    ph_[e] = in_[e] ? rp[kk] : 0.f;
                    u_[e] = in_[e] ? ru[kk] : 0.f;
                }
#pragma unroll
                for (int e = 0; e < CU; ++e) {
                    const int p = p0 + 32 * e;
                    if (p < lim) {
                        float H, Hb;
                        heaviside_pair<float>(ph_[e], a.center, a.inv_eps, H, Hb);
                        if (!in_[e]) H = Hb = 0.f;
                        const int x = (pair_slot(p >> 1) << 1) | (p & 1);
                        myck[0][x] = make_float2(H * u_[e], H);
                        myck[1][x] = make_float2(Hb * u_[e], Hb);
                    }
                }
            }
        }
        // the previous row block's store has read the output tile
        if (tid == 0) tc::bulk_wait_read0();
        __syncthreads();
        if (s_fail) break;
        // the input stage is free: load the row block after next into it
        if (tid == 0) {
            tc::fence_proxy_async_smem();
            if (rb + 2 * G < a.nrb) issue(rb + 2 * G, st);
        }
        __syncwarp();
        const int k0 = lane * R;
        if (k0 < nz) {
            // the 8 cells form one 128-byte row g of the swizzled tile (nz a multiple of 8),
            // its 16-byte chunks XOR-ed with g
            const int g = (warp * KB + k0) >> 3;
            unsigned char* orow = outs + (size_t)g * 128;
            const int gx = g & 7;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                // the window of positions k0 .. k0 + XW - 1 of field pair q, two per chunk,
                // at constant offsets from the lane's first chunk
                const float2* win0 = myck[q] + (pair_slot(k0 >> 1) << 1);
                float2 xa[XW];
#pragma unroll
                for (int t = 0; t < XW / 2; ++t) {
                    const float4 v4 = *reinterpret_cast<const float4*>(win0 + ((t + (t >> 2)) << 1));
                    xa[2 * t] = make_float2(v4.x, v4.y);
                    xa[2 * t + 1] = make_float2(v4.z, v4.w);
                }
                // window_conv of both fields at once: the same operations per component
                float2 acc[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    acc[r] = __fmul2_rn(w2[S], xa[r + SP]);
#pragma unroll
                    for (int t = 0; t < S; ++t)
                        acc[r] = __ffma2_rn(w2[t], __fadd2_rn(xa[r + t + SP - S], xa[r + 2 * S - t + SP - S]), acc[r]);
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
                    *reinterpret_cast<float2*>(orow + ((r ^ gx) << 4) + q * 8) = acc[r];
            }
        }
        // the tile's writes become visible to the TMA before the store is issued
        tc::fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::tma_store_3d(&mout, outs, 0, 0, (int)(rb * RB));
            tc::bulk_commit();
        }
    }
    if (tid == 0) {
        tc::bulk_wait0();
        if (s_fail) {
            atomicExch(a.err, 1);
            // let the loads still in flight land before the block exits
            for (int st = 0; st < 2; ++st)
                if ((inflight >> st) & 1u) tc::mbar_wait(&bars[st], (ph >> st) & 1u, 1000000000ull);
        }
    }
    __syncthreads();
}

}  // namespace im3d

// unet_kernels.cuh -- kernels of the learned Poisson warm start: a 3-level 3-D U-Net
// (16/32/64 channels, 3x3x3 convolutions) on BF16 channels-last activations.
//
// Tensors: voxel-major, channels fastest ("channels-last"), BF16, with a channel pitch
// (channels stored per voxel) and a channel offset, so that a decoder's concatenated
// input [upsampled | skip] is one tensor whose halves two producers write. Voxel index
// ((s * D + z) * H + y) * W + x for sample s: the reference's image3d order (i, j, k)
// with k contiguous.
//
// The 3x3x3 convolutions (forward, and the data gradient as a forward convolution with
// the flipped, transposed filter) run as implicit GEMMs on the tensor cores
// (conv3_tc_kernel): a CTA stages, by TMA, the halo block of one output tile -- 3
// planes x (TH + 2) rows x (TW + 2) columns of every 8-channel chunk, "chunk-planar"
// (see tc_sm100.cuh) -- with the out-of-volume halo zero-filled by the TMA unit, which
// is the convolution's zero padding. Each of the 27 taps is then the same block read
// at a row offset, so the A operand of every tap is a descriptor into one staged block:
// no im2col buffer, one HBM read of the block per tile. M = 128 output positions of the
// padded tile, N = the output channels of the launch (16 or 32), K = 16 input channels
// per instruction; the FP32 accumulators live in TMEM and are drained by 4 warps
// (bias + ReLU or the ReLU mask of the data gradient, BF16 store). The weight gradient
// (wgrad_tc_kernel) reads the same staged blocks with MN-major descriptors: M = the
// output channels (64 rows, padded), N = the input channels, K = 16 voxel positions,
// accumulated in TMEM over all tiles of a CTA and added to the FP32 gradient once.
// Pooling, the 2x2x2 transposed convolutions, the 1x1 output layer, the loss and Adam
// are small SIMT kernels.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdint>

#include "tc_sm100.cuh"

namespace im3d {
namespace unet {

typedef uint16_t bf16_t;  // raw BF16 bits in global memory

__device__ __forceinline__ float bf(bf16_t v) { return __uint_as_float(((uint32_t)v) << 16); }
__device__ __forceinline__ bf16_t to_bf(float v)
{
    return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// Geometry of one tiled 3x3x3 convolution launch (host-filled).
struct ConvGeom {
    int D, H, W;     // volume of one sample
    int nsamp;       // samples
    int TH, TW;      // tile rows (along H) and columns (along W; TW divides W, TW <= 128)
    int tiles_w, tiles_h;
    long long ntiles;  // nsamp * D * tiles_h * tiles_w
    int mtiles;      // 128-position MMA tiles per CTA tile
    int reg_bytes;   // one chunk region of the staged block (multiple of 1024)
    int tmem_cols;   // TMEM columns allocated (power of two >= 32)
};

// Position of M-tile m's first row in the padded tile plane (pitch P = TW + 2): one
// interior row per M-tile when TW == 128, else 128 consecutive positions starting at
// the first interior one (rows of the tile and the 2 halo columns between them).
__device__ __forceinline__ int mtile_start(const ConvGeom& g, int m)
{
    const int P = g.TW + 2;
    return g.TW == 128 ? (m + 1) * P + 1 : P + 1 + 128 * m;
}

struct ConvArgs {
    ConvGeom g;
    const bf16_t* wpk;     // [N-block][27][CIN/8][NOUT][8] BF16 filter of this launch
    const float* bias;     // output channels' bias (MODE 0, 2) or NULL
    void* out;             // BF16 (MODE 0, 1) or FP32 (MODE 2) channels-last
    int out_pitch, out_coff;
    const bf16_t* mask;    // MODE 1: result multiplied by (mask > 0), or NULL
    int mask_pitch, mask_coff;
    int in_coff;           // first input channel (a multiple of 8)
    int* err;              // raised when a wait gives up
};

enum { CONV_BIAS_RELU = 0, CONV_MASK = 1, CONV_BIAS_F32 = 2 };

constexpr int kGuardBytes = 8192;  // after the staged block: the last M-tile's overreach

__host__ __device__ constexpr int align_up(int x, int a) { return (x + a - 1) / a * a; }

template <int CIN, int NOUT>
__host__ __device__ constexpr int conv_weight_bytes()
{
    return 27 * (CIN / 8) * NOUT * 16;
}

// dynamic shared memory of conv3_tc_kernel<CIN, NOUT>
template <int CIN, int NOUT>
__host__ __device__ inline int conv_smem_bytes(int reg_bytes)
{
    return align_up(conv_weight_bytes<CIN, NOUT>(), 1024) + (CIN / 8) * reg_bytes + kGuardBytes + 64 + 1024;
}

template <int CIN, int NOUT, int MODE>
__global__ void __launch_bounds__(128, 1) conv3_tc_kernel(const __grid_constant__ CUtensorMap xmap, ConvArgs a)
{
    constexpr int KC = CIN / 8;
    constexpr int WB = conv_weight_bytes<CIN, NOUT>();
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const ConvGeom& g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5;
    unsigned char* wsm = smem;
    unsigned char* act = smem + align_up(WB, 1024);
    uint64_t* bars = reinterpret_cast<uint64_t*>(act + KC * g.reg_bytes + kGuardBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    __shared__ int s_fail;
    const int nb = blockIdx.y;  // block of NOUT output channels

    {
        const uint4* src = reinterpret_cast<const uint4*>(a.wpk + (size_t)nb * (WB / 2));
        uint4* dst = reinterpret_cast<uint4*>(wsm);
        for (int q = tid; q < WB / 16; q += blockDim.x) dst[q] = src[q];
    }
    if (tid == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        tc::fence_mbar_init();
        s_fail = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(tslot, (uint32_t)g.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::fence_proxy_async_smem();
    tc::tc_fence_before_sync();
    __syncthreads();
    tc::tc_fence_after_sync();
    const uint32_t tmem = *tslot;

    const int P = g.TW + 2;
    const int plane = (g.TH + 2) * P;
    const uint32_t box_bytes = 16u * (uint32_t)plane * 3u;
    const uint32_t idesc = tc::idesc_bf16(128, NOUT, false, false);
    const uint32_t act_s = tc::smem_u32(act), w_s = tc::smem_u32(wsm);
    uint32_t ph_ld = 0, ph_mma = 0;
    bool loads_in_flight = false;

    for (long long tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
        long long r = tile;
        const int tw = (int)(r % g.tiles_w);
        r /= g.tiles_w;
        const int th = (int)(r % g.tiles_h);
        r /= g.tiles_h;
        const int z = (int)(r % g.D);
        const int s = (int)(r / g.D);
        const int w0 = tw * g.TW, h0 = th * g.TH;
        if (tid == 0) {
            tc::mbar_arrive_expect_tx(&bars[0], KC * box_bytes);
            for (int c = 0; c < KC; ++c)
                tc::tma_load_5d(act + c * g.reg_bytes, &xmap, &bars[0], a.in_coff + 8 * c, w0 - 1, h0 - 1, z - 1, s);
        }
        loads_in_flight = true;
        if (!tc::mbar_wait(&bars[0], ph_ld)) s_fail = 1;
        ph_ld ^= 1;
        __syncthreads();
        if (s_fail) break;
        loads_in_flight = false;
        tc::tc_fence_after_sync();
        if (tid == 0) {
            for (int m = 0; m < g.mtiles; ++m) {
                const int qs = mtile_start(g, m);
                for (int t = 0; t < 27; ++t) {
                    const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
                    const int q = dz * plane + qs + (dy - 1) * P + (dx - 1);
#pragma unroll
                    for (int ks = 0; ks < KC / 2; ++ks) {
                        const uint64_t ad = tc::smem_desc(act_s + (uint32_t)(2 * ks * g.reg_bytes + q * 16),
                                                          (uint32_t)g.reg_bytes, 128);
                        const uint64_t bd = tc::smem_desc(w_s + (uint32_t)((t * KC + 2 * ks) * NOUT * 16),
                                                          (uint32_t)(NOUT * 16), 128);
                        tc::mma_bf16(tmem + (uint32_t)(m * NOUT), ad, bd, idesc, (t | ks) != 0);
                    }
                }
            }
            tc::mma_commit(&bars[1]);
        }
        if (!tc::mbar_wait(&bars[1], ph_mma)) s_fail = 1;
        ph_mma ^= 1;
        __syncthreads();
        if (s_fail) break;
        tc::tc_fence_after_sync();
        // epilogue: accumulator row tid of every M-tile
        for (int m = 0; m < g.mtiles; ++m) {
            const int q = mtile_start(g, m) + tid;
            const int py = q / P, px = q - (q / P) * P;
            float v[NOUT];
#pragma unroll
            for (int c0 = 0; c0 < NOUT; c0 += 16) {
                float part[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * NOUT + c0), part);
#pragma unroll
                for (int u = 0; u < 16; ++u) v[c0 + u] = part[u];
            }
            const int y = h0 + py - 1, x = w0 + px - 1;
            if (py < 1 || py > g.TH || px < 1 || px > g.TW || y >= g.H) continue;
            const long long vox = (((long long)s * g.D + z) * g.H + y) * g.W + x;
            const int c_first = nb * NOUT;
            if (MODE == CONV_BIAS_F32) {
                float* o = reinterpret_cast<float*>(a.out) + vox * a.out_pitch + a.out_coff + c_first;
#pragma unroll
                for (int n = 0; n < NOUT; ++n) o[n] = v[n] + (a.bias ? a.bias[c_first + n] : 0.f);
                continue;
            }
            if (MODE == CONV_BIAS_RELU) {
#pragma unroll
                for (int n = 0; n < NOUT; ++n) v[n] = fmaxf(v[n] + a.bias[c_first + n], 0.f);
            } else if (a.mask) {
                const uint4* mp = reinterpret_cast<const uint4*>(a.mask + vox * a.mask_pitch + a.mask_coff + c_first);
#pragma unroll
                for (int n8 = 0; n8 < NOUT / 8; ++n8) {
                    const uint4 mv = mp[n8];
                    const uint32_t w4[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        if (!(bf((bf16_t)(w4[u] & 0xffff)) > 0.f)) v[n8 * 8 + 2 * u] = 0.f;
                        if (!(bf((bf16_t)(w4[u] >> 16)) > 0.f)) v[n8 * 8 + 2 * u + 1] = 0.f;
                    }
                }
            }
            uint4* o = reinterpret_cast<uint4*>(reinterpret_cast<bf16_t*>(a.out) + vox * a.out_pitch + a.out_coff + c_first);
#pragma unroll
            for (int n8 = 0; n8 < NOUT / 8; ++n8) {
                uint4 pk;
                pk.x = (uint32_t)to_bf(v[n8 * 8 + 0]) | ((uint32_t)to_bf(v[n8 * 8 + 1]) << 16);
                pk.y = (uint32_t)to_bf(v[n8 * 8 + 2]) | ((uint32_t)to_bf(v[n8 * 8 + 3]) << 16);
                pk.z = (uint32_t)to_bf(v[n8 * 8 + 4]) | ((uint32_t)to_bf(v[n8 * 8 + 5]) << 16);
                pk.w = (uint32_t)to_bf(v[n8 * 8 + 6]) | ((uint32_t)to_bf(v[n8 * 8 + 7]) << 16);
                o[n8] = pk;
            }
        }
        tc::tc_fence_before_sync();
        __syncthreads();
    }
    if (s_fail) {
        if (tid == 0) atomicExch(a.err, 1);
        // let the copies that may still be in flight land before the block exits
        if (loads_in_flight) tc::mbar_wait(&bars[0], ph_ld ^ 1, 1000000000ull);
        __syncthreads();
    }
    tc::tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, (uint32_t)g.tmem_cols);
}

// ---------------------------------------------------------------- weight gradient
struct WgradArgs {
    ConvGeom g;      // the forward launch's tiling (TW multiple of 16)
    int zcoff;       // first channel of dZ in its tensor
    int xcoff;       // first input channel in X's tensor
    int tap0, ntaps; // taps of this launch's blockIdx.x group: tap0 + blockIdx.x * ntaps ...
    int cout;        // output channels (rows of dZ used)
    float* dw;       // FP32 gradient [cout][CIN][27] (the parameter layout), accumulated with atomics
    int* err;
};

template <int CIN>
__host__ __device__ inline int wgrad_smem_bytes(int cout, int reg_z, int reg_x)
{
    return (cout / 8) * reg_z + (CIN / 8) * reg_x + kGuardBytes + 64 + 1024;
}

// grid.x: tap groups of a.ntaps taps; grid.y: splits of the tile list.
template <int CIN>
__global__ void __launch_bounds__(128, 1) wgrad_tc_kernel(const __grid_constant__ CUtensorMap xmap,
                                                         const __grid_constant__ CUtensorMap zmap, WgradArgs a,
                                                         int reg_z, int reg_x)
{
    constexpr int KC = CIN / 8;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const ConvGeom& g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int zc = a.cout / 8;
    unsigned char* zblk = smem;                    // dZ: zc regions of one padded plane
    unsigned char* xblk = smem + zc * reg_z;       // X: KC regions of 3 padded planes
    uint64_t* bars = reinterpret_cast<uint64_t*>(xblk + KC * reg_x + kGuardBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    __shared__ int s_fail;
    const int t_first = a.tap0 + blockIdx.x * a.ntaps;
    const int nt = min(a.ntaps, 27 - t_first);
    if (tid == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        tc::fence_mbar_init();
        s_fail = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(tslot, 512u);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before_sync();
    __syncthreads();
    tc::tc_fence_after_sync();
    const uint32_t tmem = *tslot;
    const int P = g.TW + 2;
    const int plane = (g.TH + 2) * P;
    const uint32_t zbox = 16u * (uint32_t)plane, xbox = 16u * (uint32_t)plane * 3u;
    const uint32_t idesc = tc::idesc_bf16(64, CIN, true, true);
    const uint32_t zs = tc::smem_u32(zblk), xs = tc::smem_u32(xblk);
    uint32_t ph_ld = 0, ph_mma = 0;
    bool first = true, loads_in_flight = false;
    for (long long tile = blockIdx.y; tile < g.ntiles && nt > 0; tile += gridDim.y) {
        long long r = tile;
        const int tw = (int)(r % g.tiles_w);
        r /= g.tiles_w;
        const int th = (int)(r % g.tiles_h);
        r /= g.tiles_h;
        const int z = (int)(r % g.D);
        const int s = (int)(r / g.D);
        const int w0 = tw * g.TW, h0 = th * g.TH;
        const int rows = min(g.TH, g.H - h0);
        if (tid == 0) {
            tc::mbar_arrive_expect_tx(&bars[0], zc * zbox + KC * xbox);
            for (int c = 0; c < zc; ++c)
                tc::tma_load_5d(zblk + c * reg_z, &zmap, &bars[0], a.zcoff + 8 * c, w0 - 1, h0 - 1, z, s);
            for (int c = 0; c < KC; ++c)
                tc::tma_load_5d(xblk + c * reg_x, &xmap, &bars[0], a.xcoff + 8 * c, w0 - 1, h0 - 1, z - 1, s);
        }
        loads_in_flight = true;
        if (!tc::mbar_wait(&bars[0], ph_ld)) s_fail = 1;
        ph_ld ^= 1;
        __syncthreads();
        if (s_fail) break;
        loads_in_flight = false;
        tc::tc_fence_after_sync();
        if (tid == 0) {
            for (int ti = 0; ti < nt; ++ti) {
                const int t = t_first + ti;
                const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
                for (int row = 0; row < rows; ++row) {
                    const int q0 = (row + 1) * P + 1;
                    for (int k0 = 0; k0 < g.TW; k0 += 16) {
                        const int qz = q0 + k0;
                        const int qx = dz * plane + qz + (dy - 1) * P + (dx - 1);
                        const uint64_t ad = tc::smem_desc(zs + (uint32_t)(qz * 16), 128, (uint32_t)reg_z);
                        const uint64_t bd = tc::smem_desc(xs + (uint32_t)(qx * 16), 128, (uint32_t)reg_x);
                        tc::mma_bf16(tmem + (uint32_t)(ti * CIN), ad, bd, idesc, first && row == 0 && k0 == 0 ? 0u : 1u);
                    }
                }
            }
            tc::mma_commit(&bars[1]);
        }
        first = false;
        if (!tc::mbar_wait(&bars[1], ph_mma)) s_fail = 1;
        ph_mma ^= 1;
        tc::tc_fence_before_sync();
        __syncthreads();
        if (s_fail) break;
    }
    if (!s_fail && !first) {
        tc::tc_fence_after_sync();
        // M = 64 accumulator rows: row r sits in TMEM lane (r % 16) + 32 (r / 16)
        const int co = warp * 16 + lane;
        for (int ti = 0; ti < nt; ++ti) {
#pragma unroll
            for (int c0 = 0; c0 < CIN; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ti * CIN + c0), v);
                if (lane < 16 && co < a.cout) {
                    // the parameter layout [cout][CIN][27]
                    float* d = a.dw + ((size_t)co * CIN + c0) * 27 + (t_first + ti);
#pragma unroll
                    for (int u = 0; u < 16; ++u) atomicAdd(d + u * 27, v[u]);
                }
            }
        }
    }
    if (s_fail) {
        if (tid == 0) atomicExch(a.err, 2);
        if (loads_in_flight) tc::mbar_wait(&bars[0], ph_ld ^ 1, 1000000000ull);
        __syncthreads();
    }
    tc::tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512u);
}

// ------------------------------------------------------------------ SIMT kernels
// sum over voxels of dZ[v][c] (c < C) into db[c]
__global__ void bias_grad_kernel(const bf16_t* __restrict__ dz, int pitch, int coff, int C, long long n, float* db)
{
    __shared__ float acc[64];
    for (int c = threadIdx.x; c < 64; c += blockDim.x) acc[c] = 0.f;
    __syncthreads();
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    float s = 0.f;
    for (long long v = (long long)blockIdx.x * lanes + threadIdx.x / C; v < n; v += (long long)gridDim.x * lanes)
        if (threadIdx.x < lanes * C) s += bf(dz[v * pitch + coff + c]);
    if (threadIdx.x < lanes * C) atomicAdd(&acc[c], s);
    __syncthreads();
    for (int q = threadIdx.x; q < C; q += blockDim.x) atomicAdd(db + q, acc[q]);
}

// 2x2x2 max pooling of channels [coff, coff + C) of `in` (pitch ip) into out [n/8][C]
// (pitch C); idx receives the argmax child (0..7) per output value.
__global__ void pool_fwd_kernel(const bf16_t* __restrict__ in, int ip, int coff, int C, int D, int H, int W,
                                int nsamp, bf16_t* __restrict__ out, uint8_t* __restrict__ idx)
{
    const int D2 = D / 2, H2 = H / 2, W2 = W / 2;
    const long long total = (long long)nsamp * D2 * H2 * W2 * C;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        long long p = e / C;
        const int x = (int)(p % W2);
        long long r = p / W2;
        const int y = (int)(r % H2);
        r /= H2;
        const int z = (int)(r % D2);
        const int s = (int)(r / D2);
        float best = -3.0e38f;
        int bi = 0;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const long long v = (((long long)s * D + 2 * z + (o >> 2)) * H + 2 * y + ((o >> 1) & 1)) * W + 2 * x + (o & 1);
            const float f = bf(in[v * ip + coff + c]);
            if (f > best) {
                best = f;
                bi = o;
            }
        }
        out[e] = to_bf(best);
        idx[e] = (uint8_t)bi;
    }
}

// Gradient of the pooled skip tensor: for every child cell of a pooled cell,
//   g[child] = (g_skip[child] + (child == argmax ? g_pool : 0)) * (act[child] > 0)
// (act = the pooled ReLU output). g may alias g_skip (same pitch and offset).
__global__ void pool_bwd_kernel(const bf16_t* __restrict__ gpool, const uint8_t* __restrict__ idx, int C, int D,
                                int H, int W, int nsamp, const bf16_t* gskip, int sp, int soff,
                                const bf16_t* __restrict__ act, int ap, int aoff, bf16_t* g, int gp, int goff)
{
    const int D2 = D / 2, H2 = H / 2, W2 = W / 2;
    const long long total = (long long)nsamp * D2 * H2 * W2 * C;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        long long p = e / C;
        const int x = (int)(p % W2);
        long long r = p / W2;
        const int y = (int)(r % H2);
        r /= H2;
        const int z = (int)(r % D2);
        const int s = (int)(r / D2);
        const float gp_v = bf(gpool[e]);
        const int bi = idx[e];
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const long long v = (((long long)s * D + 2 * z + (o >> 2)) * H + 2 * y + ((o >> 1) & 1)) * W + 2 * x + (o & 1);
            float val = gskip ? bf(gskip[v * sp + soff + c]) : 0.f;
            if (o == bi) val += gp_v;
            if (!(bf(act[v * ap + aoff + c]) > 0.f)) val = 0.f;
            g[v * gp + goff + c] = to_bf(val);
        }
    }
}

// 2x2x2 stride-2 transposed convolution: out[child(p, o)][co] = b[co] + sum_ci
// in[p][ci] U[o][ci][co]. One thread per output voxel; U (BF16) staged in shared memory.
template <int CI, int CO>
__global__ void __launch_bounds__(128) upconv_fwd_kernel(const bf16_t* __restrict__ in, const bf16_t* __restrict__ U,
                                                         const float* __restrict__ b, int D2, int H2, int W2, int nsamp,
                                                         bf16_t* out, int op, int ooff)
{
    __shared__ bf16_t us[8 * CI * CO];
    for (int q = threadIdx.x; q < 8 * CI * CO; q += blockDim.x) us[q] = U[q];
    __syncthreads();
    const int D = 2 * D2, H = 2 * H2, W = 2 * W2;
    const long long total = (long long)nsamp * D * H * W;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < total; v += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(v % W);
        long long r = v / W;
        const int y = (int)(r % H);
        r /= H;
        const int z = (int)(r % D);
        const int s = (int)(r / D);
        const int o = ((z & 1) << 2) | ((y & 1) << 1) | (x & 1);
        const long long p = (((long long)s * D2 + (z >> 1)) * H2 + (y >> 1)) * W2 + (x >> 1);
        float acc[CO];
#pragma unroll
        for (int co = 0; co < CO; ++co) acc[co] = b[co];
        const uint4* ip = reinterpret_cast<const uint4*>(in + p * CI);
        for (int c8 = 0; c8 < CI / 8; ++c8) {
            const uint4 w4 = ip[c8];
            const uint32_t u4[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                const float xv = bf((bf16_t)(h & 1 ? u4[h >> 1] >> 16 : u4[h >> 1] & 0xffff));
                const bf16_t* urow = us + (o * CI + c8 * 8 + h) * CO;
#pragma unroll
                for (int co = 0; co < CO; ++co) acc[co] = fmaf(xv, bf(urow[co]), acc[co]);
            }
        }
        uint4* dst = reinterpret_cast<uint4*>(out + v * op + ooff);
#pragma unroll
        for (int n8 = 0; n8 < CO / 8; ++n8) {
            uint4 pk;
            pk.x = (uint32_t)to_bf(acc[n8 * 8 + 0]) | ((uint32_t)to_bf(acc[n8 * 8 + 1]) << 16);
            pk.y = (uint32_t)to_bf(acc[n8 * 8 + 2]) | ((uint32_t)to_bf(acc[n8 * 8 + 3]) << 16);
            pk.z = (uint32_t)to_bf(acc[n8 * 8 + 4]) | ((uint32_t)to_bf(acc[n8 * 8 + 5]) << 16);
            pk.w = (uint32_t)to_bf(acc[n8 * 8 + 6]) | ((uint32_t)to_bf(acc[n8 * 8 + 7]) << 16);
            dst[n8] = pk;
        }
    }
}

// Data gradient of the transposed convolution, masked by the ReLU of its input:
//   g_in[p][ci] = (sum_{o, co} g_out[child(p, o)][co] U[o][ci][co]) * (in[p][ci] > 0)
template <int CI, int CO>
__global__ void __launch_bounds__(128) upconv_bwd_kernel(const bf16_t* __restrict__ gout, int gp, int goff,
                                                         const bf16_t* __restrict__ U, const bf16_t* __restrict__ in,
                                                         int D2, int H2, int W2, int nsamp, bf16_t* __restrict__ gin)
{
    __shared__ bf16_t us[8 * CI * CO];
    for (int q = threadIdx.x; q < 8 * CI * CO; q += blockDim.x) us[q] = U[q];
    __syncthreads();
    const int D = 2 * D2, H = 2 * H2, W = 2 * W2;
    const long long total = (long long)nsamp * D2 * H2 * W2;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < total; p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % W2);
        long long r = p / W2;
        const int y = (int)(r % H2);
        r /= H2;
        const int z = (int)(r % D2);
        const int s = (int)(r / D2);
        float acc[CI];
#pragma unroll
        for (int ci = 0; ci < CI; ++ci) acc[ci] = 0.f;
        for (int o = 0; o < 8; ++o) {
            const long long v = (((long long)s * D + 2 * z + (o >> 2)) * H + 2 * y + ((o >> 1) & 1)) * W + 2 * x + (o & 1);
            const bf16_t* gr = gout + v * gp + goff;
            for (int co = 0; co < CO; ++co) {
                const float gv = bf(gr[co]);
#pragma unroll
                for (int ci = 0; ci < CI; ++ci) acc[ci] = fmaf(gv, bf(us[(o * CI + ci) * CO + co]), acc[ci]);
            }
        }
#pragma unroll
        for (int ci = 0; ci < CI; ++ci) {
            const float m = bf(in[p * CI + ci]) > 0.f ? 1.f : 0.f;
            gin[p * CI + ci] = to_bf(acc[ci] * m);
        }
    }
}

// Weight and bias gradient of the transposed convolution:
//   dU[o][ci][co] += sum_p in[p][ci] g_out[child(p, o)][co],  db[co] += sum g_out[.][co].
// Each block folds a range of p in registers (one (o, ci, co) set per thread) and adds
// its partial sums once.
template <int CI, int CO>
__global__ void __launch_bounds__(256) upconv_wgrad_kernel(const bf16_t* __restrict__ in,
                                                           const bf16_t* __restrict__ gout, int gp, int goff,
                                                           int D2, int H2, int W2, int nsamp, float* dU, float* db)
{
    constexpr int NW = 8 * CI * CO;
    constexpr int PER = (NW + 255) / 256;
    constexpr int TP = 32;  // positions staged at once
    __shared__ float xs[TP][CI];
    __shared__ float gs[TP][8][CO];
    float acc[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) acc[u] = 0.f;
    float bacc = 0.f;
    const int D = 2 * D2, H = 2 * H2, W = 2 * W2;
    const long long total = (long long)nsamp * D2 * H2 * W2;
    for (long long p0 = (long long)blockIdx.x * TP; p0 < total; p0 += (long long)gridDim.x * TP) {
        __syncthreads();
        for (int q = threadIdx.x; q < TP * CI; q += blockDim.x) {
            const long long p = p0 + q / CI;
            xs[q / CI][q % CI] = p < total ? bf(in[p * CI + q % CI]) : 0.f;
        }
        for (int q = threadIdx.x; q < TP * 8 * CO; q += blockDim.x) {
            const int pi = q / (8 * CO), o = (q / CO) % 8, co = q % CO;
            const long long p = p0 + pi;
            float gv = 0.f;
            if (p < total) {
                const int x = (int)(p % W2);
                long long r = p / W2;
                const int y = (int)(r % H2);
                r /= H2;
                const int z = (int)(r % D2);
                const int s = (int)(r / D2);
                const long long v = (((long long)s * D + 2 * z + (o >> 2)) * H + 2 * y + ((o >> 1) & 1)) * W + 2 * x + (o & 1);
                gv = bf(gout[v * gp + goff + co]);
            }
            gs[pi][o][co] = gv;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int w = threadIdx.x + u * 256;
            if (w < NW) {
                const int o = w / (CI * CO), ci = (w / CO) % CI, co = w % CO;
                float sacc = 0.f;
                for (int pi = 0; pi < TP; ++pi) sacc = fmaf(xs[pi][ci], gs[pi][o][co], sacc);
                acc[u] += sacc;
            }
        }
        if (threadIdx.x < CO)
            for (int pi = 0; pi < TP; ++pi)
                for (int o = 0; o < 8; ++o) bacc += gs[pi][o][threadIdx.x];
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
        const int w = threadIdx.x + u * 256;
        if (w < NW) atomicAdd(dU + w, acc[u]);
    }
    if (threadIdx.x < CO) atomicAdd(db + threadIdx.x, bacc);
}

// 1x1 output layer, loss and its gradient in one pass:
//   y = b + sum_c w[c] d[v][c];  diff = y - target (on the cells with weight != 0);
//   loss += diff^2 * wt; dy = 2 diff wt / count;  g_d[v][c] = dy w[c] (d[v][c] > 0);
//   dw[c] += dy d[v][c], db += dy.
// target == NULL: forward only (y written, nothing else).
template <int C>
__global__ void __launch_bounds__(256) out_layer_kernel(const bf16_t* __restrict__ d, const float* __restrict__ w,
                                                        const float* __restrict__ b, long long n, float* y,
                                                        const float* __restrict__ target,
                                                        const float* __restrict__ wt, float inv_count,
                                                        bf16_t* __restrict__ gd, float* dw, float* db, double* loss)
{
    __shared__ float sw[C];
    __shared__ float sg[C + 1];
    __shared__ double sl;
    if (threadIdx.x < C) {
        sw[threadIdx.x] = w[threadIdx.x];
        sg[threadIdx.x] = 0.f;
    }
    if (threadIdx.x == 0) {
        sg[C] = 0.f;
        sl = 0.0;
    }
    __syncthreads();
    float gl[C];
#pragma unroll
    for (int c = 0; c < C; ++c) gl[c] = 0.f;
    float gb = 0.f;
    double ls = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        float dv[C];
        const uint4* dp = reinterpret_cast<const uint4*>(d + v * C);
#pragma unroll
        for (int c8 = 0; c8 < C / 8; ++c8) {
            const uint4 q = dp[c8];
            const uint32_t u4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int h = 0; h < 8; ++h) dv[c8 * 8 + h] = bf((bf16_t)(h & 1 ? u4[h >> 1] >> 16 : u4[h >> 1] & 0xffff));
        }
        float yv = b[0];
#pragma unroll
        for (int c = 0; c < C; ++c) yv = fmaf(sw[c], dv[c], yv);
        if (y) y[v] = yv;
        if (!target) continue;
        const float wv = wt ? wt[v] : 1.f;
        const float diff = (yv - target[v]) * wv;
        ls += (double)diff * diff;
        const float dy = 2.f * diff * wv * inv_count;
        gb += dy;
        bf16_t go[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            gl[c] = fmaf(dy, dv[c], gl[c]);
            go[c] = to_bf(dv[c] > 0.f ? dy * sw[c] : 0.f);
        }
        uint4* gp = reinterpret_cast<uint4*>(gd + v * C);
#pragma unroll
        for (int c8 = 0; c8 < C / 8; ++c8) {
            uint4 q;
            q.x = (uint32_t)go[c8 * 8 + 0] | ((uint32_t)go[c8 * 8 + 1] << 16);
            q.y = (uint32_t)go[c8 * 8 + 2] | ((uint32_t)go[c8 * 8 + 3] << 16);
            q.z = (uint32_t)go[c8 * 8 + 4] | ((uint32_t)go[c8 * 8 + 5] << 16);
            q.w = (uint32_t)go[c8 * 8 + 6] | ((uint32_t)go[c8 * 8 + 7] << 16);
            gp[c8] = q;
        }
    }
    if (!target) return;
#pragma unroll
    for (int c = 0; c < C; ++c) atomicAdd(&sg[c], gl[c]);
    atomicAdd(&sg[C], gb);
    atomicAdd(&sl, ls);
    __syncthreads();
    if (threadIdx.x < C) atomicAdd(dw + threadIdx.x, sg[threadIdx.x]);
    if (threadIdx.x == 0) {
        atomicAdd(db, sg[C]);
        atomicAdd(loss, sl);
    }
}

// Adam step on FP32 master parameters (bias-corrected learning rate lr_t).
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr_t, float b1, float b2, float eps,
                            float gscale)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const float gq = g[q] * gscale;
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        p[q] -= lr_t * mq / (sqrtf(vq) + eps);
    }
}

// FP32 filter W[co][ci][27] -> BF16 operand blocks of conv3_tc_kernel.
//   forward (transpose = 0): block nb holds output channels nb*NOUT.. : [27][CIN/8][NOUT][8]
//     with element (t, kc, n, e) = W[nb*NOUT + n][kc*8 + e][t]  (CIN = layer Cin)
//   data gradient (transpose = 1): the flipped, transposed filter, CIN = layer Cout,
//     outputs = layer Cin: element (t, kc, n, e) = W[kc*8 + e][nb*NOUT + n][26 - t]
__global__ void pack_filter_kernel(const float* __restrict__ W, int cout, int cin, int nout, int transpose,
                                   bf16_t* __restrict__ out)
{
    const int kcin = transpose ? cout : cin;   // K of the GEMM
    const int nall = transpose ? cin : cout;   // N of the GEMM
    const int nblocks = nall / nout;
    const long long total = (long long)nblocks * 27 * kcin * nout;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int el = (int)(e % 8);
        long long r = e / 8;
        const int n = (int)(r % nout);
        r /= nout;
        const int kc = (int)(r % (kcin / 8));
        r /= kcin / 8;
        const int t = (int)(r % 27);
        const int nb = (int)(r / 27);
        const int k = kc * 8 + el, nn = nb * nout + n;
        const float w = transpose ? W[((size_t)k * cin + nn) * 27 + (26 - t)] : W[((size_t)nn * cin + k) * 27 + t];
        out[e] = to_bf(w);
    }
}

__global__ void to_bf16_kernel(const float* __restrict__ src, bf16_t* __restrict__ dst, long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = to_bf(src[q]);
}

__global__ void zero_f32_kernel(float* p, long long n)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        p[q] = 0.f;
}

}  // namespace unet
}  // namespace im3d

// unet.cu -- host side of the learned Poisson warm start: the 3-level 3-D U-Net
// (16/32/64 channels) whose forward and backward passes run on the kernels of
// unet_kernels.cuh, its Adam training step, and the C ABI entry points im3d_unet_*
// and im3d_conv3d_bf16 of include/im3d_b200.h.
//
// Network (all convolutions 3x3x3, zero padding; ReLU after each):
//   x0 (4 fields, padded to 16 channels) -> e1a 16 -> e1b 16 = a        (level 1)
//   pool -> e2a 32 -> e2b 32 = b                                      (level 2)
//   pool -> e3a 64 -> e3b 64 = c                                      (level 3)
//   up2 = transposed conv 2x2x2 (64 -> 32);  [up2 | b] -> d2a 32 -> d2b 32 = d2
//   up1 = transposed conv 2x2x2 (32 -> 16);  [up1 | a] -> d1a 16 -> d1b 16 = d1
//   y = 1x1 conv (16 -> 1)
// The decoders' concatenations are single tensors ([n][32] at level 1, [n][64] at level
// 2) whose two halves are written by the transposed convolution and by the encoder.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/im3d_b200.h"
#include "internal.h"
#include "unet_kernels.cuh"

using namespace im3d::unet;

namespace {

#define UN_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                              \
            return e_ == cudaErrorMemoryAllocation ? IM3D_ERR_OOM : IM3D_ERR_CUDA;                  \
        }                                                                                          \
    } while (0)

#define UN_TRY(...)                   \
    do {                              \
        int s_ = (__VA_ARGS__);       \
        if (s_ != IM3D_OK) return s_; \
    } while (0)

std::atomic<long long> g_launches{0};  // kernels launched by this unit (instrumentation)

int launch_status(std::string& err, const char* what)
{
    g_launches++;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("launch of ") + what + ": " + cudaGetErrorString(e);
        return IM3D_ERR_CUDA;
    }
    return IM3D_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// One channels-last BF16 tensor view: base, channels per voxel, volume.
struct View {
    const bf16_t* p;
    int pitch;
    int D, H, W, nsamp;
};

// Tensor map of a view for boxes of 8 channels x (TW + 2) x (TH + 2) x depth.
int make_map(const View& v, int TW, int TH, int depth, CUtensorMap* map, std::string& err)
{
    auto fn = encode_fn();
    if (!fn) {
        err = "cuTensorMapEncodeTiled is not available";
        return IM3D_ERR_CUDA;
    }
    const cuuint64_t es = 2;
    cuuint64_t dims[5] = {(cuuint64_t)v.pitch, (cuuint64_t)v.W, (cuuint64_t)v.H, (cuuint64_t)v.D,
                          (cuuint64_t)v.nsamp};
    cuuint64_t strides[4] = {v.pitch * es, v.pitch * es * v.W, v.pitch * es * v.W * v.H,
                             v.pitch * es * v.W * v.H * v.D};
    cuuint32_t box[5] = {8, (cuuint32_t)(TW + 2), (cuuint32_t)(TH + 2), (cuuint32_t)depth, 1};
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16_t*>(v.p), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return IM3D_ERR_CUDA;
    }
    return IM3D_OK;
}

int pow2_at_least(int x)
{
    int p = 32;
    while (p < x) p *= 2;
    return p;
}

// Tiling of a 3x3x3 convolution over a W x H x D volume for a kernel staging `chunks`
// 8-channel chunks and NOUT output channels.
bool plan_conv(int D, int H, int W, int nsamp, int chunks, int wbytes, int nout, ConvGeom* g, int* smem)
{
    if (W % 16 != 0) return false;
    const int TW = W <= 128 ? W : 128;
    if (W % TW != 0) return false;
    const int P = TW + 2;
    for (int pass = 0; pass < 2; ++pass) {
        const int cap = pass == 0 ? 113 * 1024 : 220 * 1024;
        const int tcap = pass == 0 ? 256 : 512;
        for (int TH : {8, 4, 2, 1}) {
            if (TH > H && TH > 1) continue;
            const int reg = align_up(3 * (TH + 2) * P * 16, 1024);
            const int mt = TW == 128 ? TH : ((TH - 1) * P + TW + 127) / 128;
            const int bytes = align_up(wbytes, 1024) + chunks * reg + kGuardBytes + 64 + 1024;
            if (bytes > cap || mt * nout > tcap) continue;
            g->D = D;
            g->H = H;
            g->W = W;
            g->nsamp = nsamp;
            g->TH = TH;
            g->TW = TW;
            g->tiles_w = W / TW;
            g->tiles_h = (H + TH - 1) / TH;
            g->ntiles = (long long)nsamp * D * g->tiles_h * g->tiles_w;
            g->mtiles = mt;
            g->reg_bytes = reg;
            g->tmem_cols = pow2_at_least(mt * nout);
            *smem = bytes;
            return true;
        }
    }
    return false;
}

int g_num_sms = 148;

template <int CIN, int NOUT, int MODE>
int conv_launch(cudaStream_t st, const View& x, int in_coff, const bf16_t* wpk, int nblocks, const float* bias,
                void* out, int out_pitch, int out_coff, const bf16_t* mask, int mask_pitch, int mask_coff, int* errf,
                std::string& err)
{
    ConvGeom g;
    int smem = 0;
    if (!plan_conv(x.D, x.H, x.W, x.nsamp, CIN / 8, conv_weight_bytes<CIN, NOUT>(), NOUT, &g, &smem)) {
        err = "no convolution tiling fits this volume (W must be a multiple of 16, and of 128 above 128)";
        return IM3D_ERR_UNSUPPORTED;
    }
    CUtensorMap map;
    UN_TRY(make_map(x, g.TW, g.TH, 3, &map, err));
    auto kern = conv3_tc_kernel<CIN, NOUT, MODE>;
    UN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ConvArgs a;
    a.g = g;
    a.wpk = wpk;
    a.bias = bias;
    a.out = out;
    a.out_pitch = out_pitch;
    a.out_coff = out_coff;
    a.mask = mask;
    a.mask_pitch = mask_pitch;
    a.mask_coff = mask_coff;
    a.in_coff = in_coff;
    a.err = errf;
    // at most 2 CTAs per SM with <= 256 TMEM columns each, else 1 with up to 512: the
    // shared-memory request enforces it, so that no CTA's TMEM allocation has to wait
    const int per_sm = smem <= 113 * 1024 && g.tmem_cols <= 256 ? 2 : 1;
    if (per_sm == 2 && smem < 77 * 1024) smem = 77 * 1024;
    if (per_sm == 1 && smem < 116 * 1024) smem = 116 * 1024;
    UN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    long long gx = (long long)g_num_sms * per_sm;
    if (gx > g.ntiles) gx = g.ntiles;
    kern<<<dim3((unsigned)gx, (unsigned)nblocks), 128, smem, st>>>(map, a);
    return launch_status(err, "conv3_tc_kernel");
}

// Dispatch on the staged input channels and the output block width.
template <int MODE>
int conv_any(cudaStream_t st, int cin, int nout, const View& x, int in_coff, const bf16_t* wpk, int nblocks,
             const float* bias, void* out, int op, int oc, const bf16_t* mask, int mp, int mc, int* errf,
             std::string& err)
{
#define UN_CASE(CI, NO)                                                                                           \
    if (cin == CI && nout == NO)                                                                                  \
        return conv_launch<CI, NO, MODE>(st, x, in_coff, wpk, nblocks, bias, out, op, oc, mask, mp, mc, errf, err);
    UN_CASE(16, 16)
    UN_CASE(16, 32)
    UN_CASE(32, 16)
    UN_CASE(32, 32)
    UN_CASE(64, 16)
    UN_CASE(64, 32)
#undef UN_CASE
    err = "unsupported convolution shape";
    return IM3D_ERR_UNSUPPORTED;
}

// Output-channel block width for a layer: 32 where the filter and the staged block
// fit beside each other, else 16.
int nout_for(int cin, int cout, int W)
{
    if (cout < 32) return 16;
    ConvGeom g;
    int smem;
    if (cin == 64) {
        const int wb = 27 * 8 * 32 * 16;
        if (!plan_conv(8, 8, W, 1, 8, wb, 32, &g, &smem)) return 16;
        return g.TH >= 2 ? 32 : 16;
    }
    return 32;
}

template <int CIN>
int wgrad_launch(cudaStream_t st, const View& x, int xcoff, const View& dz, int zcoff, int cout, float* dw,
                 int* errf, std::string& err)
{
    if (x.W % 16 != 0) {
        err = "weight gradient: W must be a multiple of 16";
        return IM3D_ERR_UNSUPPORTED;
    }
    const int TW = x.W <= 128 ? x.W : 128;
    const int P = TW + 2;
    int TH = 0, reg_z = 0, reg_x = 0, smem = 0;
    for (int th : {8, 4, 2, 1}) {
        if (th > x.H && th > 1) continue;
        const int rz = align_up((th + 2) * P * 16, 1024);
        const int rx = align_up(3 * (th + 2) * P * 16, 1024);
        // the 64-row A operand reads 8 chunk regions from the dZ block: keep them inside
        const int over = (8 - cout / 8) * rz - (CIN / 8) * rx;
        const int bytes = wgrad_smem_bytes<CIN>(cout, rz, rx) + (over > 0 ? over : 0);
        if (bytes <= 220 * 1024) {
            TH = th;
            reg_z = rz;
            reg_x = rx;
            smem = bytes;
            break;
        }
    }
    if (!TH) {
        err = "weight gradient: no tiling fits shared memory";
        return IM3D_ERR_UNSUPPORTED;
    }
    ConvGeom g;
    g.D = x.D;
    g.H = x.H;
    g.W = x.W;
    g.nsamp = x.nsamp;
    g.TH = TH;
    g.TW = TW;
    g.tiles_w = x.W / TW;
    g.tiles_h = (x.H + TH - 1) / TH;
    g.ntiles = (long long)x.nsamp * x.D * g.tiles_h * g.tiles_w;
    g.mtiles = 0;
    g.reg_bytes = reg_x;
    g.tmem_cols = 512;
    CUtensorMap xm, zm;
    UN_TRY(make_map(x, TW, TH, 3, &xm, err));
    UN_TRY(make_map(dz, TW, TH, 1, &zm, err));
    WgradArgs a;
    a.g = g;
    a.zcoff = zcoff;
    a.xcoff = xcoff;
    a.tap0 = 0;
    a.ntaps = 512 / CIN < 27 ? 512 / CIN : 27;
    a.cout = cout;
    a.dw = dw;
    a.err = errf;
    const int groups = (27 + a.ntaps - 1) / a.ntaps;
    long long splits = (g_num_sms + groups - 1) / groups;
    if (splits > g.ntiles) splits = g.ntiles;
    auto kern = wgrad_tc_kernel<CIN>;
    if (smem < 116 * 1024) smem = 116 * 1024;  // one CTA per SM: it allocates all 512 TMEM columns
    UN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<dim3((unsigned)groups, (unsigned)splits), 128, smem, st>>>(xm, zm, a, reg_z, reg_x);
    return launch_status(err, "wgrad_tc_kernel");
}

int wgrad_any(cudaStream_t st, int cin, const View& x, int xcoff, const View& dz, int zcoff, int cout, float* dw,
              int* errf, std::string& err)
{
    if (cin == 16) return wgrad_launch<16>(st, x, xcoff, dz, zcoff, cout, dw, errf, err);
    if (cin == 32) return wgrad_launch<32>(st, x, xcoff, dz, zcoff, cout, dw, errf, err);
    if (cin == 64) return wgrad_launch<64>(st, x, xcoff, dz, zcoff, cout, dw, errf, err);
    err = "unsupported weight-gradient shape";
    return IM3D_ERR_UNSUPPORTED;
}

int flat_blocks(long long n, int per = 256)
{
    long long b = (n + per - 1) / per;
    if (b > (long long)g_num_sms * 32) b = (long long)g_num_sms * 32;
    return (int)(b < 1 ? 1 : b);
}

// input fields (FP32, [s][f][n]) -> x0 (BF16 channels-last, 16 channels, 4 used)
__global__ void prep_input_kernel(const float* __restrict__ x, long long n, int nsamp, bf16_t* __restrict__ x0)
{
    const long long total = n * nsamp;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
        const long long s = q / n, v = q % n;
        const float* xs = x + s * 4 * n;
        uint4 lo, hi;
        lo.x = (uint32_t)to_bf(xs[v]) | ((uint32_t)to_bf(xs[n + v]) << 16);
        lo.y = (uint32_t)to_bf(xs[2 * n + v]) | ((uint32_t)to_bf(xs[3 * n + v]) << 16);
        lo.z = lo.w = 0;
        hi.x = hi.y = hi.z = hi.w = 0;
        uint4* d = reinterpret_cast<uint4*>(x0 + q * 16);
        d[0] = lo;
        d[1] = hi;
    }
}

}  // namespace

// ======================================================================= network
enum { E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, NCONV };
static const int kCin[NCONV] = {16, 16, 16, 32, 32, 64, 64, 32, 32, 16};
static const int kCout[NCONV] = {16, 16, 32, 32, 64, 64, 32, 32, 16, 16};

struct im3d_unet {
    int device = 0;
    // FP32 master parameters, their gradients and Adam moments
    std::vector<size_t> w_off, b_off;  // per conv layer
    size_t up2_w = 0, up2_b = 0, up1_w = 0, up1_b = 0, out_w = 0, out_b = 0;
    size_t nparams = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    long long step = 0;
    // BF16 operand copies of the filters (forward and data-gradient blocks)
    bf16_t *wf = nullptr, *wd = nullptr;
    std::vector<size_t> wf_off, wd_off;
    int nout_f[NCONV], nout_d[NCONV];
    bf16_t* upk = nullptr;  // BF16 copies of the two transposed-convolution filters
    size_t upk2 = 0, upk1 = 0;
    int* errf = nullptr;     // device flag raised by a wait that gave up
    double* loss_d = nullptr;
    // activations and gradients of the largest volume seen
    size_t cap_vox = 0;
    bf16_t *x0 = nullptr, *a1 = nullptr, *cat1 = nullptr, *p1 = nullptr, *b1 = nullptr, *cat2 = nullptr,
           *p2 = nullptr, *c1 = nullptr, *c = nullptr, *d2a = nullptr, *d2 = nullptr, *d1a = nullptr, *d1 = nullptr;
    uint8_t *idx1 = nullptr, *idx2 = nullptr;
    bf16_t *g_d1 = nullptr, *g_d1a = nullptr, *g_cat1 = nullptr, *g_d2 = nullptr, *g_d2a = nullptr,
           *g_cat2 = nullptr, *g_c = nullptr, *g_c1 = nullptr, *g_p2 = nullptr, *g_b1 = nullptr, *g_p1 = nullptr,
           *g_a1 = nullptr;
    std::vector<void*> acts;
    float* xin = nullptr;    // staged host inputs
    float* yout = nullptr;
    float* tgt = nullptr;
    size_t io_cap = 0;
    bool packed = false;     // BF16 copies current with p
};

namespace {

void free_acts(im3d_unet* n)
{
    for (void* q : n->acts) cudaFree(q);
    n->acts.clear();
    n->cap_vox = 0;
}

int alloc_acts(im3d_unet* n, size_t n1, std::string& err)
{
    if (n1 <= n->cap_vox) return IM3D_OK;
    free_acts(n);
    const size_t n2 = n1 / 8, n3 = n1 / 64;
    auto A = [&](bf16_t** dst, size_t count) -> int {
        void* q = nullptr;
        UN_CUDA(cudaMalloc(&q, count * 2 + 256));
        n->acts.push_back(q);
        *dst = static_cast<bf16_t*>(q);
        return IM3D_OK;
    };
    UN_TRY(A(&n->x0, n1 * 16));
    UN_TRY(A(&n->a1, n1 * 16));
    UN_TRY(A(&n->cat1, n1 * 32));
    UN_TRY(A(&n->p1, n2 * 16));
    UN_TRY(A(&n->b1, n2 * 32));
    UN_TRY(A(&n->cat2, n2 * 64));
    UN_TRY(A(&n->p2, n3 * 32));
    UN_TRY(A(&n->c1, n3 * 64));
    UN_TRY(A(&n->c, n3 * 64));
    UN_TRY(A(&n->d2a, n2 * 32));
    UN_TRY(A(&n->d2, n2 * 32));
    UN_TRY(A(&n->d1a, n1 * 16));
    UN_TRY(A(&n->d1, n1 * 16));
    UN_TRY(A(reinterpret_cast<bf16_t**>(&n->idx1), n2 * 8 + 16));
    UN_TRY(A(reinterpret_cast<bf16_t**>(&n->idx2), n3 * 16 + 16));
    UN_TRY(A(&n->g_d1, n1 * 16));
    UN_TRY(A(&n->g_d1a, n1 * 16));
    UN_TRY(A(&n->g_cat1, n1 * 32));
    UN_TRY(A(&n->g_d2, n2 * 32));
    UN_TRY(A(&n->g_d2a, n2 * 32));
    UN_TRY(A(&n->g_cat2, n2 * 64));
    UN_TRY(A(&n->g_c, n3 * 64));
    UN_TRY(A(&n->g_c1, n3 * 64));
    UN_TRY(A(&n->g_p2, n3 * 32));
    UN_TRY(A(&n->g_b1, n2 * 32));
    UN_TRY(A(&n->g_p1, n2 * 16));
    UN_TRY(A(&n->g_a1, n1 * 16));
    n->cap_vox = n1;
    return IM3D_OK;
}

// BF16 operand copies of the FP32 filters
int pack_params(im3d_unet* n, cudaStream_t st, std::string& err)
{
    if (n->packed) return IM3D_OK;
    for (int l = 0; l < NCONV; ++l) {
        pack_filter_kernel<<<flat_blocks(27LL * kCin[l] * kCout[l]), 256, 0, st>>>(
            n->p + n->w_off[l], kCout[l], kCin[l], n->nout_f[l], 0, n->wf + n->wf_off[l]);
        UN_TRY(launch_status(err, "pack_filter"));
        if (l != E1A) {
            pack_filter_kernel<<<flat_blocks(27LL * kCin[l] * kCout[l]), 256, 0, st>>>(
                n->p + n->w_off[l], kCout[l], kCin[l], n->nout_d[l], 1, n->wd + n->wd_off[l]);
            UN_TRY(launch_status(err, "pack_filter"));
        }
    }
    to_bf16_kernel<<<flat_blocks(8 * 64 * 32), 256, 0, st>>>(n->p + n->up2_w, n->upk + n->upk2, 8 * 64 * 32);
    to_bf16_kernel<<<flat_blocks(8 * 32 * 16), 256, 0, st>>>(n->p + n->up1_w, n->upk + n->upk1, 8 * 32 * 16);
    UN_TRY(launch_status(err, "to_bf16"));
    n->packed = true;
    return IM3D_OK;
}

// Every level's width W, W/2, W/4 is staged in tiles of min(width, 128) columns, which
// must divide it and be a multiple of 16.
int check_dims(int nsamp, int D, int H, int W, std::string& err)
{
    bool ok = nsamp >= 1 && D >= 4 && H >= 4 && D % 4 == 0 && H % 4 == 0 && W % 4 == 0;
    for (int l = 0; l < 3 && ok; ++l) {
        const int w = W >> l;
        ok = w % 16 == 0 && (w <= 128 || w % 128 == 0);
    }
    if (!ok) {
        err = "network volumes need D and H multiples of 4, and W with W, W/2 and W/4 multiples of 16 that are "
              "at most 128 or multiples of 128";
        return IM3D_ERR_UNSUPPORTED;
    }
    return IM3D_OK;
}

// Forward pass from x0 (already staged); y (FP32, n1 per sample) if not NULL.
int forward(im3d_unet* n, cudaStream_t st, int nsamp, int D, int H, int W, float* y, std::string& err)
{
    UN_TRY(pack_params(n, st, err));
    const int D2 = D / 2, H2 = H / 2, W2 = W / 2, D3 = D / 4, H3 = H / 4, W3 = W / 4;
    const long long n1 = (long long)nsamp * D * H * W, n2 = n1 / 8, n3 = n1 / 64;
    auto conv = [&](int l, const View& x, int coff, void* out, int op, int oc) -> int {
        return conv_any<CONV_BIAS_RELU>(st, kCin[l], n->nout_f[l], x, coff, n->wf + n->wf_off[l],
                                        kCout[l] / n->nout_f[l], n->p + n->b_off[l], out, op, oc, nullptr, 0, 0,
                                        n->errf, err);
    };
    const View L1{nullptr, 16, D, H, W, nsamp};
    View v = L1;
    v.p = n->x0;
    UN_TRY(conv(E1A, v, 0, n->a1, 16, 0));
    v.p = n->a1;
    UN_TRY(conv(E1B, v, 0, n->cat1, 32, 16));                    // a -> cat1[16:32]
    pool_fwd_kernel<<<flat_blocks(n2 * 16), 256, 0, st>>>(n->cat1, 32, 16, 16, D, H, W, nsamp, n->p1, n->idx1);
    UN_TRY(launch_status(err, "pool_fwd"));
    View v2{n->p1, 16, D2, H2, W2, nsamp};
    UN_TRY(conv(E2A, v2, 0, n->b1, 32, 0));
    v2.p = n->b1;
    v2.pitch = 32;
    UN_TRY(conv(E2B, v2, 0, n->cat2, 64, 32));                   // b -> cat2[32:64]
    pool_fwd_kernel<<<flat_blocks(n3 * 32), 256, 0, st>>>(n->cat2, 64, 32, 32, D2, H2, W2, nsamp, n->p2, n->idx2);
    UN_TRY(launch_status(err, "pool_fwd"));
    View v3{n->p2, 32, D3, H3, W3, nsamp};
    UN_TRY(conv(E3A, v3, 0, n->c1, 64, 0));
    v3.p = n->c1;
    v3.pitch = 64;
    UN_TRY(conv(E3B, v3, 0, n->c, 64, 0));
    upconv_fwd_kernel<64, 32><<<flat_blocks(n2, 128), 128, 0, st>>>(n->c, n->upk + n->upk2, n->p + n->up2_b, D3, H3,
                                                                    W3, nsamp, n->cat2, 64, 0);
    UN_TRY(launch_status(err, "upconv_fwd"));
    View c2{n->cat2, 64, D2, H2, W2, nsamp};
    UN_TRY(conv(D2A, c2, 0, n->d2a, 32, 0));
    c2.p = n->d2a;
    c2.pitch = 32;
    UN_TRY(conv(D2B, c2, 0, n->d2, 32, 0));
    upconv_fwd_kernel<32, 16><<<flat_blocks(n1, 128), 128, 0, st>>>(n->d2, n->upk + n->upk1, n->p + n->up1_b, D2, H2,
                                                                    W2, nsamp, n->cat1, 32, 0);
    UN_TRY(launch_status(err, "upconv_fwd"));
    View c1v{n->cat1, 32, D, H, W, nsamp};
    UN_TRY(conv(D1A, c1v, 0, n->d1a, 16, 0));
    c1v.p = n->d1a;
    c1v.pitch = 16;
    UN_TRY(conv(D1B, c1v, 0, n->d1, 16, 0));
    if (y) {
        out_layer_kernel<16><<<flat_blocks(n1), 256, 0, st>>>(n->d1, n->p + n->out_w, n->p + n->out_b, n1, y,
                                                              nullptr, nullptr, 0.f, nullptr, nullptr, nullptr,
                                                              nullptr);
        UN_TRY(launch_status(err, "out_layer"));
    }
    return IM3D_OK;
}

// Backward pass after forward(); gradients accumulate into n->g (zeroed here).
int backward(im3d_unet* n, cudaStream_t st, int nsamp, int D, int H, int W, const float* target, const float* wt,
             float* y, std::string& err)
{
    const int D2 = D / 2, H2 = H / 2, W2 = W / 2, D3 = D / 4, H3 = H / 4, W3 = W / 4;
    const long long n1 = (long long)nsamp * D * H * W, n2 = n1 / 8, n3 = n1 / 64;
    zero_f32_kernel<<<flat_blocks(n->nparams), 256, 0, st>>>(n->g, (long long)n->nparams);
    UN_CUDA(cudaMemsetAsync(n->loss_d, 0, sizeof(double), st));
    out_layer_kernel<16><<<flat_blocks(n1), 256, 0, st>>>(n->d1, n->p + n->out_w, n->p + n->out_b, n1, y, target, wt,
                                                          1.f / (float)n1, n->g_d1, n->g + n->out_w, n->g + n->out_b,
                                                          n->loss_d);
    UN_TRY(launch_status(err, "out_layer"));
    // data gradient of layer l: dZ (pitch zp, offset zo) -> out (masked by `mask`)
    auto dgrad = [&](int l, const View& dz, int zo, void* out, int op, int oc, const bf16_t* mask, int mp, int mc) {
        return conv_any<CONV_MASK>(st, kCout[l], n->nout_d[l], dz, zo, n->wd + n->wd_off[l], kCin[l] / n->nout_d[l],
                                   nullptr, out, op, oc, mask, mp, mc, n->errf, err);
    };
    auto wgrad = [&](int l, const View& x, int xo, const View& dz, int zo) {
        int s = wgrad_any(st, kCin[l], x, xo, dz, zo, kCout[l], n->g + n->w_off[l], n->errf, err);
        if (s != IM3D_OK) return s;
        const long long nv = (long long)dz.nsamp * dz.D * dz.H * dz.W;
        bias_grad_kernel<<<flat_blocks(nv), 256, 0, st>>>(dz.p, dz.pitch, zo, kCout[l], nv, n->g + n->b_off[l]);
        return launch_status(err, "bias_grad");
    };
    // level 1 decoder
    View gd1{n->g_d1, 16, D, H, W, nsamp};
    UN_TRY(wgrad(D1B, View{n->d1a, 16, D, H, W, nsamp}, 0, gd1, 0));
    UN_TRY(dgrad(D1B, gd1, 0, n->g_d1a, 16, 0, n->d1a, 16, 0));
    View gd1a{n->g_d1a, 16, D, H, W, nsamp};
    UN_TRY(wgrad(D1A, View{n->cat1, 32, D, H, W, nsamp}, 0, gd1a, 0));
    UN_TRY(dgrad(D1A, gd1a, 0, n->g_cat1, 32, 0, nullptr, 0, 0));  // [d up1 | d a (skip, raw)]
    // transposed convolution 1
    upconv_wgrad_kernel<32, 16><<<flat_blocks(n2, 32), 256, 0, st>>>(n->d2, n->g_cat1, 32, 0, D2, H2, W2, nsamp,
                                                                      n->g + n->up1_w, n->g + n->up1_b);
    UN_TRY(launch_status(err, "upconv_wgrad"));
    upconv_bwd_kernel<32, 16><<<flat_blocks(n2, 128), 128, 0, st>>>(n->g_cat1, 32, 0, n->upk + n->upk1, n->d2, D2, H2,
                                                                    W2, nsamp, n->g_d2);
    UN_TRY(launch_status(err, "upconv_bwd"));
    // level 2 decoder
    View gd2{n->g_d2, 32, D2, H2, W2, nsamp};
    UN_TRY(wgrad(D2B, View{n->d2a, 32, D2, H2, W2, nsamp}, 0, gd2, 0));
    UN_TRY(dgrad(D2B, gd2, 0, n->g_d2a, 32, 0, n->d2a, 32, 0));
    View gd2a{n->g_d2a, 32, D2, H2, W2, nsamp};
    UN_TRY(wgrad(D2A, View{n->cat2, 64, D2, H2, W2, nsamp}, 0, gd2a, 0));
    UN_TRY(dgrad(D2A, gd2a, 0, n->g_cat2, 64, 0, nullptr, 0, 0));  // [d up2 | d b (skip, raw)]
    // transposed convolution 2
    upconv_wgrad_kernel<64, 32><<<flat_blocks(n3, 32), 256, 0, st>>>(n->c, n->g_cat2, 64, 0, D3, H3, W3, nsamp,
                                                                      n->g + n->up2_w, n->g + n->up2_b);
    UN_TRY(launch_status(err, "upconv_wgrad"));
    upconv_bwd_kernel<64, 32><<<flat_blocks(n3, 128), 128, 0, st>>>(n->g_cat2, 64, 0, n->upk + n->upk2, n->c, D3, H3,
                                                                    W3, nsamp, n->g_c);
    UN_TRY(launch_status(err, "upconv_bwd"));
    // level 3
    View gc{n->g_c, 64, D3, H3, W3, nsamp};
    UN_TRY(wgrad(E3B, View{n->c1, 64, D3, H3, W3, nsamp}, 0, gc, 0));
    UN_TRY(dgrad(E3B, gc, 0, n->g_c1, 64, 0, n->c1, 64, 0));
    View gc1{n->g_c1, 64, D3, H3, W3, nsamp};
    UN_TRY(wgrad(E3A, View{n->p2, 32, D3, H3, W3, nsamp}, 0, gc1, 0));
    UN_TRY(dgrad(E3A, gc1, 0, n->g_p2, 32, 0, nullptr, 0, 0));
    // pooling 2: g_b = (g_skip + scatter(g_p2)) * (b > 0), in place in g_cat2[32:64]
    pool_bwd_kernel<<<flat_blocks(n3 * 32), 256, 0, st>>>(n->g_p2, n->idx2, 32, D2, H2, W2, nsamp, n->g_cat2, 64, 32,
                                                          n->cat2, 64, 32, n->g_cat2, 64, 32);
    UN_TRY(launch_status(err, "pool_bwd"));
    View gb{n->g_cat2, 64, D2, H2, W2, nsamp};
    UN_TRY(wgrad(E2B, View{n->b1, 32, D2, H2, W2, nsamp}, 0, gb, 32));
    UN_TRY(dgrad(E2B, gb, 32, n->g_b1, 32, 0, n->b1, 32, 0));
    View gb1{n->g_b1, 32, D2, H2, W2, nsamp};
    UN_TRY(wgrad(E2A, View{n->p1, 16, D2, H2, W2, nsamp}, 0, gb1, 0));
    UN_TRY(dgrad(E2A, gb1, 0, n->g_p1, 16, 0, nullptr, 0, 0));
    // pooling 1: g_a in place in g_cat1[16:32]
    pool_bwd_kernel<<<flat_blocks(n2 * 16), 256, 0, st>>>(n->g_p1, n->idx1, 16, D, H, W, nsamp, n->g_cat1, 32, 16,
                                                          n->cat1, 32, 16, n->g_cat1, 32, 16);
    UN_TRY(launch_status(err, "pool_bwd"));
    View ga{n->g_cat1, 32, D, H, W, nsamp};
    UN_TRY(wgrad(E1B, View{n->a1, 16, D, H, W, nsamp}, 0, ga, 16));
    UN_TRY(dgrad(E1B, ga, 16, n->g_a1, 16, 0, n->a1, 16, 0));
    View ga1{n->g_a1, 16, D, H, W, nsamp};
    UN_TRY(wgrad(E1A, View{n->x0, 16, D, H, W, nsamp}, 0, ga1, 0));
    return IM3D_OK;
}

int check_err_flag(im3d_unet* n, cudaStream_t st, std::string& err)
{
    int h = 0;
    UN_CUDA(cudaMemcpyAsync(&h, n->errf, sizeof(int), cudaMemcpyDeviceToHost, st));
    UN_CUDA(cudaStreamSynchronize(st));
    if (h) {
        cudaMemsetAsync(n->errf, 0, sizeof(int), st);
        err = "a tensor-core kernel gave up waiting for its data (code " + std::to_string(h) + ")";
        return IM3D_ERR_CUDA;
    }
    return IM3D_OK;
}

bool is_dev(const void* p)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int stage_io(im3d_unet* n, size_t count, std::string& err)
{
    if (count <= n->io_cap) return IM3D_OK;
    cudaFree(n->xin);
    cudaFree(n->yout);
    cudaFree(n->tgt);
    n->xin = n->yout = n->tgt = nullptr;
    n->io_cap = 0;
    UN_CUDA(cudaMalloc(&n->xin, 4 * count * sizeof(float)));
    UN_CUDA(cudaMalloc(&n->yout, count * sizeof(float)));
    UN_CUDA(cudaMalloc(&n->tgt, count * sizeof(float)));
    n->io_cap = count;
    return IM3D_OK;
}

}  // namespace

// -------------------------------------------------- internal entry points (loop)
namespace im3d {
namespace unet {

int net_forward_fields(im3d_unet* n, cudaStream_t st, const float* x, int nsamp, int D, int H, int W, float* y,
                       std::string& err)
{
    UN_TRY(check_dims(nsamp, D, H, W, err));
    const long long n1 = (long long)nsamp * D * H * W;
    UN_TRY(alloc_acts(n, (size_t)n1, err));
    prep_input_kernel<<<flat_blocks(n1), 256, 0, st>>>(x, (long long)D * H * W, nsamp, n->x0);
    UN_TRY(launch_status(err, "prep_input"));
    UN_TRY(forward(n, st, nsamp, D, H, W, y, err));
    return check_err_flag(n, st, err);
}

int net_train_fields(im3d_unet* n, cudaStream_t st, const float* x, const float* target, const float* wt, int nsamp,
                     int D, int H, int W, double lr, double* loss, float* grads_host, std::string& err)
{
    UN_TRY(check_dims(nsamp, D, H, W, err));
    const long long n1 = (long long)nsamp * D * H * W;
    UN_TRY(alloc_acts(n, (size_t)n1, err));
    prep_input_kernel<<<flat_blocks(n1), 256, 0, st>>>(x, (long long)D * H * W, nsamp, n->x0);
    UN_TRY(launch_status(err, "prep_input"));
    UN_TRY(forward(n, st, nsamp, D, H, W, nullptr, err));
    UN_TRY(backward(n, st, nsamp, D, H, W, target, wt, nullptr, err));
    if (grads_host)
        UN_CUDA(cudaMemcpyAsync(grads_host, n->g, n->nparams * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (lr > 0) {
        n->step++;
        const float b1 = 0.9f, b2 = 0.999f;
        const double c1 = 1.0 - std::pow((double)b1, (double)n->step), c2 = 1.0 - std::pow((double)b2, (double)n->step);
        const float lr_t = (float)(lr * std::sqrt(c2) / c1);
        adam_kernel<<<flat_blocks((long long)n->nparams), 256, 0, st>>>(n->p, n->g, n->m, n->v,
                                                                        (long long)n->nparams, lr_t, b1, b2, 1e-8f, 1.f);
        UN_TRY(launch_status(err, "adam"));
        n->packed = false;
    }
    double l = 0;
    UN_CUDA(cudaMemcpyAsync(&l, n->loss_d, sizeof(double), cudaMemcpyDeviceToHost, st));
    UN_TRY(check_err_flag(n, st, err));
    if (loss) *loss = l / (double)n1;
    return IM3D_OK;
}

int net_device(const im3d_unet* n) { return n->device; }

long long launch_total() { return g_launches.load(); }

}  // namespace unet
}  // namespace im3d

// ===================================================================== C ABI
extern "C" {

int im3d_unet_create(im3d_ctx* ctx, uint64_t seed, im3d_unet** out)
{
    if (!ctx || !out) return IM3D_ERR_INVALID_ARG;
    *out = nullptr;
    std::string& err = im3d_ctx_error_ref(ctx);
    const int dev = im3d_ctx_device(ctx);
    UN_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    UN_CUDA(cudaGetDeviceProperties(&prop, dev));
    g_num_sms = prop.multiProcessorCount;
    im3d_unet* n = new im3d_unet();
    n->device = dev;
    size_t off = 0;
    for (int l = 0; l < NCONV; ++l) {
        n->w_off.push_back(off);
        off += (size_t)kCout[l] * kCin[l] * 27;
        n->b_off.push_back(off);
        off += (size_t)kCout[l];
    }
    n->up2_w = off; off += 8 * 64 * 32;
    n->up2_b = off; off += 32;
    n->up1_w = off; off += 8 * 32 * 16;
    n->up1_b = off; off += 16;
    n->out_w = off; off += 16;
    n->out_b = off; off += 1;
    n->nparams = off;
    // He-normal initialisation (fan-in), zero biases; the 12 unused input channels of
    // the first layer get zero weights
    std::vector<float> host(off, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int l = 0; l < NCONV; ++l) {
        const int fan = (l == E1A ? 4 : kCin[l]) * 27;
        const float sd = std::sqrt(2.f / fan);
        for (int co = 0; co < kCout[l]; ++co)
            for (int ci = 0; ci < kCin[l]; ++ci)
                for (int t = 0; t < 27; ++t)
                    host[n->w_off[l] + ((size_t)co * kCin[l] + ci) * 27 + t] = (l == E1A && ci >= 4) ? 0.f : sd * nd(rng);
    }
    for (size_t q = 0; q < 8 * 64 * 32; ++q) host[n->up2_w + q] = std::sqrt(2.f / 64) * nd(rng);
    for (size_t q = 0; q < 8 * 32 * 16; ++q) host[n->up1_w + q] = std::sqrt(2.f / 32) * nd(rng);
    for (int q = 0; q < 16; ++q) host[n->out_w + q] = 0.f;  // the network starts by predicting no correction
    size_t wf = 0, wd = 0;
    for (int l = 0; l < NCONV; ++l) {
        n->nout_f[l] = nout_for(kCin[l], kCout[l], 128);
        n->nout_d[l] = nout_for(kCout[l], kCin[l], 128);
        n->wf_off.push_back(wf);
        wf += (size_t)27 * kCin[l] * kCout[l];
        n->wd_off.push_back(wd);
        wd += (size_t)27 * kCin[l] * kCout[l];
    }
    auto fail = [&](int code) {
        im3d_unet_destroy(n);
        return code;
    };
    if (cudaMalloc(&n->p, off * 4) != cudaSuccess || cudaMalloc(&n->g, off * 4) != cudaSuccess ||
        cudaMalloc(&n->m, off * 4) != cudaSuccess || cudaMalloc(&n->v, off * 4) != cudaSuccess ||
        cudaMalloc(&n->wf, wf * 2) != cudaSuccess || cudaMalloc(&n->wd, wd * 2) != cudaSuccess ||
        cudaMalloc(&n->upk, (8 * 64 * 32 + 8 * 32 * 16) * 2) != cudaSuccess ||
        cudaMalloc(&n->errf, sizeof(int)) != cudaSuccess || cudaMalloc(&n->loss_d, sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        err = "cudaMalloc of the network's parameters failed";
        return fail(IM3D_ERR_OOM);
    }
    n->upk2 = 0;
    n->upk1 = 8 * 64 * 32;
    if (cudaMemcpy(n->p, host.data(), off * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(n->m, 0, off * 4) != cudaSuccess || cudaMemset(n->v, 0, off * 4) != cudaSuccess ||
        cudaMemset(n->errf, 0, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        err = "initialising the network's parameters failed";
        return fail(IM3D_ERR_CUDA);
    }
    *out = n;
    return IM3D_OK;
}

int im3d_unet_destroy(im3d_unet* n)
{
    if (!n) return IM3D_OK;
    cudaSetDevice(n->device);
    cudaDeviceSynchronize();
    free_acts(n);
    for (void* q : {(void*)n->p, (void*)n->g, (void*)n->m, (void*)n->v, (void*)n->wf, (void*)n->wd, (void*)n->upk,
                    (void*)n->errf, (void*)n->loss_d, (void*)n->xin, (void*)n->yout, (void*)n->tgt})
        if (q) cudaFree(q);
    delete n;
    return IM3D_OK;
}

int64_t im3d_unet_param_count(const im3d_unet* n) { return n ? (int64_t)n->nparams : 0; }

int im3d_unet_get_params(im3d_ctx* ctx, im3d_unet* n, float* host, int64_t count)
{
    if (!ctx || !n || !host || count != (int64_t)n->nparams) return IM3D_ERR_INVALID_ARG;
    std::string& err = im3d_ctx_error_ref(ctx);
    UN_CUDA(cudaSetDevice(n->device));
    UN_CUDA(cudaMemcpy(host, n->p, n->nparams * 4, cudaMemcpyDeviceToHost));
    return IM3D_OK;
}

int im3d_unet_set_params(im3d_ctx* ctx, im3d_unet* n, const float* host, int64_t count)
{
    if (!ctx || !n || !host || count != (int64_t)n->nparams) return IM3D_ERR_INVALID_ARG;
    std::string& err = im3d_ctx_error_ref(ctx);
    UN_CUDA(cudaSetDevice(n->device));
    UN_CUDA(cudaDeviceSynchronize());
    UN_CUDA(cudaMemcpy(n->p, host, n->nparams * 4, cudaMemcpyHostToDevice));
    UN_CUDA(cudaMemset(n->m, 0, n->nparams * 4));
    UN_CUDA(cudaMemset(n->v, 0, n->nparams * 4));
    n->step = 0;
    n->packed = false;
    return IM3D_OK;
}

int im3d_unet_forward(im3d_ctx* ctx, im3d_unet* n, const float* x, int nsamp, int nx, int ny, int nz, float* y)
{
    if (!ctx || !n || !x || !y) return IM3D_ERR_INVALID_ARG;
    std::string& err = im3d_ctx_error_ref(ctx);
    err.clear();
    UN_CUDA(cudaSetDevice(n->device));
    cudaStream_t st = im3d_ctx_stream(ctx);
    UN_TRY(check_dims(nsamp, nx, ny, nz, err));
    const size_t cnt = (size_t)nsamp * nx * ny * nz;
    const float* xd = x;
    float* yd = y;
    if (!is_dev(x) || !is_dev(y)) UN_TRY(stage_io(n, cnt, err));
    if (!is_dev(x)) {
        UN_CUDA(cudaMemcpyAsync(n->xin, x, 4 * cnt * sizeof(float), cudaMemcpyHostToDevice, st));
        xd = n->xin;
    }
    if (!is_dev(y)) yd = n->yout;
    UN_TRY(im3d::unet::net_forward_fields(n, st, xd, nsamp, nx, ny, nz, yd, err));
    if (yd != y) {
        UN_CUDA(cudaMemcpyAsync(y, yd, cnt * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    UN_CUDA(cudaStreamSynchronize(st));
    return IM3D_OK;
}

int im3d_unet_train_step(im3d_ctx* ctx, im3d_unet* n, const float* x, const float* target, int nsamp, int nx,
                         int ny, int nz, double lr, double* loss, float* grads)
{
    if (!ctx || !n || !x || !target || !(lr >= 0)) return IM3D_ERR_INVALID_ARG;
    std::string& err = im3d_ctx_error_ref(ctx);
    err.clear();
    UN_CUDA(cudaSetDevice(n->device));
    cudaStream_t st = im3d_ctx_stream(ctx);
    UN_TRY(check_dims(nsamp, nx, ny, nz, err));
    const size_t cnt = (size_t)nsamp * nx * ny * nz;
    const float* xd = x;
    const float* td = target;
    if (!is_dev(x) || !is_dev(target)) UN_TRY(stage_io(n, cnt, err));
    if (!is_dev(x)) {
        UN_CUDA(cudaMemcpyAsync(n->xin, x, 4 * cnt * sizeof(float), cudaMemcpyHostToDevice, st));
        xd = n->xin;
    }
    if (!is_dev(target)) {
        UN_CUDA(cudaMemcpyAsync(n->tgt, target, cnt * sizeof(float), cudaMemcpyHostToDevice, st));
        td = n->tgt;
    }
    return im3d::unet::net_train_fields(n, st, xd, td, nullptr, nsamp, nx, ny, nz, lr, loss, grads, err);
}

int im3d_conv3d_bf16(im3d_ctx* ctx, const uint16_t* x, int c_pitch, int c_off, int cin, const float* w,
                     const float* bias, int cout, int nsamp, int nx, int ny, int nz, float* out)
{
    if (!ctx || !x || !w || !out) return IM3D_ERR_INVALID_ARG;
    std::string& err = im3d_ctx_error_ref(ctx);
    err.clear();
    if ((cin != 16 && cin != 32 && cin != 64) || (cout != 16 && cout != 32 && cout != 64) || c_off % 8 ||
        c_off < 0 || c_pitch < c_off + cin || c_pitch % 8 || nsamp < 1 || nx < 1 || ny < 1 || nz < 16) {
        err = "conv3d: cin, cout in {16, 32, 64}; channel offset and pitch multiples of 8; nz >= 16";
        return IM3D_ERR_INVALID_ARG;
    }
    if (!is_dev(x) || !is_dev(w) || !is_dev(out) || (bias && !is_dev(bias))) {
        err = "conv3d: x, w, bias and out must be device memory";
        return IM3D_ERR_INVALID_ARG;
    }
    UN_CUDA(cudaSetDevice(im3d_ctx_device(ctx)));
    cudaStream_t st = im3d_ctx_stream(ctx);
    cudaDeviceProp prop;
    UN_CUDA(cudaGetDeviceProperties(&prop, im3d_ctx_device(ctx)));
    g_num_sms = prop.multiProcessorCount;
    const int nout = cout == 16 ? 16 : 32;
    bf16_t* wpk = nullptr;
    int* errf = nullptr;
    UN_CUDA(cudaMalloc(&wpk, (size_t)27 * cin * cout * 2));
    if (cudaMalloc(&errf, sizeof(int)) != cudaSuccess) {
        cudaFree(wpk);
        err = "cudaMalloc failed";
        return IM3D_ERR_OOM;
    }
    cudaMemsetAsync(errf, 0, sizeof(int), st);
    pack_filter_kernel<<<flat_blocks(27LL * cin * cout), 256, 0, st>>>(w, cout, cin, nout, 0, wpk);
    int s = launch_status(err, "pack_filter");
    const View v{reinterpret_cast<const bf16_t*>(x), c_pitch, nx, ny, nz, nsamp};
    if (s == IM3D_OK)
        s = conv_any<CONV_BIAS_F32>(st, cin, nout, v, c_off, wpk, cout / nout, bias, out, cout, 0, nullptr, 0, 0,
                                    errf, err);
    int h = 0;
    if (s == IM3D_OK && cudaMemcpyAsync(&h, errf, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        cudaStreamSynchronize(st) == cudaSuccess && h) {
        err = "conv3d: a wait gave up";
        s = IM3D_ERR_CUDA;
    }
    cudaStreamSynchronize(st);
    cudaFree(wpk);
    cudaFree(errf);
    return s;
}

}  // extern "C"

// im3d_b200.cu -- host side of the sm_100a backend: context, device buffers, the
// iteration of segm::rsfe_splitbregman<T>::apply, and the C ABI of include/im3d_b200.h.
//
// No CPU fallback: every numerical step below is a kernel of kernels.cuh. The host
// only validates arguments, stages host buffers and steers the loop.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/im3d_b200.h"
#include "common.cuh"
#include "internal.h"
#include "conv_tma.cuh"
#include "kernels.cuh"
#include "worklist.cuh"

#include <cudaTypedefs.h>

using namespace im3d;

// The library is built from this file twice: unit 1 (compiled with -fmad=false, so that
// the FP64 path keeps the reference's operations bit for bit) holds the context, the
// generic entry points and the _f64 ones; unit 2 (im3d_b200_f32.cu, compiled with
// contracted multiply-adds) holds the _f32 entry points. 0 builds everything.
#ifndef IM3D_UNIT
#define IM3D_UNIT 0
#endif

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct im3d_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    std::string err;
    long long launches = 0;
    std::unordered_map<std::string, DevBuf> bufs;
    Ctrl* ctrl_d = nullptr;
    Ctrl* ctrl_h = nullptr;  // pinned
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // [3]: tolerance copy done
    // per-stage device timing (im3d_ctx_set_profiling): events recorded on the
    // launching stream around each launch, resolved at the next synchronisation
    int prof = 0;  // 1: every stage; 2: the Poisson solves as a whole only
    std::vector<cudaEvent_t> ev_pool;
    struct Pending {
        std::string name;
        cudaEvent_t a, b;
        bool closed;  // b recorded (prof_end)
        bool done;    // folded into the totals
    };
    std::vector<Pending> pending;
    struct Acc {
        double ms = 0;
        long long count = 0;
    };
    std::vector<std::pair<std::string, Acc>> prof_acc;
    // worker contexts of the batched entry points (own stream and buffers each)
    std::vector<im3d_ctx*> workers;
    // per-volume contexts of a work-list batch (buffers and control block of each
    // volume; their launches go to this context's stream), and the group's pinned
    // control blocks
    std::vector<im3d_ctx*> vols;
    Ctrl* wl_ctrl_h = nullptr;
    int wl_ctrl_cap = 0;
    cudaEvent_t wl_ev[2] = {nullptr, nullptr};  // work-list solve phase: start, this worker done
    int batch_mode = IM3D_BATCH_AUTO;
    int tile_loads = 1;  // the FP32 Heaviside pass moves its rows with TMA where it can
    int num_sms = 148;
    int ifit_chunks = 0;  // i chunks of the marching fit stage (0: cost model)
    size_t mem_limit = 0;  // device bytes the context may hold in buffers (0: no limit)
    size_t mem_held = 0;   // device bytes it holds in buffers now
    // per-iteration observer (im3d_ctx_set_observer) and its host copy of the state
    im3d_rsfe_observer obs = nullptr;
    void* obs_user = nullptr;
    int obs_every = 0;
    int obs_state = 0;
    std::vector<unsigned char> obs_host;
    // learned warm start of the Poisson solves (im3d_ctx_set_warm_start)
    im3d_unet* ws_net = nullptr;
    int ws_mode = IM3D_WS_OFF;
    double ws_lr = 0;
    // pending resume of the next segmentation (im3d_ctx_set_resume)
    bool resume = false;
    int resume_esize = 0;
    im3d_rsfe_checkpoint resume_from{};
    long long residual_checks = 0;  // rb_check calls, for the statistics
};

namespace {

#define IM3D_CUDA(ctx, call)                                                                  \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                  \
            return e_ == cudaErrorMemoryAllocation ? IM3D_ERR_OOM : IM3D_ERR_CUDA;             \
        }                                                                                     \
    } while (0)

#define IM3D_TRY(...)                   \
    do {                                \
        int s_ = (__VA_ARGS__);         \
        if (s_ != IM3D_OK) return s_;   \
    } while (0)

int fail(im3d_ctx* ctx, int code, const std::string& msg)
{
    ctx->err = msg;
    return code;
}

int check_launch(im3d_ctx* ctx, const char* what)
{
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx->err = std::string("launch of ") + what + ": " + cudaGetErrorString(e);
        return IM3D_ERR_CUDA;
    }
    return IM3D_OK;
}

cudaEvent_t prof_event(im3d_ctx* ctx)
{
    if (!ctx->ev_pool.empty()) {
        cudaEvent_t e = ctx->ev_pool.back();
        ctx->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Start of a profiled launch: returns the pending slot (-1 when profiling is off).
int prof_begin(im3d_ctx* ctx, const char* name)
{
    if (!ctx->prof) return -1;
    if (ctx->prof == 2 && std::strcmp(name, "poisson_solve") != 0) return -1;
    im3d_ctx::Pending pd{name, prof_event(ctx), prof_event(ctx), false, false};
    cudaEventRecord(pd.a, ctx->stream);
    ctx->pending.push_back(pd);
    return (int)ctx->pending.size() - 1;
}

void prof_end(im3d_ctx* ctx, int slot)
{
    if (slot < 0) return;
    cudaEventRecord(ctx->pending[slot].b, ctx->stream);
    ctx->pending[slot].closed = true;
}

// After a stream synchronisation: fold the closed event pairs into the totals. A
// stage that encloses synchronisations (the whole Poisson solve) stays pending until
// it is closed; the slots keep their indices until every pair is folded.
void prof_resolve(im3d_ctx* ctx)
{
    bool all = true;
    for (auto& pd : ctx->pending) {
        if (pd.done) continue;
        if (!pd.closed) {
            all = false;
            continue;
        }
        pd.done = true;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, pd.a, pd.b) != cudaSuccess) {
            cudaGetLastError();
            ms = 0;
        }
        bool found = false;
        for (auto& kv : ctx->prof_acc)
            if (kv.first == pd.name) {
                kv.second.ms += ms;
                kv.second.count++;
                found = true;
                break;
            }
        if (!found) {
            im3d_ctx::Acc a;
            a.ms = ms;
            a.count = 1;
            ctx->prof_acc.push_back({pd.name, a});
        }
        ctx->ev_pool.push_back(pd.a);
        ctx->ev_pool.push_back(pd.b);
    }
    if (all) ctx->pending.clear();
}

// Device buffer of at least `bytes` under `name`, reused across calls.
int buf(im3d_ctx* ctx, const char* name, size_t bytes, void** out, bool zero = false)
{
    DevBuf& b = ctx->bufs[name];
    if (b.bytes < bytes) {
        // the context's memory budget (IM3D_OPT_DEVICE_MEMORY_LIMIT) is checked before
        // anything is freed or allocated
        if (ctx->mem_limit && ctx->mem_held - b.bytes + bytes > ctx->mem_limit) {
            ctx->err = std::string("device memory limit of the context (") +
                       std::to_string(ctx->mem_limit) + " bytes) reached: buffer " + name + " needs " +
                       std::to_string(bytes) + " bytes, " + std::to_string(ctx->mem_held - b.bytes) +
                       " are held";
            return IM3D_ERR_OOM;
        }
        if (b.p) cudaFree(b.p);
        ctx->mem_held -= b.bytes;
        b.p = nullptr;
        b.bytes = 0;
        cudaError_t e = cudaMalloc(&b.p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ctx->err = std::string("cudaMalloc(") + name + ", " + std::to_string(bytes) +
                       " bytes): " + cudaGetErrorString(e);
            return IM3D_ERR_OOM;
        }
        b.bytes = bytes;
        ctx->mem_held += bytes;
    }
    if (zero) IM3D_CUDA(ctx, cudaMemsetAsync(b.p, 0, bytes, ctx->stream));
    *out = b.p;
    return IM3D_OK;
}

template <typename T>
int tbuf(im3d_ctx* ctx, const char* name, size_t count, T** out, bool zero = false)
{
    void* p = nullptr;
    IM3D_TRY(buf(ctx, name, count * sizeof(T) + 256, &p, zero));
    *out = static_cast<T*>(p);
    return IM3D_OK;
}

bool is_device_ptr(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Input: a device pointer is used in place; a host pointer is copied to `slot`.
template <typename T>
int dev_in(im3d_ctx* ctx, const T* p, size_t count, const char* slot, const T** out)
{
    if (is_device_ptr(p)) {
        *out = p;
        return IM3D_OK;
    }
    T* d = nullptr;
    IM3D_TRY(tbuf<T>(ctx, slot, count, &d));
    IM3D_CUDA(ctx, cudaMemcpyAsync(d, p, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    *out = d;
    return IM3D_OK;
}

// Output staging: a device pointer is written directly; a host one goes through
// `slot` and is copied back by out_finish.
template <typename T>
int dev_out(im3d_ctx* ctx, T* p, size_t count, const char* slot, T** out)
{
    if (!p) {
        *out = nullptr;
        return IM3D_OK;
    }
    if (is_device_ptr(p)) {
        *out = p;
        return IM3D_OK;
    }
    return tbuf<T>(ctx, slot, count, out);
}

template <typename T>
int out_finish(im3d_ctx* ctx, T* user, const T* dev, size_t count)
{
    if (!user || user == dev) return IM3D_OK;
    IM3D_CUDA(ctx, cudaMemcpyAsync(user, dev, count * sizeof(T), cudaMemcpyDeviceToHost,
                                   ctx->stream));
    return IM3D_OK;
}

int sync(im3d_ctx* ctx)
{
    IM3D_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!ctx->pending.empty()) prof_resolve(ctx);
    return IM3D_OK;
}

int check_dims(im3d_ctx* ctx, int nx, int ny, int nz, double hx, double hy, double hz)
{
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "dimensions must be positive");
    if (nz == 1)
        return fail(ctx, IM3D_ERR_UNSUPPORTED, "2-D volumes (nz == 1) are not supported by the "
                                               "GPU backend");
    if (nx < 3 || ny < 3 || nz < 3)
        return fail(ctx, IM3D_ERR_UNSUPPORTED, "every dimension must be at least 3 (the "
                                               "one-sided stencils read 3 points)");
    if (!(hx > 0) || !(hy > 0) || !(hz > 0))
        return fail(ctx, IM3D_ERR_INVALID_ARG, "spacings must be positive");
    if ((long long)nx * ny > 0x7fffffffLL || nx > 65535 || ny > 65535)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "volume too large for the launch geometry");
    return IM3D_OK;
}

dim3 grid_vol(const Dims& d, dim3 blk) { return dim3((d.nz + blk.x - 1) / blk.x, (d.ny + blk.y - 1) / blk.y, d.nx); }

const dim3 kBlkVol(32, 8, 1);

int flat_grid(long long n)
{
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

// ------------------------------------------------------------- Gaussian taps
// One axis of conv::filtering<T>::build_gaussian_filter (convolution_imp.hxx:22-80):
// Nh = ceil(2 radius sigma / h), made odd; g[t] = exp(-(t-S)^2 h^2 / (2 sigma^2)).
// The 3-D kernel normalised by its L1 norm is the product of these normalised 1-D
// kernels, so each axis is normalised to unit sum.
int gauss_taps_host(double sigma, double radius, double h, std::vector<double>& w)
{
    int nh = (int)std::ceil(2 * radius * sigma / h);
    if (nh % 2 == 0) nh++;
    if (nh > NH_MAX) return -1;
    int S = nh / 2;
    w.assign(nh, 0.0);
    double s = 0;
    for (int t = 0; t < nh; ++t) {
        double dd = (double)(t - S);
        w[t] = std::exp(-dd * dd * h * h / (2 * sigma * sigma));
        s += w[t];
    }
    for (int t = 0; t < nh; ++t) w[t] /= s;
    return nh;
}

template <typename T>
struct Taps {
    const T* w[3];
    int nh[3];
    T host[3][NH_MAX];  // the same taps on the host (kernels that take them by value)
};

template <typename T>
int upload_taps(im3d_ctx* ctx, const char* slot, double sigma, double radius, double hx, double hy,
                double hz, int pixel_approach, Taps<T>* out)
{
    if (!(sigma > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "sigma must be greater than zero");
    if (!(radius > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "radius must be greater than zero");
    const double hs[3] = {pixel_approach ? 1. : hx, pixel_approach ? 1. : hy,
                          pixel_approach ? 1. : hz};
    std::vector<T> host(3 * NH_MAX, T(0));
    int nh[3];
    for (int a = 0; a < 3; ++a) {
        std::vector<double> w;
        nh[a] = gauss_taps_host(sigma, radius, hs[a], w);
        if (nh[a] < 0)
            return fail(ctx, IM3D_ERR_UNSUPPORTED,
                        "Gaussian support exceeds " + std::to_string(NH_MAX) +
                            " taps (sigma*radius/h too large)");
        for (int t = 0; t < nh[a]; ++t) host[a * NH_MAX + t] = (T)w[t];
    }
    T* d = nullptr;
    IM3D_TRY(tbuf<T>(ctx, slot, 3 * NH_MAX, &d));
    IM3D_CUDA(ctx, cudaMemcpyAsync(d, host.data(), 3 * NH_MAX * sizeof(T), cudaMemcpyHostToDevice,
                                   ctx->stream));
    // the host vector must outlive the async copy
    IM3D_TRY(sync(ctx));
    for (int a = 0; a < 3; ++a) {
        out->w[a] = d + a * NH_MAX;
        out->nh[a] = nh[a];
        for (int t = 0; t < NH_MAX; ++t) out->host[a][t] = host[a * NH_MAX + t];
    }
    return IM3D_OK;
}

// --------------------------------------------------------- convolution passes
constexpr int TK = 128, RK = 2;
constexpr int TW = 32, TY = 8;
template <typename T> struct TileA { static constexpr int v = 64; };
template <> struct TileA<double> { static constexpr int v = 32; };

template <typename K>
int set_smem(im3d_ctx* ctx, K kernel, size_t bytes)
{
    if (bytes > 48 * 1024)
        IM3D_CUDA(ctx, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)bytes));
    return IM3D_OK;
}

// Register-window k pass: blocks of RKR rows x TKT threads, 4 RG outputs per thread.
constexpr int kKwT = 32, kKwR = 4;  // 4 rows per block: measured fastest (8: 6 % slower, 16: 13 %)
template <typename T, int N> struct KWinRG { static constexpr int v = 1; };
template <typename T, int N, int S>
constexpr size_t k_win_smem()
{
    return (size_t)N * kKwR * (kKwT * 4 * KWinRG<T, N>::v + 2 * ((S + 3) & ~3)) * sizeof(T);
}
template <typename T, int N>
dim3 k_win_grid(const Dims& d)
{
    constexpr int TK = kKwT * 4 * KWinRG<T, N>::v;
    const long long rows = (long long)d.nx * d.ny;
    return dim3((unsigned)((rows + kKwR - 1) / kKwR), (d.nz + TK - 1) / TK);
}

template <typename T, int N, int S, class Ld, class St>
int pass_k_win(im3d_ctx* ctx, Ld ld, St st, const Dims& d, const T* w, const char* name)
{
    constexpr int TKT = kKwT, RKR = kKwR;
    const size_t smem = k_win_smem<T, N, S>();
    auto kern = conv_k_win_kernel<T, N, S, TKT, RKR, Ld, St, KWinRG<T, N>::v>;
    IM3D_TRY(set_smem(ctx, kern, smem));
    const dim3 grid = k_win_grid<T, N>(d);
    const int pf = prof_begin(ctx, name);
    kern<<<grid, dim3(TKT, RKR), smem, ctx->stream>>>(ld, st, d, w);
    prof_end(ctx, pf);
    return check_launch(ctx, name);
}

template <typename T, int N, class Ld, class St>
int pass_k(im3d_ctx* ctx, Ld ld, St st, const Dims& d, const T* w, int nh,
           const char* name = "conv_k")
{
    if (nh == 19) return pass_k_win<T, N, 9>(ctx, ld, st, d, w, name);
    if (nh == 25) return pass_k_win<T, N, 12>(ctx, ld, st, d, w, name);
    const int S = nh / 2;
    size_t smem = (size_t)RK * (TK + 2 * S) * sizeof(Vec<T, N>) + nh * sizeof(T) + 16;
    auto kern = conv_k_kernel<T, N, TK, RK, Ld, St>;
    IM3D_TRY(set_smem(ctx, kern, smem));
    long long rows = (long long)d.nx * d.ny;
    dim3 grid((unsigned)((rows + RK - 1) / RK), (d.nz + TK - 1) / TK);
    const int pf = prof_begin(ctx, name);
    kern<<<grid, dim3(TK, RK), smem, ctx->stream>>>(ld, st, d, w, nh);
    prof_end(ctx, pf);
    return check_launch(ctx, name);
}

// ------------------------------------------- Heaviside pass with TMA-moved rows (FP32)
// cuTensorMapEncodeTiled of the driver, resolved once.
[[maybe_unused]] PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// Whether the TMA pass takes this volume: FP32 rows of a multiple of 8 cells, at most 256
// (one box), 16-byte aligned buffers, 19 or 25 taps.
[[maybe_unused]] inline bool heav_tma_eligible(const im3d_ctx* ctx, const Dims& d, int nh, const void* phi,
                                               const void* u0, const void* out)
{
    auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
    return ctx->tile_loads && (nh == 19 || nh == 25) && d.nz % 8 == 0 && d.nz <= 256 && al(phi) && al(u0) &&
           al(out) && (long long)d.nx * d.ny < (1ll << 31);
}

// The Heaviside pass (LdHeaviside + StVec<float, 4>) on conv_k_heav_tma_kernel, 4 rows per
// block (measured at 256^3: 4 rows as fast as conv_k_win_kernel or faster; 2 and 8 rows
// slower).
template <int S>
int pass_heav_tma(im3d_ctx* ctx, const float* phi, const float* u0, Vec<float, 4>* out, const Dims& d,
                  const float* taps, float center, float inv_eps, const char* name)
{
    constexpr int RB = 4;
    auto enc = tmap_encoder();
    if (!enc) return fail(ctx, IM3D_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const int KB = (d.nz + 15) & ~15;
    const long long rows = (long long)d.nx * d.ny;
    const size_t smem = HeavTmaLayout<RB, S>::total(KB);
    auto kern = conv_k_heav_tma_kernel<RB, S>;
    IM3D_TRY(set_smem(ctx, kern, smem));
    int occ = 0;
    IM3D_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, RB * 32, smem));
    if (occ < 1) return fail(ctx, IM3D_ERR_UNSUPPORTED, "the TMA Heaviside pass does not fit an SM");
    CUtensorMap mp, mu, mo;
    {
        cuuint64_t dims[2] = {(cuuint64_t)d.nz, (cuuint64_t)rows};
        cuuint64_t str[1] = {(cuuint64_t)d.nz * 4};
        cuuint32_t box[2] = {(cuuint32_t)KB, (cuuint32_t)RB};
        cuuint32_t es[2] = {1, 1};
        for (int f = 0; f < 2; ++f) {
            const CUresult r = enc(f ? &mu : &mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                                   const_cast<float*>(f ? u0 : phi), dims, str, box, es,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS)
                return fail(ctx, IM3D_ERR_CUDA, "cuTensorMapEncodeTiled (rows) failed: " + std::to_string((int)r));
        }
    }
    {
        // the output viewed as rows x (nz / 8) groups x 32 floats (8 cells of 4 fields)
        cuuint64_t dims[3] = {32, (cuuint64_t)(d.nz / 8), (cuuint64_t)rows};
        cuuint64_t str[2] = {128, (cuuint64_t)d.nz * 16};
        cuuint32_t box[3] = {32, (cuuint32_t)(KB / 8), (cuuint32_t)RB};
        cuuint32_t es[3] = {1, 1, 1};
        const CUresult r = enc(&mo, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, reinterpret_cast<float*>(out), dims, str,
                               box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            return fail(ctx, IM3D_ERR_CUDA, "cuTensorMapEncodeTiled (cells) failed: " + std::to_string((int)r));
    }
    HeavTmaArgs a;
    a.d = d;
    a.taps = taps;
    a.center = center;
    a.inv_eps = inv_eps;
    a.KB = KB;
    a.nrb = (rows + RB - 1) / RB;
    a.err = &ctx->ctrl_d->flag[0];
    const long long G = std::min<long long>(a.nrb, (long long)occ * ctx->num_sms);
    const int pf = prof_begin(ctx, name);
    kern<<<(unsigned)G, RB * 32, smem, ctx->stream>>>(mp, mu, mo, a);
    prof_end(ctx, pf);
    return check_launch(ctx, name);
}

// Register-window j / i pass: TW x TY blocks, R outputs per thread along the axis.
template <typename T> struct SWinR { static constexpr int v = sizeof(T) == 4 ? 8 : 4; };
template <typename T, int N, int S>
constexpr size_t s_win_smem() { return (size_t)N * (TY * SWinR<T>::v + 2 * S) * TW * sizeof(T); }
template <typename T, int AXIS>
dim3 s_win_grid(const Dims& d)
{
    constexpr int TA = TY * SWinR<T>::v;
    const int len = AXIS == 0 ? d.nx : d.ny;
    const int other = AXIS == 0 ? d.ny : d.nx;
    return dim3((d.nz + TW - 1) / TW, (len + TA - 1) / TA, other);
}

template <typename T, int N, int AXIS, int S, class Ld, class St>
int pass_s_win(im3d_ctx* ctx, Ld ld, St st, const Dims& d, const T* w, const char* name)
{
    constexpr int R = SWinR<T>::v;
    const size_t smem = s_win_smem<T, N, S>();
    const dim3 grid = s_win_grid<T, AXIS>(d);
    auto run = [&](auto kern) -> int {
        IM3D_TRY(set_smem(ctx, kern, smem));
        const int pf = prof_begin(ctx, name);
        kern<<<grid, dim3(TW, TY), smem, ctx->stream>>>(ld, st, d, w);
        prof_end(ctx, pf);
        return check_launch(ctx, name);
    };
    if constexpr (kPairedS<T, N>)
        return run(conv_s_win_pair_kernel<T, N, AXIS, S, TW, TY, R, Ld, St>);
    else
        return run(conv_s_win_kernel<T, N, AXIS, S, TW, TY, R, Ld, St>);
}

template <typename T, int N, int AXIS, class Ld, class St>
int pass_s(im3d_ctx* ctx, Ld ld, St st, const Dims& d, const T* w, int nh,
           const char* name = AXIS == 0 ? "conv_s_i" : "conv_s_j")
{
    if (nh == 19) return pass_s_win<T, N, AXIS, 9>(ctx, ld, st, d, w, name);
    if (nh == 25) return pass_s_win<T, N, AXIS, 12>(ctx, ld, st, d, w, name);
    constexpr int TA = TileA<T>::v;
    const int S = nh / 2;
    size_t smem = (size_t)(TA + 2 * S) * TW * sizeof(Vec<T, N>) + nh * sizeof(T) + 16;
    auto kern = conv_s_kernel<T, N, AXIS, TW, TY, TA, Ld, St>;
    IM3D_TRY(set_smem(ctx, kern, smem));
    const int len = AXIS == 0 ? d.nx : d.ny;
    const int other = AXIS == 0 ? d.ny : d.nx;
    dim3 grid((d.nz + TW - 1) / TW, (len + TA - 1) / TA, other);
    const int pf = prof_begin(ctx, name);
    kern<<<grid, dim3(TW, TY), smem, ctx->stream>>>(ld, st, d, w, nh);
    prof_end(ctx, pf);
    return check_launch(ctx, name);
}

template <typename T, int S>
constexpr size_t fit_win_smem()
{
    constexpr int TA = TileA<T>::v;
    constexpr int RA = (TA + 2 * S + TY - 1) / TY;
    constexpr int H2 = TY * RA, H1 = H2 + 2 * S;
    return (size_t)(4 * H1 + 2 * H2) * TW * sizeof(T);
}
template <typename T>
dim3 fit_win_grid(const Dims& d)
{
    return dim3((d.nz + TW - 1) / TW, (d.nx + TileA<T>::v - 1) / TileA<T>::v, d.ny);
}

template <typename T, int S>
int pass_i_fit_win(im3d_ctx* ctx, const Vec<T, 4>* in, Vec<T, 2>* out, T* f1, T* f2,
                   const Dims& d, const T* w, T l1, T l2)
{
    constexpr int TA = TileA<T>::v;
    const size_t smem = fit_win_smem<T, S>();
    auto kern = conv_i_fit_win_kernel<T, S, TW, TY, TA>;
    IM3D_TRY(set_smem(ctx, kern, smem));
    const dim3 grid = fit_win_grid<T>(d);
    const int pf = prof_begin(ctx, "conv_i_fit");
    kern<<<grid, dim3(TW, TY), smem, ctx->stream>>>(in, out, f1, f2, d, w, l1, l2);
    prof_end(ctx, pf);
    return check_launch(ctx, "conv_i_fit");
}

// Marching i-stage (FP32): one (j, k) column per thread, chunks of i per blockIdx.z.
// The kernel is issue-bound, so the chunk count minimises the planes one SM streams:
// ceil(blocks / SMs) x (chunk + 4S), where each chunk re-streams 4S halo planes
// (measured at 256^3: 1, 2, 3, 4 chunks take 152, 144, 160, 164 us; this picks 2).
// The context option IM3D_OPT_FIT_CHUNKS overrides it.
// 4 blocks of 128 threads per SM for 19 taps (126 registers, no spills); 2 for 25
// taps (3 would spill)
constexpr int kMarchJB = 4, kMarchD = 16, kMarchU = 4;
template <int S> struct MarchMinB { static constexpr int v = S <= 9 ? 4 : 2; };

// planes of i per block of the marching i-stage, and its grid
template <int S>
int march_chunk(const im3d_ctx* ctx, const Dims& d, dim3* grid)
{
    constexpr int JB = kMarchJB;
    const long long cols = (long long)((d.nz + 31) / 32) * ((d.ny + JB - 1) / JB);
    int chunks = ctx->ifit_chunks;
    if (chunks <= 0) {
        long long best = 0;
        for (int c = 1; c <= 8 && c <= d.nx; ++c) {
            const int chunk = (d.nx + c - 1) / c;
            const long long per_sm = (cols * c + ctx->num_sms - 1) / ctx->num_sms;
            const long long cost = per_sm * (chunk + 4 * S);
            if (c == 1 || cost < best) {
                best = cost;
                chunks = c;
            }
        }
    }
    chunks = std::min(chunks, d.nx);
    const int chunk = (d.nx + chunks - 1) / chunks;
    *grid = dim3((d.nz + 31) / 32, (d.ny + JB - 1) / JB, (d.nx + chunk - 1) / chunk);
    return chunk;
}

template <int S>
TapPairs<S> tap_pairs(const float* hw)
{
    TapPairs<S> tp;
    for (int t = 0; t <= S; ++t) tp.w[t] = make_float2(hw[t], hw[t]);
    return tp;
}

template <int S>
int pass_i_fit_march(im3d_ctx* ctx, const Vec<float, 4>* in, Vec<float, 2>* out, float* f1,
                     float* f2, const Dims& d, const float* hw, float l1, float l2)
{
    constexpr int JB = kMarchJB, D = kMarchD, U = kMarchU, MINB = MarchMinB<S>::v;
    auto kern = conv_i_fit_march_kernel<S, JB, D, U, MINB>;
    dim3 grid;
    const int chunk = march_chunk<S>(ctx, d, &grid);
    const TapPairs<S> tp = tap_pairs<S>(hw);
    const int pf = prof_begin(ctx, "conv_i_fit");
    kern<<<grid, dim3(32, JB), 0, ctx->stream>>>(reinterpret_cast<const float4*>(in),
                                                 reinterpret_cast<float2*>(out), f1, f2, d, tp,
                                                 l1, l2, chunk);
    prof_end(ctx, pf);
    return check_launch(ctx, "conv_i_fit");
}

template <typename T>
int pass_i_fit(im3d_ctx* ctx, const Vec<T, 4>* in, Vec<T, 2>* out, T* f1, T* f2, const Dims& d,
               const T* w, const T* hw, int nh, T l1, T l2)
{
    if constexpr (sizeof(T) == 4) {
        if (nh == 19) return pass_i_fit_march<9>(ctx, in, out, f1, f2, d, hw, l1, l2);
        if (nh == 25) return pass_i_fit_march<12>(ctx, in, out, f1, f2, d, hw, l1, l2);
    }
    if (nh == 19) return pass_i_fit_win<T, 9>(ctx, in, out, f1, f2, d, w, l1, l2);
    if (nh == 25) return pass_i_fit_win<T, 12>(ctx, in, out, f1, f2, d, w, l1, l2);
    constexpr int TA = TileA<T>::v;
    const int S = nh / 2;
    size_t smem = (size_t)(TA + 4 * S) * TW * sizeof(Vec<T, 4>) +
                  (size_t)(TA + 2 * S) * TW * sizeof(Vec<T, 2>) + nh * sizeof(T) + 16;
    auto kern = conv_i_fit_kernel<T, TW, TY, TA>;
    IM3D_TRY(set_smem(ctx, kern, smem));
    dim3 grid((d.nz + TW - 1) / TW, (d.nx + TA - 1) / TA, d.ny);
    const int pf = prof_begin(ctx, "conv_i_fit");
    kern<<<grid, dim3(TW, TY), smem, ctx->stream>>>(in, out, f1, f2, d, w, nh, l1, l2);
    prof_end(ctx, pf);
    return check_launch(ctx, "conv_i_fit");
}

// Scalar Gaussian filter: in -> out through the three passes (tmp1, tmp2 scratch).
template <typename T, class Ld>
int gauss_scalar(im3d_ctx* ctx, Ld ld, T* out, const Dims& d, const Taps<T>& tp)
{
    Vec<T, 1>* t1 = nullptr;
    Vec<T, 1>* t2 = nullptr;
    IM3D_TRY(tbuf<Vec<T, 1>>(ctx, "gs_tmp1", d.n(), &t1));
    IM3D_TRY(tbuf<Vec<T, 1>>(ctx, "gs_tmp2", d.n(), &t2));
    IM3D_TRY((pass_k<T, 1>(ctx, ld, StVec<T, 1>{t1, d}, d, tp.w[2], tp.nh[2])));
    IM3D_TRY((pass_s<T, 1, 1>(ctx, LdVec<T, 1>{t1, d}, StVec<T, 1>{t2, d}, d, tp.w[1], tp.nh[1])));
    IM3D_TRY((pass_s<T, 1, 0>(ctx, LdVec<T, 1>{t2, d}, StScalar<T>{out, d}, d, tp.w[0], tp.nh[0])));
    return IM3D_OK;
}

// -------------------------------------------------------------- Gauss-Seidel
template <typename T>
GsCoef<T> make_coef(double hx, double hy, double hz, double dt, double bc, int neu)
{
    GsCoef<T> c;
    c.hx = hx; c.hy = hy; c.hz = hz; c.dt = dt;
    c.ihx2 = (T)(1.0 / (hx * hx));
    c.ihy2 = (T)(1.0 / (hy * hy));
    c.ihz2 = (T)(1.0 / (hz * hz));
    c.idt = (T)(1.0 / dt);
    for (int m = 0; m < 8; ++m) {
        // poisson_imp.hxx:115-139 / :398: htilde = 1/(1/dt + c_x/hx^2 + c_y/hy^2 + c_z/hz^2)
        double cx = (m & 1) ? 2. : 1., cy = (m & 2) ? 2. : 1., cz = (m & 4) ? 2. : 1.;
        double ht = 1. / dt + cx / (hx * hx) + cy / (hy * hy) + cz / (hz * hz);
        c.htilde[m] = (T)(1. / ht);
        c.htilde_lo[m] = sizeof(T) == 4 ? (T)(1. / ht - (double)c.htilde[m]) : T(0);
    }
    // oblique normals of NeuGaussSeidel (poisson_imp.hxx:155-159): 1, 1/sqrt2, 1/sqrt3
    const T tb = (T)bc;
    T ne = T(1); ne /= (T)std::sqrt(2.);
    T na = T(1); na /= (T)std::sqrt(3.);
    c.bcn[0] = tb; c.bcn[1] = tb; c.bcn[2] = ne * tb; c.bcn[3] = na * tb;
    for (int q = 0; q < 4; ++q) c.bcnd[q] = (double)c.bcn[q];
    c.bc = tb;
    c.neu = neu;
    c.ihx2d = 1.0 / (hx * hx);
    c.ihy2d = 1.0 / (hy * hy);
    c.ihz2d = 1.0 / (hz * hz);
    c.diagd = 1.0 / dt + 2.0 * c.ihx2d + 2.0 * c.ihy2d + 2.0 * c.ihz2d;
    return c;
}

// One lexicographic sweep, reference order, natural layout, in place.
template <typename T>
int lex_sweep(im3d_ctx* ctx, T* r, const T* b, const Dims& d, const GsCoef<T>& c)
{
    if (!c.neu) {
        dir_faces_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(r, d, c.bc);
        IM3D_TRY(check_launch(ctx, "dir_faces"));
    }
    const int lo = c.neu ? 0 : 1;
    const int hix = d.nx - lo, hiy = d.ny - lo, hiz = d.nz - lo;
    if (hix <= lo || hiy <= lo || hiz <= lo) return IM3D_OK;
    const dim3 blk(32, 4);
    const int pf = prof_begin(ctx, "lex_sweep");
    for (int s = 3 * lo; s <= (hix - 1) + (hiy - 1) + (hiz - 1); ++s) {
        const int i0 = std::max(lo, s - (hiy - 1) - (hiz - 1));
        const int i1 = std::min(hix - 1, s - 2 * lo);
        if (i0 > i1) continue;
        const int j0 = std::max(lo, s - i1 - (hiz - 1));
        const int j1 = std::min(hiy - 1, s - i0 - lo);
        if (j0 > j1) continue;
        dim3 grid((j1 - j0 + 1 + blk.x - 1) / blk.x, (i1 - i0 + 1 + blk.y - 1) / blk.y);
        lex_plane_kernel<T><<<grid, blk, 0, ctx->stream>>>(r, b, d, c, s, lo, i0, j0);
        IM3D_TRY(check_launch(ctx, "lex_plane"));
    }
    prof_end(ctx, pf);
    return IM3D_OK;
}

constexpr int kNI = 8;  // planes per thread of the scalar column-marching kernels
constexpr int kNV = 2;  // planes per thread of the vectorised kernels (measured best on B200)
constexpr int kNVres = 2;  // planes per thread of the residual check
const dim3 kBlkVec(32, 4, 1);

// half-sweep and residual grid: the (vector group, row) pairs of a plane flattened over
// x blocks
template <typename T>
dim3 grid_rb_flat(const Dims& d, dim3 blk, int zmul = 1, int ni = kNV)
{
    const long long pairs = (long long)(d.hz() / V16<T>::W) * d.ny;
    const long long per = (long long)blk.x * blk.y;
    return dim3((unsigned)((pairs + per - 1) / per), 1, ((d.nx + ni - 1) / ni) * zmul);
}

// natural-layout vectorised kernels: (vector group, row) pairs flattened over x blocks
template <typename T>
dim3 grid_vec(const Dims& d, dim3 blk)
{
    const long long pairs = (long long)(d.nz / V16<T>::W) * d.ny;
    const long long per = (long long)blk.x * blk.y;
    return dim3((unsigned)((pairs + per - 1) / per), 1, (d.nx + kNV - 1) / kNV);
}

dim3 grid_col(const Dims& d, dim3 blk, int ni = kNI)
{
    return dim3((d.nz + blk.x - 1) / blk.x, (d.ny + blk.y - 1) / blk.y, (d.nx + ni - 1) / ni);
}

// planes per thread of the column Bregman kernel (it holds every load of its planes)
constexpr int kNIbr = 2;

// Launch as a programmatic dependent of the previous kernel on the stream: the kernel
// must begin with griddepcontrol.wait (rb_half_vec_kernel does), which holds it until
// the previous grid's writes are visible.
template <typename... KArgs, typename... Args>
int launch_dependent(im3d_ctx* ctx, void (*kern)(KArgs...), dim3 grid, dim3 blk, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = blk;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    IM3D_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
    return IM3D_OK;
}

// Whether every cell offset of the solve's two colour-packed fields fits an int (the
// half-sweep and the residual check then take 32-bit offsets: fewer instructions per
// address; the streaming kernels measured no gain or a loss from it).
inline bool fits_int32(const Dims& d)
{
    return 2 * d.npk() < (1ll << 31);
}

template <typename T>
int rb_sweep(im3d_ctx* ctx, T* U, const T* B, const Dims& d, const GsCoef<T>& c, int use_self,
             double omega)
{
    // the b_eff solve (no own value, omega 1) gets instantiations without the unused
    // paths; with Dirichlet conditions and FP32 it fits 8 blocks per SM
    const bool self = use_self || omega != 1.0;
    const dim3 grid = grid_rb_flat<T>(d, kBlkVec);
    for (int color = 0; color < 2; ++color) {
        const int pf = prof_begin(ctx, "rb_half");
        // red walks the planes forward, black backward: each half-sweep starts on the
        // planes the previous one wrote last, which are still in L2
        const int reverse = color;
        if (self)
            IM3D_TRY(launch_dependent(ctx, rb_half_vec_kernel<T, kNV, true, true>, grid, kBlkVec, U,
                                      B, d, c, color, use_self, (T)omega, reverse));
        else if (c.neu)
            IM3D_TRY(launch_dependent(ctx, rb_half_vec_kernel<T, kNV, false, true>, grid, kBlkVec,
                                      U, B, d, c, color, 0, T(1), reverse));
        else if (fits_int32(d))
            IM3D_TRY(launch_dependent(ctx, rb_half_vec_kernel<T, kNV, false, false, sizeof(T) == 4 ? 8 : 1, int>,
                                      grid, kBlkVec, U, B, d, c, color, 0, T(1), reverse));
        else
            IM3D_TRY(launch_dependent(ctx, rb_half_vec_kernel<T, kNV, false, false, sizeof(T) == 4 ? 8 : 1>,
                                      grid, kBlkVec, U, B, d, c, color, 0, T(1), reverse));
        prof_end(ctx, pf);
        IM3D_TRY(check_launch(ctx, "rb_half"));
    }
    return IM3D_OK;
}

// Per-block partial sums of a reduction launch (nvals values per block).
int part_buf(im3d_ctx* ctx, dim3 grid, int nvals, double** out)
{
    const long long nb = (long long)grid.x * grid.y * grid.z;
    return tbuf<double>(ctx, "partials", (size_t)(nb * nvals), out);
}

// Folds the partials of the last reduction launch into ctrl->sum[slot .. slot+nvals).
int finalize(im3d_ctx* ctx, const double* part, dim3 grid, int nvals, int slot)
{
    const long long nb = (long long)grid.x * grid.y * grid.z;
    finalize_sums_kernel<<<1, kFinThreads, 0, ctx->stream>>>(part, nb, nvals, ctx->ctrl_d->sum, slot);
    return check_launch(ctx, "finalize_sums");
}

// Next residual check of the Poisson solve. check_every > 0: a fixed interval.
// Otherwise the remaining sweeps are predicted from the contraction rate,
//   need = log(tol / r_s) / log(rate),
// and the next check is ceil(need) sweeps later, clamped to [1, 32]. The rate is
// (r_s / r_prev)^(1/(s - s_prev)) once two residuals of this solve are known, else the
// rate carried over from the previous solve (rate_hint in (0, 1)), else the next
// check is 4 sweeps later. *rate_used receives the rate a prediction used.
int next_check(int s, double r_s, int s_prev, double r_prev, double tol, int check_every,
               double rate_hint, double* rate_used)
{
    if (check_every > 0) return s + check_every;
    double rate;
    if (s_prev > 0 && r_prev > r_s && r_s > 0) rate = std::pow(r_s / r_prev, 1.0 / (double)(s - s_prev));
    else if (rate_hint > 0 && rate_hint < 1 && r_s > 0) rate = rate_hint;
    else return s + 4;
    *rate_used = rate;
    const double need = std::log(tol / r_s) / std::log(rate);
    int step = 32;
    if (need == need && need < 32.0) step = (int)std::ceil(need);
    if (step < 1) step = 1;
    return s + step;
}

int zero_ctrl(im3d_ctx* ctx)
{
    IM3D_CUDA(ctx, cudaMemsetAsync(ctx->ctrl_d, 0, sizeof(Ctrl), ctx->stream));
    return IM3D_OK;
}

int read_ctrl(im3d_ctx* ctx)
{
    IM3D_CUDA(ctx, cudaMemcpyAsync(ctx->ctrl_h, ctx->ctrl_d, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                                   ctx->stream));
    return sync(ctx);
}

// FP64 residual of the packed state, and sum b_eff^2 on the first call (*beff2 < 0);
// returns the relative residual in *rel.
template <typename T>
int rb_check(im3d_ctx* ctx, const T* U, const T* B, const Dims& d, const GsCoef<T>& c,
             double* beff2, double* rel)
{
    const dim3 grid = grid_rb_flat<T>(d, kBlkVec, 2, kNVres);
    const int nvals = *beff2 < 0 ? 2 : 1;
    double* part = nullptr;
    IM3D_TRY(part_buf(ctx, grid, nvals, &part));
    ctx->residual_checks++;
    const int pf = prof_begin(ctx, "rb_residual");
    if (fits_int32(d))
        rb_residual_vec_kernel<T, kNVres, int><<<grid, kBlkVec, 0, ctx->stream>>>(U, B, d, c, part, nvals == 2 ? 1 : 0);
    else
        rb_residual_vec_kernel<T, kNVres><<<grid, kBlkVec, 0, ctx->stream>>>(U, B, d, c, part, nvals == 2 ? 1 : 0);
    prof_end(ctx, pf);
    IM3D_TRY(check_launch(ctx, "rb_residual"));
    IM3D_TRY(finalize(ctx, part, grid, nvals, SUM_RES2));
    IM3D_TRY(read_ctrl(ctx));
    if (*beff2 < 0) *beff2 = ctx->ctrl_h->sum[SUM_BEFF2];
    const double rr = ctx->ctrl_h->sum[SUM_RES2];
    *rel = *beff2 > 0 ? std::sqrt(rr) / std::sqrt(*beff2) : std::sqrt(rr);
    return IM3D_OK;
}

// Red-black solve on the packed layout (U holds u_in on entry, B = b_eff packed).
// Residual on the schedule of next_check, the first one after first_check sweeps
// (0: after 4); sum b_eff^2 is taken on the first check. *rate_out (may be NULL)
// receives the last contraction rate the schedule used (rate_hint if none), so that
// the next solve of a segmentation can start from it.
template <typename T>
int rb_solve(im3d_ctx* ctx, T* U, const T* B, const Dims& d, const GsCoef<T>& c, double tol,
             int max_sweeps, int check_every, double omega, int* sweeps, double* rel, bool* conv,
             int first_check = 0, double rate_hint = 0, double* rate_out = nullptr)
{
    if (check_every < 0) check_every = 0;
    if (max_sweeps < 1) max_sweeps = 1;
    double beff2 = -1;
    int s = 0, s_prev = 0;
    double r_prev = -1, rate_used = 0;
    int next = check_every > 0 ? check_every : (first_check > 0 ? first_check : 4);
    if (rate_out) *rate_out = rate_hint;
    *conv = false;
    *rel = -1;
    while (s < max_sweeps) {
        IM3D_TRY(rb_sweep(ctx, U, B, d, c, 0, omega));
        ++s;
        if (s >= next || s == max_sweeps) {
            double r = 0;
            IM3D_TRY(rb_check<T>(ctx, U, B, d, c, &beff2, &r));
            *rel = r;
            if (r <= tol) {
                *conv = true;
                break;
            }
            next = next_check(s, r, s_prev, r_prev, tol, check_every, rate_hint, &rate_used);
            if (next > max_sweeps) next = max_sweeps;
            s_prev = s;
            r_prev = r;
        }
    }
    if (rate_out) *rate_out = rate_used > 0 ? rate_used : rate_hint;
    *sweeps = s;
    return IM3D_OK;
}

// Exact minimum and maximum of a device volume (FP64 order keys of the values).
double order_key_to_double(unsigned long long k)
{
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double v;
    std::memcpy(&v, &b, sizeof v);
    return v;
}

// *nonfinite (may be NULL) receives whether any value is NaN or Inf.
template <typename T>
int minmax(im3d_ctx* ctx, const T* p, long long n, T* mn, T* mx, bool* nonfinite = nullptr)
{
    IM3D_CUDA(ctx, cudaMemsetAsync(ctx->ctrl_d->umax, 0, 4 * sizeof(unsigned long long), ctx->stream));
    minmax_kernel<T><<<flat_grid(n), 256, 0, ctx->stream>>>(p, n, ctx->ctrl_d->umax);
    IM3D_TRY(check_launch(ctx, "minmax"));
    IM3D_TRY(read_ctrl(ctx));
    *mx = (T)order_key_to_double(ctx->ctrl_h->umax[0]);
    *mn = (T)(-order_key_to_double(ctx->ctrl_h->umax[1]));
    if (nonfinite) *nonfinite = ctx->ctrl_h->umax[3] != 0;
    return IM3D_OK;
}

// image3d<T>::connected_component (image3d_imp.hxx:1694-2120) on device buffers; res
// may be img (the result is written element by element after the last read).
template <typename T>
int cc_run(im3d_ctx* ctx, const T* img, T* res, const Dims& d, const T* init, int i, int j, int k,
           double threshold, int full, int binary, int* passes)
{
    const long long n = d.n();
    T mn, mx;
    IM3D_TRY(minmax<T>(ctx, img, n, &mn, &mx));
    if (threshold > 1 || threshold < 0) {
        ctx->err = "WARNING::im_to_black_and_white: threshold must be between 0 and 1, "
                   "otherwise default value 0.5 is applied";
        threshold = 0.5;
    }
    // pivot (min + (max - min) * threshold), the difference in T (image3d_imp.hxx:1603)
    const T span = mx - mn;
    const T pivot = (T)((double)mn + (double)span * threshold);
    int negative = 0;
    long long seed = -1;
    if (!init) {
        // the seed moved off the faces (:1700-1736)
        unsigned I = (unsigned)i, J = (unsigned)j, K = (unsigned)k;
        if (I == 0) ++I;
        if (J == 0) ++J;
        if (I >= (unsigned)d.nx - 1) I = d.nx - 2;
        if (J >= (unsigned)d.ny - 1) J = d.ny - 2;
        if (d.nz == 1) {
            K = 0;
        } else {
            if (K == 0) ++K;
            if (K >= (unsigned)d.nz - 1) K = d.nz - 2;
        }
        seed = d.idx((int)I, (int)J, (int)K);
        T v;
        IM3D_CUDA(ctx, cudaMemcpyAsync(&v, img + seed, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
        IM3D_TRY(sync(ctx));
        negative = v < pivot;  // a dark seed: the component of the negative image (:1740-1745)
    }
    unsigned char* m0 = nullptr;
    unsigned char* m1 = nullptr;
    IM3D_TRY(tbuf<unsigned char>(ctx, "cc_mask0", (size_t)n, &m0));
    IM3D_TRY(tbuf<unsigned char>(ctx, "cc_mask1", (size_t)n, &m1));
    cc_init_kernel<T><<<flat_grid(n), 256, 0, ctx->stream>>>(img, init, m0, n, pivot, negative, seed);
    IM3D_TRY(check_launch(ctx, "cc_init"));
    const dim3 grid((d.nz + kCcK - 1) / kCcK, (d.ny + kCcJ - 1) / kCcJ, (d.nx + kCcI - 1) / kCcI);
    const dim3 blk(kCcK, kCcJ);
    unsigned long long* flag = ctx->ctrl_d->umax + 2;
    long long np = 0;
    for (;;) {
        IM3D_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(unsigned long long), ctx->stream));
        for (int r = 0; r < 4; ++r) {
            const int pf = prof_begin(ctx, "cc_grow");
            if (full) cc_grow_kernel<true><<<grid, blk, 0, ctx->stream>>>(m0, m1, d, flag);
            else cc_grow_kernel<false><<<grid, blk, 0, ctx->stream>>>(m0, m1, d, flag);
            prof_end(ctx, pf);
            IM3D_TRY(check_launch(ctx, "cc_grow"));
            std::swap(m0, m1);
            ++np;
        }
        IM3D_TRY(read_ctrl(ctx));
        if (ctx->ctrl_h->umax[2] == 0) break;
        // every pass that does not end the loop adds a cell
        if (np > n + 8) return fail(ctx, IM3D_ERR_CUDA, "connected_component: no fixed point");
    }
    cc_output_kernel<T><<<flat_grid(n), 256, 0, ctx->stream>>>(m0, img, res, n, binary, mn, pivot);
    IM3D_TRY(check_launch(ctx, "cc_output"));
    if (passes) *passes = (int)(np < 0x7fffffff ? np : 0x7fffffff);
    return IM3D_OK;
}

template <typename T>
int connected_component_op(im3d_ctx* ctx, const T* img_user, T* res_user, int nx, int ny, int nz,
                           const T* init_user, int i, int j, int k, double threshold, int full,
                           int binary, int* passes)
{
    if (!img_user || !res_user) return fail(ctx, IM3D_ERR_INVALID_ARG, "NULL volume");
    if (nx < 2 || ny < 2 || nz < 1)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "connected_component needs nx, ny >= 2 and nz >= 1");
    if ((long long)nx * ny > 0x7fffffffLL || nx > 262000 || ny > 524000)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "volume too large for the launch geometry");
    ctx->err.clear();
    const Dims d{nx, ny, nz};
    const T* img = nullptr;
    const T* init = nullptr;
    T* res = nullptr;
    IM3D_TRY(dev_in<T>(ctx, img_user, d.n(), "in_a", &img));
    if (init_user) IM3D_TRY(dev_in<T>(ctx, init_user, d.n(), "in_b", &init));
    IM3D_TRY(dev_out<T>(ctx, res_user, d.n(), "out_a", &res));
    IM3D_TRY(cc_run<T>(ctx, img, res, d, init, i, j, k, threshold, full, binary, passes));
    IM3D_TRY(out_finish<T>(ctx, res_user, res, d.n()));
    return sync(ctx);
}

// extract_connected_component, automatic case (rsfe_splitbregman_imp.hxx:448-536), on
// the clamped level set: *replaced = true when phi became its (rescaled) component.
template <typename T>
int extract_cc(im3d_ctx* ctx, T* phi, const Dims& d, double hx, double hy, double hz,
               const im3d_rsfe_params* p, bool* replaced)
{
    *replaced = false;
    const int i = (int)std::floor(p->cc_init_pixel_x / hx);
    const int j = (int)std::floor(p->cc_init_pixel_y / hy);
    const int k = (int)std::floor(p->cc_init_pixel_z / hz);
    if (i < 0 || j < 0 || (d.nz != 1 && k < 0)) return IM3D_OK;
    const unsigned I = (unsigned)i, J = (unsigned)j, K = (unsigned)k;
    if (I > (unsigned)d.nx - 1 || J > (unsigned)d.ny - 1 || (d.nz != 1 && K > (unsigned)d.nz - 1))
        return IM3D_OK;
    // white at the seed after im_to_black_and_white(phi, (alpha - a0) / (b0 - a0)), in T
    const T alpha = (T)p->alpha, a0 = (T)p->a0, b0 = (T)p->b0;
    double thr = (double)((alpha - a0) / (b0 - a0));
    if (thr > 1 || thr < 0) thr = 0.5;
    T mn, mx;
    IM3D_TRY(minmax<T>(ctx, phi, d.n(), &mn, &mx));
    const T span = mx - mn;
    const T pivot = (T)((double)mn + (double)span * thr);
    T v;
    IM3D_CUDA(ctx, cudaMemcpyAsync(&v, phi + d.idx((int)I, (int)J, (int)K), sizeof(T),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    IM3D_TRY(sync(ctx));
    if (v < pivot) return IM3D_OK;
    // phi = connected_component(phi, I, J, K, 0.5, face connectivity, cc_binary_output)
    IM3D_TRY(cc_run<T>(ctx, phi, phi, d, nullptr, (int)I, (int)J, (int)K, 0.5, 0,
                       p->cc_binary_output, nullptr));
    // change_range_of_intensity(b0, a0) (image3d_imp.hxx:1628-1636)
    T cmn, cmx;
    IM3D_TRY(minmax<T>(ctx, phi, d.n(), &cmn, &cmx));
    const T shifted_max = cmx - cmn;
    const T sc = shifted_max / (b0 - a0);
    affine_kernel<T><<<flat_grid(d.n()), 256, 0, ctx->stream>>>(phi, d.n(), cmn, sc, a0);
    IM3D_TRY(check_launch(ctx, "affine"));
    *replaced = true;
    return IM3D_OK;
}

// ------------------------------------------------------- learned warm start
// The fields of one solve, gathered for the network (FP32 only).
struct WsBufs {
    float* x;      // 4 input volumes
    float* y;      // the network's correction / the training target
    float* upk0;   // the solve's start (packed u_in)
};

int ws_status(im3d_ctx* ctx, int st)
{
    if (st != IM3D_OK && ctx->err.empty()) ctx->err = "learned warm start failed";
    return st;
}

// Before a solve: IM3D_WS_PREDICT adds the network's correction to u_in when that
// lowers the residual; both modes keep u_in in w.upk0. (FP32 entry points only.)
[[maybe_unused]] int ws_before(im3d_ctx* ctx, const Dims& d, const GsCoef<float>& c, float* upk,
                               const float* bpk, const float* prevu, const float* divdb,
                               const float* phi, float inv_dt, int dirichlet, const WsBufs& w,
                               int* used, int* rejected)
{
    ws_fields_kernel<<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(bpk, upk, prevu, divdb, phi, d, inv_dt, w.x);
    IM3D_TRY(check_launch(ctx, "ws_fields"));
    IM3D_CUDA(ctx, cudaMemcpyAsync(w.upk0, upk, 2 * (size_t)d.npk() * sizeof(float), cudaMemcpyDeviceToDevice,
                                   ctx->stream));
    if (ctx->ws_mode != IM3D_WS_PREDICT) return IM3D_OK;
    const int pf = prof_begin(ctx, "ws_network");
    const long long l0 = im3d::unet::launch_total();
    IM3D_TRY(ws_status(ctx, im3d::unet::net_forward_fields(ctx->ws_net, ctx->stream, w.x, 1, d.nx, d.ny, d.nz, w.y,
                                                            ctx->err)));
    ctx->launches += im3d::unet::launch_total() - l0;
    prof_end(ctx, pf);
    double beff2 = -1, r0 = 0, r1 = 0;
    IM3D_TRY(rb_check<float>(ctx, upk, bpk, d, c, &beff2, &r0));
    ws_apply_kernel<<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(upk, w.y, d, dirichlet);
    IM3D_TRY(check_launch(ctx, "ws_apply"));
    IM3D_TRY(rb_check<float>(ctx, upk, bpk, d, c, &beff2, &r1));
    if (r1 < r0) {
        ++*used;
    } else {
        IM3D_CUDA(ctx, cudaMemcpyAsync(upk, w.upk0, 2 * (size_t)d.npk() * sizeof(float), cudaMemcpyDeviceToDevice,
                                       ctx->stream));
        ++*rejected;
    }
    return IM3D_OK;
}

// After a solve (IM3D_WS_TRAIN): one training step on the solve's fields and the
// correction it made. (FP32 entry points only.)
[[maybe_unused]] int ws_after(im3d_ctx* ctx, const Dims& d, const float* upk, const WsBufs& w,
                              double* loss)
{
    ws_target_kernel<<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(upk, w.upk0, d, w.y);
    IM3D_TRY(check_launch(ctx, "ws_target"));
    const int pf = prof_begin(ctx, "ws_train");
    const long long l0 = im3d::unet::launch_total();
    IM3D_TRY(ws_status(ctx, im3d::unet::net_train_fields(ctx->ws_net, ctx->stream, w.x, w.y, nullptr, 1, d.nx, d.ny,
                                                          d.nz, ctx->ws_lr, loss, nullptr, ctx->err)));
    ctx->launches += im3d::unet::launch_total() - l0;
    prof_end(ctx, pf);
    return IM3D_OK;
}

// --------------------------------------------------------------- the loop
// The setters' checks (rsfe_splitbregman_imp.hxx:806-1440), with their WARNING texts.
int check_params(im3d_ctx* ctx, const im3d_rsfe_params* p)
{
    if (!(p->sigma > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_sigma: sigma must be greater than zero");
    if (!(p->lamda > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_lamda: lamda must be greater than zero");
    if (!(p->lamda1 > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_lamda1: lamda1 must be greater than zero");
    if (!(p->lamda2 > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_lamda2: lamda2 must be greater than zero");
    if (!(p->dt > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_dt: dt must be greater than zero");
    if (!(p->epsilon > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_epsilon: epsilon must be greater than zero");
    if (!(p->nu >= 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_nu: nu must be non negative");
    if (!(p->beta >= 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_beta: beta must be non negative");
    if (!(p->tol >= 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_tol: tol must be greater than zero");
    if (!(p->ls_tol >= 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_tol: tol must be positive");
    if (p->ls_steps <= 0) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_ls_steps: ls_steps must be greater than 0");
    if (!(p->edge_detector_sigma >= 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_edge_detector_sigma: edge_detector_sigma must be greater than zero");
    if (p->bc != IM3D_BC_DEFAULT && p->bc != IM3D_BC_NEU && p->bc != IM3D_BC_DIR)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "WARNING::set_bc: specify a proper bc_type condition");
    if (!(p->b0 > p->a0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "b0 has to be greater than a0");
    if (p->gs_rel_res_tol > 0 && !(p->omega > 0 && p->omega < 2))
        return fail(ctx, IM3D_ERR_INVALID_ARG, "omega must lie in (0, 2)");
    return IM3D_OK;
}

// One volume's device state and loop counters (rsfe_prepare fills it).
template <typename T>
struct VolState {
    Dims d;
    long long n = 0, npk2 = 0;
    double chosen_bc = 0, hhh = 1;
    T a0 = 0, b0 = 1, center = 0, inv_eps = 0;
    const T* u0 = nullptr;
    T *phi = nullptr, *other = nullptr, *g = nullptr, *divdb = nullptr, *b3 = nullptr, *dmb = nullptr,
      *kones = nullptr, *rhs = nullptr, *upk = nullptr, *bpk = nullptr, *prev = nullptr;
    Vec<T, 4>*W1 = nullptr, *W2 = nullptr;
    Vec<T, 2>*P1 = nullptr, *P2 = nullptr;
    T *u_d = nullptr, *f1_d = nullptr, *f2_d = nullptr;
    Taps<T> tp;
    GsCoef<T> coef;
    int t0 = 0;  // outer iterations already done (a resumed run)
    double tollerance = 1000;
    int init_variables = 0;
    int sched_first = 0;  // residual schedule carried between Poisson solves
    double sched_rate = 0;
};

// Everything before the outer loop of rsfe_splitbregman<T>::apply for one volume, on
// the context's stream and in its buffers: inputs, the refusal of non-finite values,
// the initial level set (or a checkpoint's state), taps, kones and the edge detector
// (rsfe_splitbregman_imp.hxx:1547-1660). `from` resumes from a checkpoint; `wsb`
// receives the learned warm start's buffers.
template <typename T>
int rsfe_prepare(im3d_ctx* ctx, VolState<T>& v, const T* myim_user, const T* init_user, int nx,
                 int ny, int nz, double hx, double hy, double hz, const im3d_rsfe_params* p,
                 T* u_user, T* f1_user, T* f2_user, const im3d_rsfe_checkpoint* from, WsBufs* wsb)
{
    const bool resuming = from != nullptr;
    const bool ws = wsb != nullptr;
    // the convolution passes take the plug-in's boundary; no other kernel reads cyc
    Dims d{nx, ny, nz};
    d.cyc = p->conv_cyclic ? 1 : 0;
    const long long n = d.n();
    const long long npk2 = 2 * d.npk();
    const bool solve = p->gs_rel_res_tol > 0;
    const bool lex = !solve && p->sweep == IM3D_SWEEP_LEXICOGRAPHIC;
    const bool neu = p->bc == IM3D_BC_NEU;
    // chosen_bc (rsfe_splitbregman_imp.hxx:1735-1743): NEU (also the ctor default) -> 0
    const double chosen_bc = p->bc == IM3D_BC_DIR ? p->a0 : 0.0;
    const T a0 = (T)p->a0, b0 = (T)p->b0;

    const T* u0 = nullptr;
    const T* init = nullptr;
    IM3D_TRY(dev_in<T>(ctx, myim_user, n, "in_myim", &u0));
    if (init_user && !resuming) IM3D_TRY(dev_in<T>(ctx, init_user, n, "in_init", &init));

    T *phiA, *phiB, *g, *divdb, *b3, *dmb, *kones = nullptr, *rhs = nullptr, *upk = nullptr,
      *bpk = nullptr, *prev = nullptr;
    Vec<T, 4>*W1, *W2;
    Vec<T, 2>*P1, *P2;
    IM3D_TRY(tbuf<T>(ctx, "phiA", n, &phiA));
    IM3D_TRY(tbuf<T>(ctx, "phiB", n, &phiB));
    IM3D_TRY(tbuf<T>(ctx, "g", n, &g));
    IM3D_TRY(tbuf<T>(ctx, "divdb", n, &divdb, true));
    IM3D_TRY(tbuf<T>(ctx, "b3", 3 * n, &b3, true));
    IM3D_TRY(tbuf<T>(ctx, "dmb", 3 * n, &dmb));
    IM3D_TRY(tbuf<Vec<T, 4>>(ctx, "W1", n, &W1));
    IM3D_TRY(tbuf<Vec<T, 4>>(ctx, "W2", n, &W2));
    IM3D_TRY(tbuf<Vec<T, 2>>(ctx, "P1", n, &P1));
    IM3D_TRY(tbuf<Vec<T, 2>>(ctx, "P2", n, &P2));
    if (p->lamda1 != p->lamda2) IM3D_TRY(tbuf<T>(ctx, "kones", n, &kones));
    if (lex) IM3D_TRY(tbuf<T>(ctx, "rhs", n, &rhs));
    else {
        IM3D_TRY(tbuf<T>(ctx, "upk", npk2, &upk, true));
        IM3D_TRY(tbuf<T>(ctx, "bpk", npk2, &bpk, true));
    }
    if (p->ls_tol != 0 && !solve) IM3D_TRY(tbuf<T>(ctx, "prev", lex ? n : npk2, &prev, true));
    T *u_d = nullptr, *f1_d = nullptr, *f2_d = nullptr;
    IM3D_TRY(dev_out<T>(ctx, u_user, n, "out_u", &u_d));
    IM3D_TRY(dev_out<T>(ctx, f1_user, n, "out_f1", &f1_d));
    IM3D_TRY(dev_out<T>(ctx, f2_user, n, "out_f2", &f2_d));
    if (f1_d && !f2_d) IM3D_TRY(tbuf<T>(ctx, "out_f2", n, &f2_d));
    if (f2_d && !f1_d) IM3D_TRY(tbuf<T>(ctx, "out_f1", n, &f1_d));
    if (ws) {
        IM3D_TRY(tbuf<float>(ctx, "ws_x", 4 * (size_t)n, &wsb->x));
        IM3D_TRY(tbuf<float>(ctx, "ws_y", (size_t)n, &wsb->y));
        IM3D_TRY(tbuf<float>(ctx, "ws_upk0", (size_t)npk2, &wsb->upk0));
        // the previous solve's u: the clamp kernel writes it (before the clamp)
        if (!u_d) IM3D_TRY(tbuf<T>(ctx, "ws_prevu", n, &u_d));
    }

    IM3D_TRY(zero_ctrl(ctx));
    {
        // NaN or Inf in the image: refused here (the reference's debug build traps the
        // floating-point exception they raise, exceptions.hxx:25-35)
        T mn, mx;
        bool bad = false;
        IM3D_TRY(minmax<T>(ctx, u0, n, &mn, &mx, &bad));
        if (bad) return fail(ctx, IM3D_ERR_NONFINITE, "myim holds NaN or Inf values");
    }
    int t0 = 0;  // outer iterations already done (a resumed run)
    double tollerance = 1000;
    int init_variables = p->init_variables;
    int sched_first = 0;  // residual schedule carried between Poisson solves
    double sched_rate = 0;
    if (resuming) {
        // the state of the checkpoint instead of the initial level set
        IM3D_CUDA(ctx, cudaMemcpyAsync(phiA, from->phi, n * sizeof(T), cudaMemcpyDefault, ctx->stream));
        IM3D_CUDA(ctx, cudaMemcpyAsync(b3, from->b, 3 * n * sizeof(T), cudaMemcpyDefault, ctx->stream));
        IM3D_CUDA(ctx, cudaMemcpyAsync(divdb, from->divdb, n * sizeof(T), cudaMemcpyDefault, ctx->stream));
        t0 = from->t;
        tollerance = from->tollerance;
        init_variables = from->init_variables;
        sched_first = from->sched_first;
        sched_rate = from->sched_rate;
    } else {
        // initial level set (rsfe_splitbregman_imp.hxx:99-170 / :48-95), then
        // change_range_of_intensity(b0, a0) (image3d_imp.hxx:1628-1636)
        if (init) {
            IM3D_CUDA(ctx, cudaMemcpyAsync(phiA, init, n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
        } else {
            const int ix = (int)(nx * 0.33), iy = (int)(ny * 0.33), iz = (int)(nz * 0.33);
            const int fx = (int)(nx * (1 - 0.33)), fy = (int)(ny * (1 - 0.33)), fz = (int)(nz * (1 - 0.33));
            cube_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(phiA, d, ix, iy, iz, fx,
                                                                               fy, fz, a0, b0);
            IM3D_TRY(check_launch(ctx, "cube"));
        }
        T mn, mx;
        bool bad = false;
        IM3D_TRY(minmax<T>(ctx, phiA, n, &mn, &mx, &bad));
        if (bad) return fail(ctx, IM3D_ERR_NONFINITE, "init holds NaN or Inf values");
        const T shifted_max = mx - mn;
        const T s = shifted_max / (T)(b0 - a0);
        affine_kernel<T><<<flat_grid(n), 256, 0, ctx->stream>>>(phiA, n, mn, s, a0);
        IM3D_TRY(check_launch(ctx, "affine"));
    }
    // the first solve's "previous u" is the initial level set
    if (ws) IM3D_CUDA(ctx, cudaMemcpyAsync(u_d, phiA, n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));

    // filters, kones (only used when lamda1 != lamda2), edge detector
    Taps<T> tp;
    IM3D_TRY(upload_taps<T>(ctx, "taps", p->sigma, 3.0, hx, hy, hz, p->gaussian_pixel_approach, &tp));
    if (kones) IM3D_TRY(gauss_scalar<T>(ctx, LdOne<T>{}, kones, d, tp));
    {
        const T* src = u0;
        if (p->edge_detector_sigma != 0) {
            Taps<T> te;
            IM3D_TRY(upload_taps<T>(ctx, "taps_eds", p->edge_detector_sigma, 3.0, hx, hy, hz,
                                    p->gaussian_pixel_approach, &te));
            T* blurred = nullptr;
            IM3D_TRY(tbuf<T>(ctx, "eds_blur", n, &blurred));
            IM3D_TRY(gauss_scalar<T>(ctx, LdScalar<T>{u0, d}, blurred, d, te));
            src = blurred;
        }
        edge_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(
            src, g, d, hx, hy, hz, (T)p->beta, (T)p->lamda, (T)p->nu);
        IM3D_TRY(check_launch(ctx, "edge"));
    }

    v.d = d;
    v.n = n;
    v.npk2 = npk2;
    v.chosen_bc = chosen_bc;
    v.hhh = hx * hy * hz;
    v.a0 = a0;
    v.b0 = b0;
    v.center = (T)((p->a0 + p->b0) / 2.);
    v.inv_eps = (T)(1.0 / p->epsilon);
    v.u0 = u0;
    v.phi = phiA;
    v.other = phiB;
    v.g = g;
    v.divdb = divdb;
    v.b3 = b3;
    v.dmb = dmb;
    v.kones = kones;
    v.rhs = rhs;
    v.upk = upk;
    v.bpk = bpk;
    v.prev = prev;
    v.W1 = W1;
    v.W2 = W2;
    v.P1 = P1;
    v.P2 = P2;
    v.u_d = u_d;
    v.f1_d = f1_d;
    v.f2_d = f2_d;
    v.tp = tp;
    v.coef = make_coef<T>(hx, hy, hz, p->dt, chosen_bc, neu ? 1 : 0);
    v.t0 = t0;
    v.tollerance = tollerance;
    v.init_variables = init_variables;
    v.sched_first = sched_first;
    v.sched_rate = sched_rate;
    return IM3D_OK;
}

template <typename T>
struct Outs {
    T* phi;
    T* u;
    T* f1;
    T* f2;
};

template <typename T>
int rsfe_apply(im3d_ctx* ctx, const T* myim_user, const T* init_user, int nx, int ny, int nz,
               double hx, double hy, double hz, const im3d_rsfe_params* p, T* phi_user, T* u_user,
               T* f1_user, T* f2_user, im3d_rsfe_stats* stats)
{
    IM3D_TRY(check_dims(ctx, nx, ny, nz, hx, hy, hz));
    if (!p) return fail(ctx, IM3D_ERR_INVALID_ARG, "params must not be NULL");
    if (!myim_user || !phi_user) return fail(ctx, IM3D_ERR_INVALID_ARG, "myim and phi_out are required");
    IM3D_TRY(check_params(ctx, p));
    const bool ws = ctx->ws_net && ctx->ws_mode != IM3D_WS_OFF && p->gs_rel_res_tol > 0;
    if (ws && !std::is_same<T, float>::value)
        return fail(ctx, IM3D_ERR_UNSUPPORTED, "the learned warm start runs with the FP32 entry point");

    // a pending resume is consumed by this call, whatever its outcome
    const bool resuming = ctx->resume;
    const im3d_rsfe_checkpoint from = ctx->resume_from;
    ctx->resume = false;
    if (resuming) {
        if (ctx->resume_esize != (int)sizeof(T))
            return fail(ctx, IM3D_ERR_INVALID_ARG, "the checkpoint's element size does not match this call");
        if (!from.phi || !from.b || !from.divdb || from.t < 0)
            return fail(ctx, IM3D_ERR_INVALID_ARG, "a checkpoint needs phi, b, divdb and t >= 0");
    }

    IM3D_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    const bool solve = p->gs_rel_res_tol > 0;
    const bool lex = !solve && p->sweep == IM3D_SWEEP_LEXICOGRAPHIC;
    const bool neu = p->bc == IM3D_BC_NEU;
    VolState<T> vs;
    WsBufs wsb{nullptr, nullptr, nullptr};
    IM3D_TRY(rsfe_prepare<T>(ctx, vs, myim_user, init_user, nx, ny, nz, hx, hy, hz, p, u_user, f1_user,
                             f2_user, resuming ? &from : nullptr, ws ? &wsb : nullptr));
    IM3D_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    const Dims d = vs.d;
    const long long n = vs.n;
    const long long npk2 = vs.npk2;
    const double chosen_bc = vs.chosen_bc;
    const T a0 = vs.a0, b0 = vs.b0;
    const T* u0 = vs.u0;
    T *g = vs.g, *divdb = vs.divdb, *b3 = vs.b3, *dmb = vs.dmb, *kones = vs.kones, *rhs = vs.rhs,
      *upk = vs.upk, *bpk = vs.bpk, *prev = vs.prev;
    Vec<T, 4>*W1 = vs.W1, *W2 = vs.W2;
    Vec<T, 2>*P1 = vs.P1, *P2 = vs.P2;
    T *u_d = vs.u_d, *f1_d = vs.f1_d, *f2_d = vs.f2_d;
    const Taps<T>& tp = vs.tp;
    const GsCoef<T> coef = vs.coef;
    const T center = vs.center;
    const T inv_eps = vs.inv_eps;
    const double hhh = vs.hhh;
    const int t0 = vs.t0;
    double tollerance = vs.tollerance;
    int init_variables = vs.init_variables;
    int sched_first = vs.sched_first;
    double sched_rate = vs.sched_rate;
    int ws_used = 0, ws_rejected = 0, ws_steps = 0;
    double ws_loss = 0;
    long long total_sweeps = 0;
    int last_sweeps = 0, not_conv = 0, t;
    const long long checks0 = ctx->residual_checks;
    double last_rel = -1, last_ls_err = -1;
    T* phi = vs.phi;  // current level set (natural)
    T* other = vs.other;

    for (t = t0 + 1; tollerance > p->tol && t <= p->maxiter; ++t) {
        // stage 1-5: Heaviside, the four convolutions, fitting terms, forcing term
        bool tma_done = false;
        if constexpr (std::is_same<T, float>::value) {
            if (heav_tma_eligible(ctx, d, tp.nh[2], phi, u0, W1)) {
                if (tp.nh[2] == 19)
                    IM3D_TRY(pass_heav_tma<9>(ctx, phi, u0, W1, d, tp.w[2], center, inv_eps, "conv_k_heaviside"));
                else
                    IM3D_TRY(pass_heav_tma<12>(ctx, phi, u0, W1, d, tp.w[2], center, inv_eps, "conv_k_heaviside"));
                tma_done = true;
            }
        }
        if (!tma_done)
            IM3D_TRY((pass_k<T, 4>(ctx, LdHeaviside<T>{phi, u0, d, center, inv_eps}, StVec<T, 4>{W1, d},
                                   d, tp.w[2], tp.nh[2], "conv_k_heaviside")));
        IM3D_TRY((pass_s<T, 4, 1>(ctx, LdVec<T, 4>{W1, d}, StVec<T, 4>{W2, d}, d, tp.w[1], tp.nh[1],
                                  "conv_s_j4")));
        IM3D_TRY(pass_i_fit<T>(ctx, W2, P1, f1_d, f2_d, d, tp.w[0], tp.host[0], tp.nh[0], (T)p->lamda1,
                               (T)p->lamda2));
        IM3D_TRY((pass_s<T, 2, 1>(ctx, LdVec<T, 2>{P1, d}, StVec<T, 2>{P2, d}, d, tp.w[1], tp.nh[1],
                                  "conv_s_j2")));
        {
            StRhs<T> st;
            st.u0 = u0; st.kones = kones; st.divdb = divdb; st.phi = phi;
            st.out = lex ? rhs : bpk;
            st.upk = upk;
            st.beff2 = nullptr;
            st.d = d;
            st.l12 = (T)(p->lamda1 - p->lamda2);
            st.lamda = (T)p->lamda;
            st.inv_lamda = (T)(1.0 / p->lamda);
            st.inv_dt = (T)(1.0 / p->dt);
            st.bc = (T)chosen_bc;
            st.mode = lex ? 0 : (solve ? 2 : 1);
            st.dirichlet = neu ? 0 : 1;
            IM3D_TRY((pass_k<T, 2>(ctx, LdVec<T, 2>{P2, d}, st, d, tp.w[2], tp.nh[2], "conv_k_rhs")));
        }

        // the Poisson step (rsfe_splitbregman_imp.hxx:1768-1785)
        T* uu;  // where the solved u lives (natural `phi` for lex, packed otherwise)
        if (solve) {
            int sw = 0;
            double rel = -1;
            bool conv = false;
            // each solve's residual schedule starts from the previous one: the first
            // check after as many sweeps as it needed, its contraction rate as the first
            // prediction (the sweep counts of consecutive solves differ by a sweep or two)
            double rate = 0;
            // the whole solve, warm start included, as one more profiled stage (it
            // encloses the half-sweep and residual stages): the time to tolerance
            const int pfs = prof_begin(ctx, "poisson_solve");
            if constexpr (std::is_same<T, float>::value) {
                if (ws)
                    IM3D_TRY(ws_before(ctx, d, coef, upk, bpk, u_d, divdb, phi, (float)(1.0 / p->dt), neu ? 0 : 1,
                                       wsb, &ws_used, &ws_rejected));
            }
            IM3D_TRY(rb_solve<T>(ctx, upk, bpk, d, coef, p->gs_rel_res_tol, p->gs_max_sweeps,
                                 p->gs_check_every, p->omega, &sw, &rel, &conv, sched_first,
                                 sched_rate, &rate));
            prof_end(ctx, pfs);
            if constexpr (std::is_same<T, float>::value) {
                if (ws && ctx->ws_mode == IM3D_WS_TRAIN) {
                    double l = 0;
                    IM3D_TRY(ws_after(ctx, d, upk, wsb, &l));
                    ws_loss += l;
                    ++ws_steps;
                }
            }
            sched_first = conv ? sw : 0;
            sched_rate = conv ? rate : 0;
            if (!conv) not_conv++;
            total_sweeps += sw;
            last_sweeps = sw;
            last_rel = rel;
            uu = upk;
        } else {
            if (lex) IM3D_CUDA(ctx, cudaMemcpyAsync(other, phi, n * sizeof(T), cudaMemcpyDeviceToDevice,
                                                    ctx->stream));
            T* work = lex ? phi : upk;
            const long long cnt = lex ? n : npk2;
            double ls_err = p->ls_tol ? 1000. : -1.;
            int s;
            for (s = 0; s < p->ls_steps || ls_err > p->ls_tol; ++s) {
                if (s >= 100000) {
                    not_conv++;
                    break;
                }
                if (p->ls_tol != 0)
                    IM3D_CUDA(ctx, cudaMemcpyAsync(prev, work, cnt * sizeof(T), cudaMemcpyDeviceToDevice,
                                                   ctx->stream));
                if (lex) IM3D_TRY(lex_sweep<T>(ctx, phi, rhs, d, coef));
                else IM3D_TRY(rb_sweep<T>(ctx, upk, bpk, d, coef, 1, 1.0));
                if (p->ls_tol != 0 && s >= p->ls_steps - 1) {
                    const dim3 grid(flat_grid(cnt));
                    double* part = nullptr;
                    IM3D_TRY(part_buf(ctx, grid, 2, &part));
                    diff_sums_kernel<T><<<grid, 256, 0, ctx->stream>>>(work, prev, cnt, part);
                    IM3D_TRY(check_launch(ctx, "diff_sums"));
                    IM3D_TRY(finalize(ctx, part, grid, 2, SUM_A));
                    IM3D_TRY(read_ctrl(ctx));
                    ls_err = std::sqrt(hhh * ctx->ctrl_h->sum[SUM_A]) /
                             std::sqrt(hhh * ctx->ctrl_h->sum[SUM_B]);
                }
            }
            total_sweeps += s;
            last_sweeps = s;
            last_ls_err = ls_err;
            uu = lex ? phi : upk;
        }

        // clamp, tolerance, Bregman update, div(d - b)
        T* phi_new = lex ? other : phi;  // lex: `other` holds phiold and receives the clamp
        // automatic connected-component extraction at this iteration (:1809): phiold is
        // kept for the tolerance, which the reference takes after the extraction
        const bool cc_now = p->auto_extract_conn_comp && p->auto_extract_conn_comp_freq != 0 &&
                            t % p->auto_extract_conn_comp_freq == 0;
        T* cc_old = nullptr;
        if (cc_now) {
            IM3D_TRY(tbuf<T>(ctx, "cc_phiold", (size_t)n, &cc_old));
            IM3D_CUDA(ctx, cudaMemcpyAsync(cc_old, phi_new, n * sizeof(T), cudaMemcpyDeviceToDevice,
                                           ctx->stream));
        }
        // vector path: rows 16-byte aligned (nz multiple of the width) and an aligned u_out
        const bool vec = d.nz % V16<T>::W == 0 && ((uintptr_t)u_d % 16) == 0;
        {
            const dim3 grid = vec ? grid_vec<T>(d, kBlkVec) : grid_col(d, kBlkVol);
            const dim3 blk = vec ? kBlkVec : kBlkVol;
            double* part = nullptr;
            IM3D_TRY(part_buf(ctx, grid, 2, &part));
            const int pf = prof_begin(ctx, "clamp_tol");
            if (vec && lex)
                clamp_tol_vec_kernel<T, false, kNV><<<grid, blk, 0, ctx->stream>>>(
                    uu, phi_new, u_d, d, a0, b0, part);
            else if (vec)
                clamp_tol_vec_kernel<T, true, kNV><<<grid, blk, 0, ctx->stream>>>(
                    uu, phi_new, u_d, d, a0, b0, part);
            else if (lex)
                clamp_tol_kernel<T, false, kNI><<<grid, kBlkVol, 0, ctx->stream>>>(
                    uu, phi_new, u_d, d, a0, b0, part);
            else
                clamp_tol_kernel<T, true, kNI><<<grid, kBlkVol, 0, ctx->stream>>>(
                    uu, phi_new, u_d, d, a0, b0, part);
            prof_end(ctx, pf);
            IM3D_TRY(check_launch(ctx, "clamp_tol"));
            IM3D_TRY(finalize(ctx, part, grid, 2, SUM_DPHI2));
        }
        if (cc_now) {
            bool replaced = false;
            IM3D_TRY(extract_cc<T>(ctx, phi_new, d, hx, hy, hz, p, &replaced));
            if (replaced) {
                if (p->cc_init_variables) init_variables = 1;
                const dim3 grid(flat_grid(n));
                double* part = nullptr;
                IM3D_TRY(part_buf(ctx, grid, 2, &part));
                diff_sums_kernel<T><<<grid, 256, 0, ctx->stream>>>(phi_new, cc_old, n, part);
                IM3D_TRY(check_launch(ctx, "diff_sums"));
                IM3D_TRY(finalize(ctx, part, grid, 2, SUM_DPHI2));
            }
        }
        // the tolerance sums are final here: copy them out now and wait only for that
        // copy after the Bregman update is queued, so that the next iteration's kernels
        // queue behind work that is still running
        IM3D_CUDA(ctx, cudaMemcpyAsync(ctx->ctrl_h, ctx->ctrl_d, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                                       ctx->stream));
        IM3D_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
        if (init_variables) {
            IM3D_CUDA(ctx, cudaMemsetAsync(divdb, 0, n * sizeof(T), ctx->stream));
            IM3D_CUDA(ctx, cudaMemsetAsync(b3, 0, 3 * n * sizeof(T), ctx->stream));
            init_variables = 0;
        } else {
            const int pf = prof_begin(ctx, "bregman");
            if (vec)
                bregman_vec_kernel<T, kNV><<<grid_vec<T>(d, kBlkVec), kBlkVec, 0, ctx->stream>>>(
                    phi_new, b3, dmb, g, d, hx, hy, hz);
            else
                bregman_kernel<T, kNIbr><<<grid_col(d, kBlkVol, kNIbr), kBlkVol, 0, ctx->stream>>>(
                    phi_new, b3, dmb, g, d, hx, hy, hz);
            prof_end(ctx, pf);
            IM3D_TRY(check_launch(ctx, "bregman"));
            const int pf2 = prof_begin(ctx, "div");
            if (vec)
                div_vec_kernel<T, kNV><<<grid_vec<T>(d, kBlkVec), kBlkVec, 0, ctx->stream>>>(
                    dmb, divdb, d, hx, hy, hz);
            else
                div_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(dmb, divdb, d, hx, hy, hz);
            prof_end(ctx, pf2);
            IM3D_TRY(check_launch(ctx, "div"));
        }
        if (cudaEventSynchronize(ctx->ev[3]) != cudaSuccess) IM3D_TRY(sync(ctx));
        if (ctx->ctrl_h->flag[0])
            return fail(ctx, IM3D_ERR_CUDA, "a TMA load of the Heaviside pass did not complete in time");
        tollerance = std::sqrt(hhh * ctx->ctrl_h->sum[SUM_DPHI2]) /
                     std::sqrt(hhh * ctx->ctrl_h->sum[SUM_PHIOLD2]);
        if (lex) std::swap(phi, other);
        // dumps and checkpoints: the reference's rule t % dumpfrequency == 0, t != maxiter
        // (rsfe_splitbregman_imp.hxx:1940-1951)
        if (ctx->obs && ctx->obs_every > 0 && t % ctx->obs_every == 0 && t != p->maxiter) {
            const size_t nb = (size_t)n * sizeof(T);
            ctx->obs_host.resize(ctx->obs_state ? 5 * nb : nb);
            T* hp = reinterpret_cast<T*>(ctx->obs_host.data());
            IM3D_CUDA(ctx, cudaMemcpyAsync(hp, phi, nb, cudaMemcpyDeviceToHost, ctx->stream));
            if (ctx->obs_state) {
                IM3D_CUDA(ctx, cudaMemcpyAsync(hp + n, b3, 3 * nb, cudaMemcpyDeviceToHost, ctx->stream));
                IM3D_CUDA(ctx, cudaMemcpyAsync(hp + 4 * n, divdb, nb, cudaMemcpyDeviceToHost, ctx->stream));
            }
            IM3D_TRY(sync(ctx));
            im3d_rsfe_checkpoint ck{};
            ck.t = t;
            ck.init_variables = init_variables;
            ck.sched_first = sched_first;
            ck.sched_rate = sched_rate;
            ck.tollerance = tollerance;
            ck.phi = hp;
            ck.b = ctx->obs_state ? hp + n : nullptr;
            ck.divdb = ctx->obs_state ? hp + 4 * n : nullptr;
            if (ctx->obs(ctx->obs_user, &ck) != 0) {
                ++t;  // the loop ends after this iteration, as with end_now
                break;
            }
        }
    }
    IM3D_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));

    // outputs
    if (is_device_ptr(phi_user)) {
        IM3D_CUDA(ctx, cudaMemcpyAsync(phi_user, phi, n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        IM3D_CUDA(ctx, cudaMemcpyAsync(phi_user, phi, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    }
    IM3D_TRY(out_finish<T>(ctx, u_user, u_d, n));
    IM3D_TRY(out_finish<T>(ctx, f1_user, f1_d, n));
    IM3D_TRY(out_finish<T>(ctx, f2_user, f2_d, n));
    IM3D_TRY(sync(ctx));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->iterations = t - 1;
        stats->last_tol = tollerance;
        stats->total_sweeps = total_sweeps;
        stats->last_sweeps = last_sweeps;
        stats->last_rel_res = last_rel;
        stats->last_ls_err = last_ls_err;
        stats->not_converged = not_conv;
        stats->residual_checks = (int32_t)(ctx->residual_checks - checks0);
        stats->ws_used = ws_used;
        stats->ws_rejected = ws_rejected;
        stats->ws_loss = ws_steps ? ws_loss / ws_steps : 0.0;
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        stats->setup_ms = ms;
        cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
        stats->loop_ms = ms;
    }
    return IM3D_OK;
}

// ------------------------------------------------------ standalone operators
template <typename T>
int gauss_filter(im3d_ctx* ctx, const T* in_user, T* out_user, int nx, int ny, int nz, double hx,
                 double hy, double hz, double sigma, double radius, int pixel_approach,
                 int cyclic = 0)
{
    IM3D_TRY(check_dims(ctx, nx, ny, nz, hx, hy, hz));
    if (!in_user || !out_user) return fail(ctx, IM3D_ERR_INVALID_ARG, "NULL volume");
    Dims d{nx, ny, nz};
    d.cyc = cyclic ? 1 : 0;
    const T* in = nullptr;
    T* out = nullptr;
    IM3D_TRY(dev_in<T>(ctx, in_user, d.n(), "in_a", &in));
    IM3D_TRY(dev_out<T>(ctx, out_user, d.n(), "out_a", &out));
    Taps<T> tp;
    IM3D_TRY(upload_taps<T>(ctx, "taps_op", sigma, radius, hx, hy, hz, pixel_approach, &tp));
    IM3D_TRY(gauss_scalar<T>(ctx, LdScalar<T>{in, d}, out, d, tp));
    IM3D_TRY(out_finish<T>(ctx, out_user, out, d.n()));
    return sync(ctx);
}

template <typename T>
int grad_op(im3d_ctx* ctx, const T* in_user, T* out_user, int nx, int ny, int nz, double hx,
            double hy, double hz)
{
    IM3D_TRY(check_dims(ctx, nx, ny, nz, hx, hy, hz));
    if (!in_user || !out_user) return fail(ctx, IM3D_ERR_INVALID_ARG, "NULL volume");
    const Dims d{nx, ny, nz};
    const T* in = nullptr;
    T* out = nullptr;
    IM3D_TRY(dev_in<T>(ctx, in_user, d.n(), "in_a", &in));
    IM3D_TRY(dev_out<T>(ctx, out_user, 3 * d.n(), "out_a", &out));
    grad_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(in, out, d, hx, hy, hz);
    IM3D_TRY(check_launch(ctx, "grad"));
    IM3D_TRY(out_finish<T>(ctx, out_user, out, 3 * d.n()));
    return sync(ctx);
}

template <typename T>
int div_op(im3d_ctx* ctx, const T* in_user, T* out_user, int nx, int ny, int nz, double hx,
           double hy, double hz)
{
    IM3D_TRY(check_dims(ctx, nx, ny, nz, hx, hy, hz));
    if (!in_user || !out_user) return fail(ctx, IM3D_ERR_INVALID_ARG, "NULL volume");
    const Dims d{nx, ny, nz};
    const T* in = nullptr;
    T* out = nullptr;
    IM3D_TRY(dev_in<T>(ctx, in_user, 3 * d.n(), "in_a", &in));
    IM3D_TRY(dev_out<T>(ctx, out_user, d.n(), "out_a", &out));
    div_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(in, out, d, hx, hy, hz);
    IM3D_TRY(check_launch(ctx, "div"));
    IM3D_TRY(out_finish<T>(ctx, out_user, out, d.n()));
    return sync(ctx);
}

template <typename T>
int poisson_sweeps(im3d_ctx* ctx, T* res_user, const T* b_user, int nx, int ny, int nz, double hx,
                   double hy, double hz, double dt, double bc, int bc_type, int order, int sweeps)
{
    IM3D_TRY(check_dims(ctx, nx, ny, nz, hx, hy, hz));
    if (!res_user || !b_user) return fail(ctx, IM3D_ERR_INVALID_ARG, "NULL volume");
    if (!(dt > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "dt must be greater than zero");
    if (sweeps < 0) return fail(ctx, IM3D_ERR_INVALID_ARG, "sweeps must be non negative");
    if (order != IM3D_SWEEP_LEXICOGRAPHIC && order != IM3D_SWEEP_REDBLACK)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "unknown sweep order");
    const Dims d{nx, ny, nz};
    const long long n = d.n();
    const GsCoef<T> c = make_coef<T>(hx, hy, hz, dt, bc, bc_type == IM3D_BC_NEU ? 1 : 0);
    const T* b = nullptr;
    T* r = nullptr;
    IM3D_TRY(dev_in<T>(ctx, b_user, n, "in_b", &b));
    if (is_device_ptr(res_user)) r = res_user;
    else {
        IM3D_TRY(tbuf<T>(ctx, "io_res", n, &r));
        IM3D_CUDA(ctx, cudaMemcpyAsync(r, res_user, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    }
    if (order == IM3D_SWEEP_LEXICOGRAPHIC) {
        for (int s = 0; s < sweeps; ++s) IM3D_TRY(lex_sweep<T>(ctx, r, b, d, c));
    } else if (sweeps > 0) {
        // DirGaussSeidel assigns the boundary value before sweeping (poisson_imp.hxx:366-391)
        if (!c.neu) {
            dir_faces_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(r, d, c.bc);
            IM3D_TRY(check_launch(ctx, "dir_faces"));
        }
        T *U, *B;
        IM3D_TRY(tbuf<T>(ctx, "op_upk", 2 * d.npk(), &U, true));
        IM3D_TRY(tbuf<T>(ctx, "op_bpk", 2 * d.npk(), &B, true));
        pack_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(r, U, d);
        IM3D_TRY(check_launch(ctx, "pack"));
        pack_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(b, B, d);
        IM3D_TRY(check_launch(ctx, "pack"));
        for (int s = 0; s < sweeps; ++s) IM3D_TRY(rb_sweep<T>(ctx, U, B, d, c, 1, 1.0));
        unpack_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(U, r, d);
        IM3D_TRY(check_launch(ctx, "unpack"));
    }
    if (r != res_user)
        IM3D_CUDA(ctx, cudaMemcpyAsync(res_user, r, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    return sync(ctx);
}

template <typename T>
int poisson_solve(im3d_ctx* ctx, T* u_user, const T* b_user, int nx, int ny, int nz, double hx,
                  double hy, double hz, double dt, double bc, int bc_type, double tol,
                  int max_sweeps, int check_every, double omega, int* sweeps_done, double* rel_res)
{
    IM3D_TRY(check_dims(ctx, nx, ny, nz, hx, hy, hz));
    if (!u_user || !b_user) return fail(ctx, IM3D_ERR_INVALID_ARG, "NULL volume");
    if (!(dt > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "dt must be greater than zero");
    if (!(omega > 0 && omega < 2)) return fail(ctx, IM3D_ERR_INVALID_ARG, "omega must lie in (0, 2)");
    const Dims d{nx, ny, nz};
    const long long n = d.n();
    const int neu = bc_type == IM3D_BC_NEU ? 1 : 0;
    const GsCoef<T> c = make_coef<T>(hx, hy, hz, dt, bc, neu);
    const T* b = nullptr;
    T* r = nullptr;
    IM3D_TRY(dev_in<T>(ctx, b_user, n, "in_b", &b));
    if (is_device_ptr(u_user)) r = u_user;
    else {
        IM3D_TRY(tbuf<T>(ctx, "io_res", n, &r));
        IM3D_CUDA(ctx, cudaMemcpyAsync(r, u_user, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    }
    T *U, *B;
    IM3D_TRY(tbuf<T>(ctx, "op_upk", 2 * d.npk(), &U, true));
    IM3D_TRY(tbuf<T>(ctx, "op_bpk", 2 * d.npk(), &B, true));
    pack_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(r, U, d);
    IM3D_TRY(check_launch(ctx, "pack"));
    make_beff_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(b, U, B, d,
                                                                          (T)(1.0 / dt), (T)bc,
                                                                          neu ? 0 : 1, nullptr);
    IM3D_TRY(check_launch(ctx, "make_beff"));
    int sw = 0;
    double rel = -1;
    bool conv = false;
    IM3D_TRY(rb_solve<T>(ctx, U, B, d, c, tol, max_sweeps, check_every, omega, &sw, &rel, &conv));
    unpack_kernel<T><<<grid_vol(d, kBlkVol), kBlkVol, 0, ctx->stream>>>(U, r, d);
    IM3D_TRY(check_launch(ctx, "unpack"));
    if (r != u_user)
        IM3D_CUDA(ctx, cudaMemcpyAsync(u_user, r, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    IM3D_TRY(sync(ctx));
    if (sweeps_done) *sweeps_done = sw;
    if (rel_res) *rel_res = rel;
    if (!conv) return fail(ctx, IM3D_ERR_NOT_CONVERGED, "sweep cap reached before the tolerance");
    return IM3D_OK;
}

#if IM3D_UNIT != 1
// ------------------------------------------------ Gaussian filter, no allocation
// Fixed scratch of im3d_gauss_filter_f32_noalloc: two intermediate volumes of up to
// kNoAllocMaxVoxels voxels, then the three axes' taps.
constexpr long long kNoAllocMaxVoxels = 1LL << 21;
constexpr long long kNoAllocFloats = 2 * kNoAllocMaxVoxels + 3 * NH_MAX;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

struct NoAllocTaps {
    float w[3 * NH_MAX];
};

// Writes the taps (passed by value) into the scratch array; device code names the
// array directly.
__global__ void noalloc_taps_kernel(NoAllocTaps t)
{
    for (int q = threadIdx.x; q < 3 * NH_MAX; q += blockDim.x)
        g_noalloc_scratch[2 * kNoAllocMaxVoxels + q] = t.w[q];
}

// Device address of g_noalloc_scratch per device, looked up once with that device
// current (in host code the array's name is only a host-side stand-in).
float* noalloc_scratch_address(int device, cudaError_t* err)
{
    static float* addr[256] = {nullptr};
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 256) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    if (!addr[device]) {
        void* ptr = nullptr;
        *err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (*err != cudaSuccess) return nullptr;
        addr[device] = static_cast<float*>(ptr);
    }
    *err = cudaSuccess;
    return addr[device];
}

// A device pointer of the current device (the kernels would otherwise touch another
// GPU's memory, which faults without peer access).
bool on_current_device(const void* p, int device)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

// One launch on the caller's stream; the launch's own status is returned, so the call
// reports its errors without reading (and clearing) an error the caller left pending.
template <typename... KArgs, typename... Args>
cudaError_t launch_on(cudaStream_t stream, void (*kern)(KArgs...), dim3 grid, dim3 blk, size_t smem,
                      Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = blk;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
    if (e != cudaSuccess) cudaGetLastError();  // the error this launch raised
    return e;
}

int gauss_filter_noalloc(const float* in, float* out, int nx, int ny, int nz, double hx,
                         double hy, double hz, double sigma, double radius, int pixel_approach,
                         cudaStream_t stream)
{
    if (!in || !out || nx <= 0 || ny <= 0 || nz <= 0) return IM3D_ERR_INVALID_ARG;
    if (nz == 1 || nx < 3 || ny < 3 || nz < 3) return IM3D_ERR_UNSUPPORTED;
    if (!(hx > 0) || !(hy > 0) || !(hz > 0) || !(sigma > 0) || !(radius > 0))
        return IM3D_ERR_INVALID_ARG;
    // the launch geometry of the j and i passes puts nx and ny on grid.z
    if (nx > 65535 || ny > 65535) return IM3D_ERR_INVALID_ARG;
    const Dims d{nx, ny, nz};
    if (d.n() > kNoAllocMaxVoxels) return IM3D_ERR_TOO_LARGE;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return IM3D_ERR_CUDA;
    }
    if (!on_current_device(in, device) || !on_current_device(out, device)) return IM3D_ERR_INVALID_ARG;
    // taps on the host stack: conv::filtering<T>::build_gaussian_filter per axis
    NoAllocTaps taps;
    int nh[3];
    const double hs[3] = {pixel_approach ? 1. : hx, pixel_approach ? 1. : hy,
                          pixel_approach ? 1. : hz};
    for (int a = 0; a < 3; ++a) {
        int m = (int)std::ceil(2 * radius * sigma / hs[a]);
        if (m % 2 == 0) m++;
        if (m > NH_MAX) return IM3D_ERR_UNSUPPORTED;
        nh[a] = m;
        const int S = m / 2;
        double w[NH_MAX];
        double sum = 0;
        for (int t = 0; t < m; ++t) {
            const double dd = (double)(t - S);
            w[t] = std::exp(-dd * dd * hs[a] * hs[a] / (2 * sigma * sigma));
            sum += w[t];
        }
        for (int t = 0; t < NH_MAX; ++t) taps.w[a * NH_MAX + t] = t < m ? (float)(w[t] / sum) : 0.f;
    }
    cudaError_t e = cudaSuccess;
    float* base = noalloc_scratch_address(device, &e);
    if (!base) {
        cudaGetLastError();
        return IM3D_ERR_CUDA;
    }
    Vec<float, 1>* t1 = reinterpret_cast<Vec<float, 1>*>(base);
    Vec<float, 1>* t2 = reinterpret_cast<Vec<float, 1>*>(base + kNoAllocMaxVoxels);
    const float* w = base + 2 * kNoAllocMaxVoxels;
    if (launch_on(stream, noalloc_taps_kernel, dim3(1), dim3(128), 0, taps) != cudaSuccess)
        return IM3D_ERR_CUDA;
    {
        const int S = nh[2] / 2;
        const size_t smem = (size_t)RK * (TK + 2 * S) * sizeof(Vec<float, 1>) + nh[2] * sizeof(float) + 16;
        auto kern = conv_k_kernel<float, 1, TK, RK, LdScalar<float>, StVec<float, 1>>;
        if (smem > 48 * 1024 &&
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return IM3D_ERR_CUDA;
        }
        const long long rows = (long long)nx * ny;
        if (launch_on(stream, kern, dim3((unsigned)((rows + RK - 1) / RK), (nz + TK - 1) / TK), dim3(TK, RK),
                      smem, LdScalar<float>{in, d}, StVec<float, 1>{t1, d}, d, w + 2 * NH_MAX, nh[2]) != cudaSuccess)
            return IM3D_ERR_CUDA;
    }
    {
        constexpr int TA = TileA<float>::v;
        const int S = nh[1] / 2;
        const size_t smem = (size_t)(TA + 2 * S) * TW * sizeof(Vec<float, 1>) + nh[1] * sizeof(float) + 16;
        auto kern = conv_s_kernel<float, 1, 1, TW, TY, TA, LdVec<float, 1>, StVec<float, 1>>;
        if (smem > 48 * 1024 &&
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return IM3D_ERR_CUDA;
        }
        if (launch_on(stream, kern, dim3((nz + TW - 1) / TW, (ny + TA - 1) / TA, nx), dim3(TW, TY), smem,
                      LdVec<float, 1>{t1, d}, StVec<float, 1>{t2, d}, d, w + NH_MAX, nh[1]) != cudaSuccess)
            return IM3D_ERR_CUDA;
    }
    {
        constexpr int TA = TileA<float>::v;
        const int S = nh[0] / 2;
        const size_t smem = (size_t)(TA + 2 * S) * TW * sizeof(Vec<float, 1>) + nh[0] * sizeof(float) + 16;
        auto kern = conv_s_kernel<float, 1, 0, TW, TY, TA, LdVec<float, 1>, StScalar<float>>;
        if (smem > 48 * 1024 &&
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return IM3D_ERR_CUDA;
        }
        if (launch_on(stream, kern, dim3((nz + TW - 1) / TW, (nx + TA - 1) / TA, ny), dim3(TW, TY), smem,
                      LdVec<float, 1>{t2, d}, StScalar<float>{out, d}, d, w, nh[0]) != cudaSuccess)
            return IM3D_ERR_CUDA;
    }
    // a stream being captured into a graph cannot be synchronized: the graph orders the
    // work and its launch is the caller's to wait for
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
        cudaGetLastError();
        return IM3D_ERR_CUDA;
    }
    if (cs != cudaStreamCaptureStatusNone) return IM3D_OK;
    if (cudaStreamSynchronize(stream) != cudaSuccess) {
        cudaGetLastError();
        return IM3D_ERR_CUDA;
    }
    return IM3D_OK;
}

#endif  // IM3D_UNIT != 1

template <typename T>
int rsfe_apply(im3d_ctx* ctx, const T* myim_user, const T* init_user, int nx, int ny, int nz,
               double hx, double hy, double hz, const im3d_rsfe_params* p, T* phi_user, T* u_user,
               T* f1_user, T* f2_user, im3d_rsfe_stats* stats);

// Worker contexts of the batched entry points: own stream and buffers each.
int ensure_workers(im3d_ctx* ctx, int n)
{
    while ((int)ctx->workers.size() < n) {
        im3d_ctx* w = nullptr;
        const int st = im3d_ctx_create(ctx->device, &w);
        if (st != IM3D_OK) return fail(ctx, st, "cannot create a worker context");
        w->mem_limit = ctx->mem_limit;
        w->ifit_chunks = ctx->ifit_chunks;
        w->tile_loads = ctx->tile_loads;
        ctx->workers.push_back(w);
    }
    for (im3d_ctx* w : ctx->workers) w->prof = 0;
    return IM3D_OK;
}

// ------------------------------------------------------------ work-list batch
// Volumes of a group advance their outer iterations together; each stage of the loop
// is one launch over every volume that runs it (worklist.cuh).

template <class Job>
struct JobTable {
    std::vector<JobSlot<Job>> h;
    JobSlot<Job>* d = nullptr;
};

template <class Job>
int upload_jobs(im3d_ctx* ctx, const char* name, JobTable<Job>& t)
{
    IM3D_TRY(tbuf<JobSlot<Job>>(ctx, name, t.h.size(), &t.d));
    IM3D_CUDA(ctx, cudaMemcpyAsync(t.d, t.h.data(), t.h.size() * sizeof(JobSlot<Job>),
                                   cudaMemcpyHostToDevice, ctx->stream));
    return IM3D_OK;
}

WorkList make_worklist(const std::vector<int>& sel, const int* flags)
{
    WorkList wl;
    wl.n = (int)sel.size();
    for (int e = 0; e < wl.n; ++e) {
        wl.vol[e] = sel[e];
        wl.flag[e] = flags ? flags[e] : 0;
    }
    return wl;
}

// One launch of a stage over the volumes `sel` (indices into the job table).
template <class Job, int THREADS, int MINB>
int wl_launch(im3d_ctx* ctx, const JobTable<Job>& t, const std::vector<int>& sel, const int* flags,
              dim3 blk, size_t smem, const char* name, bool dependent = false)
{
    if (sel.empty()) return IM3D_OK;
    WorkList wl = make_worklist(sel, flags);
    long long total = 0;
    for (int e = 0; e < wl.n; ++e) {
        const dim3 g = t.h[sel[e]].grid;
        wl.first[e] = (unsigned)total;
        total += (long long)g.x * g.y * g.z;
        if (total > 0x7fffffffLL) break;
    }
    wl.first[wl.n] = (unsigned)total;
    if (total > 0x7fffffffLL) return fail(ctx, IM3D_ERR_INVALID_ARG, "work list too large for one launch");
    auto kern = worklist_kernel<Job, THREADS, MINB>;
    IM3D_TRY(set_smem(ctx, kern, smem));
    const int pf = prof_begin(ctx, name);
    if (dependent) IM3D_TRY(launch_dependent(ctx, kern, dim3((unsigned)total), blk, t.d, wl));
    else kern<<<dim3((unsigned)total), blk, smem, ctx->stream>>>(t.d, wl);
    prof_end(ctx, pf);
    return check_launch(ctx, name);
}

// The partials of the last reduction of `sel` folded into each volume's control block.
int wl_finalize(im3d_ctx* ctx, const FinalizeJob* jobs, const std::vector<int>& sel, const int* flags,
                int nvals, int slot)
{
    if (sel.empty()) return IM3D_OK;
    const WorkList wl = make_worklist(sel, flags);
    finalize_worklist_kernel<<<wl.n, kFinThreads, 0, ctx->stream>>>(jobs, wl, nvals, slot);
    return check_launch(ctx, "finalize_sums");
}

// Whether a batch can run as a work list (the volumes were checked by check_dims).
template <typename T>
bool worklist_eligible(const im3d_rsfe_params* p, int nvol, const im3d_volume_desc* vols, int* nh_out)
{
    if (!(p->gs_rel_res_tol > 0) || p->omega != 1.0 || p->auto_extract_conn_comp || p->conv_cyclic)
        return false;
    int nh0 = 0;
    for (int v = 0; v < nvol; ++v) {
        std::vector<double> w;
        const double hs[3] = {p->gaussian_pixel_approach ? 1. : vols[v].hx,
                              p->gaussian_pixel_approach ? 1. : vols[v].hy,
                              p->gaussian_pixel_approach ? 1. : vols[v].hz};
        for (int a = 0; a < 3; ++a) {
            const int nh = gauss_taps_host(p->sigma, 3.0, hs[a], w);
            if (nh != 19 && nh != 25) return false;
            if (nh0 == 0) nh0 = nh;
            if (nh != nh0) return false;
        }
    }
    *nh_out = nh0;
    return true;
}

// Solve state of one subgroup of a work-list group (bytes of u and b_eff): about half
// of the 126 MB L2
constexpr size_t kSolveGroupBytes = 64ull << 20;

// Per-volume loop counters of a work-list group.
struct WlCount {
    bool done = false;
    long long total_sweeps = 0;
    int last_sweeps = 0, not_conv = 0, checks = 0, iterations = 0;
    double last_rel = -1;
    // the current Poisson solve (rb_solve's state)
    int s = 0, s_prev = 0, next = 0;
    double r_prev = -1, rate_used = 0, beff2 = -1, rel = -1;
    bool conv = false;
};

template <typename T, int S>
int worklist_group(im3d_ctx* ctx, const std::vector<int>& ids, const im3d_volume_desc* vols,
                   const im3d_rsfe_params* p, int streams, im3d_rsfe_stats* stats, double* latency_ms,
                   std::chrono::steady_clock::time_point t_start)
{
    const int nv = (int)ids.size();
    IM3D_TRY(ensure_workers(ctx, streams));
    const bool neu = p->bc == IM3D_BC_NEU;
    while ((int)ctx->vols.size() < nv) {
        im3d_ctx* v = nullptr;
        const int st = im3d_ctx_create(ctx->device, &v);
        if (st != IM3D_OK) return fail(ctx, st, "cannot create a volume context");
        ctx->vols.push_back(v);
    }
    if (ctx->wl_ctrl_cap < nv) {
        if (ctx->wl_ctrl_h) cudaFreeHost(ctx->wl_ctrl_h);
        ctx->wl_ctrl_h = nullptr;
        ctx->wl_ctrl_cap = 0;
        IM3D_CUDA(ctx, cudaMallocHost(&ctx->wl_ctrl_h, kMaxListVols * sizeof(Ctrl)));
        ctx->wl_ctrl_cap = kMaxListVols;
    }
    Ctrl* ctrl = nullptr;
    IM3D_TRY(tbuf<Ctrl>(ctx, "wl_ctrl", kMaxListVols, &ctrl, true));

    // set-up of every volume (its own buffers, on this stream); the device-memory
    // budget of the context covers the group as a whole
    std::vector<VolState<T>> V(nv);
    std::vector<double*> part_res(nv), part_cl(nv);
    for (int q = 0; q < nv; ++q) {
        im3d_ctx* vc = ctx->vols[q];
        vc->stream = ctx->stream;
        vc->ifit_chunks = ctx->ifit_chunks;
        vc->prof = 0;
        vc->err.clear();
        if (ctx->mem_limit) {
            size_t others = ctx->mem_held;
            for (int r = 0; r < (int)ctx->vols.size(); ++r)
                if (r != q) others += ctx->vols[r]->mem_held;
            vc->mem_limit = ctx->mem_limit > others ? ctx->mem_limit - others : 1;
        } else {
            vc->mem_limit = 0;
        }
        const im3d_volume_desc& dsc = vols[ids[q]];
        int st = rsfe_prepare<T>(vc, V[q], static_cast<const T*>(dsc.myim), static_cast<const T*>(dsc.init),
                                 dsc.nx, dsc.ny, dsc.nz, dsc.hx, dsc.hy, dsc.hz, p, nullptr, nullptr,
                                 nullptr, nullptr, nullptr);
        const Dims& d = V[q].d;
        const dim3 gr = grid_rb_flat<T>(d, kBlkVec, 2, kNVres);
        const bool vec = d.nz % V16<T>::W == 0;
        const dim3 gc = vec ? grid_vec<T>(d, kBlkVec) : grid_col(d, kBlkVol);
        if (st == IM3D_OK)
            st = tbuf<double>(vc, "wl_part_res", 2 * (size_t)gr.x * gr.y * gr.z, &part_res[q]);
        if (st == IM3D_OK)
            st = tbuf<double>(vc, "wl_part_clamp", 2 * (size_t)gc.x * gc.y * gc.z, &part_cl[q]);
        if (st != IM3D_OK) return fail(ctx, st, "volume " + std::to_string(ids[q]) + ": " + vc->err);
    }

    // job tables: every stage's arguments and grid, per volume
    constexpr int R = SWinR<T>::v;
    using KHeav = ConvKWinJob<T, 4, S, kKwT, kKwR, LdHeaviside<T>, StVec<T, 4>, KWinRG<T, 4>::v>;
    using SJ4 = ConvSWinJob<T, 4, 1, S, TW, TY, R, LdVec<T, 4>, StVec<T, 4>>;
    using SJ2 = ConvSWinJob<T, 2, 1, S, TW, TY, R, LdVec<T, 2>, StVec<T, 2>>;
    using KRhs = ConvKWinJob<T, 2, S, kKwT, kKwR, LdVec<T, 2>, StRhs<T>, KWinRG<T, 2>::v>;
    using FitM = FitMarchJob<S, kMarchJB, kMarchD, kMarchU, MarchMinB<S>::v>;
    using FitW = FitWinJob<T, S, TW, TY, TileA<T>::v>;
    constexpr int RB_MINB = sizeof(T) == 4 ? 8 : 1;
    using RbD = RbHalfJob<T, kNV, false, RB_MINB>;
    using RbN = RbHalfJob<T, kNV, true, 1>;
    using Res = RbResidualJob<T, kNVres>;
    using ClV = ClampTolJob<T, kNV, true>;
    using ClS = ClampTolJob<T, kNI, false>;
    using BrV = BregmanJob<T, kNV, true>;
    using BrS = BregmanJob<T, kNIbr, false>;
    using DvV = DivJob<T, kNV, true>;
    using DvS = DivJob<T, 0, false>;
    JobTable<KHeav> jk;
    JobTable<SJ4> js4;
    JobTable<SJ2> js2;
    JobTable<KRhs> jr;
    JobTable<FitM> jfm;
    JobTable<FitW> jfw;
    JobTable<RbD> jrd[2];
    JobTable<RbN> jrn[2];
    JobTable<Res> jres;
    JobTable<ClV> jclv;
    JobTable<ClS> jcls;
    JobTable<BrV> jbrv;
    JobTable<BrS> jbrs;
    JobTable<DvV> jdvv;
    JobTable<DvS> jdvs;
    std::vector<FinalizeJob> fin_res(nv), fin_cl(nv);
    std::vector<char> vecrow(nv);
    const T l1 = (T)p->lamda1, l2 = (T)p->lamda2;
    for (int q = 0; q < nv; ++q) {
        const VolState<T>& v = V[q];
        const Dims& d = v.d;
        const double hx = vols[ids[q]].hx, hy = vols[ids[q]].hy, hz = vols[ids[q]].hz;
        jk.h.push_back({KHeav{LdHeaviside<T>{v.phi, v.u0, d, v.center, v.inv_eps}, StVec<T, 4>{v.W1, d}, d,
                              v.tp.w[2]}, k_win_grid<T, 4>(d)});
        js4.h.push_back({SJ4{LdVec<T, 4>{v.W1, d}, StVec<T, 4>{v.W2, d}, d, v.tp.w[1]}, s_win_grid<T, 1>(d)});
        js2.h.push_back({SJ2{LdVec<T, 2>{v.P1, d}, StVec<T, 2>{v.P2, d}, d, v.tp.w[1]}, s_win_grid<T, 1>(d)});
        StRhs<T> st;
        st.u0 = v.u0; st.kones = v.kones; st.divdb = v.divdb; st.phi = v.phi;
        st.out = v.bpk;
        st.upk = v.upk;
        st.beff2 = nullptr;
        st.d = d;
        st.l12 = (T)(p->lamda1 - p->lamda2);
        st.lamda = (T)p->lamda;
        st.inv_lamda = (T)(1.0 / p->lamda);
        st.inv_dt = (T)(1.0 / p->dt);
        st.bc = (T)v.chosen_bc;
        st.mode = 2;
        st.dirichlet = neu ? 0 : 1;
        jr.h.push_back({KRhs{LdVec<T, 2>{v.P2, d}, st, d, v.tp.w[2]}, k_win_grid<T, 2>(d)});
        if constexpr (sizeof(T) == 4) {
            dim3 g;
            const int chunk = march_chunk<S>(ctx->vols[q], d, &g);
            jfm.h.push_back({FitM{reinterpret_cast<const float4*>(v.W2), reinterpret_cast<float2*>(v.P1),
                                  v.f1_d, v.f2_d, d, tap_pairs<S>(v.tp.host[0]), l1, l2, chunk}, g});
        } else {
            jfw.h.push_back({FitW{v.W2, v.P1, v.f1_d, v.f2_d, d, v.tp.w[0], l1, l2}, fit_win_grid<T>(d)});
        }
        const dim3 gpk = grid_rb_flat<T>(d, kBlkVec);
        for (int c = 0; c < 2; ++c) {
            // red walks the planes forward, black backward (rb_sweep)
            jrd[c].h.push_back({RbD{v.upk, v.bpk, d, v.coef, c, c}, gpk});
            jrn[c].h.push_back({RbN{v.upk, v.bpk, d, v.coef, c, c}, gpk});
        }
        const dim3 gr = grid_rb_flat<T>(d, kBlkVec, 2, kNVres);
        jres.h.push_back({Res{v.upk, v.bpk, d, v.coef, part_res[q]}, gr});
        fin_res[q] = FinalizeJob{part_res[q], (long long)gr.x * gr.y * gr.z, ctrl[q].sum};
        vecrow[q] = d.nz % V16<T>::W == 0;
        const dim3 gv = grid_vec<T>(d, kBlkVec), gcol = grid_col(d, kBlkVol), gvol = grid_vol(d, kBlkVol);
        jclv.h.push_back({ClV{v.upk, v.phi, nullptr, d, v.a0, v.b0, part_cl[q]}, gv});
        jcls.h.push_back({ClS{v.upk, v.phi, nullptr, d, v.a0, v.b0, part_cl[q]}, gcol});
        const dim3 gcl = vecrow[q] ? gv : gcol;
        fin_cl[q] = FinalizeJob{part_cl[q], (long long)gcl.x * gcl.y * gcl.z, ctrl[q].sum};
        jbrv.h.push_back({BrV{v.phi, v.b3, v.dmb, v.g, d, hx, hy, hz}, gv});
        jbrs.h.push_back({BrS{v.phi, v.b3, v.dmb, v.g, d, hx, hy, hz}, grid_col(d, kBlkVol, kNIbr)});
        jdvv.h.push_back({DvV{v.dmb, v.divdb, d, hx, hy, hz}, gv});
        jdvs.h.push_back({DvS{v.dmb, v.divdb, d, hx, hy, hz}, gvol});
    }
    IM3D_TRY(upload_jobs(ctx, "wl_k_heaviside", jk));
    IM3D_TRY(upload_jobs(ctx, "wl_s_j4", js4));
    IM3D_TRY(upload_jobs(ctx, "wl_s_j2", js2));
    IM3D_TRY(upload_jobs(ctx, "wl_k_rhs", jr));
    if constexpr (sizeof(T) == 4) IM3D_TRY(upload_jobs(ctx, "wl_fit", jfm));
    else IM3D_TRY(upload_jobs(ctx, "wl_fit", jfw));
    for (int c = 0; c < 2; ++c) {
        if (neu) IM3D_TRY(upload_jobs(ctx, c ? "wl_rb1" : "wl_rb0", jrn[c]));
        else IM3D_TRY(upload_jobs(ctx, c ? "wl_rb1" : "wl_rb0", jrd[c]));
    }
    IM3D_TRY(upload_jobs(ctx, "wl_residual", jres));
    IM3D_TRY(upload_jobs(ctx, "wl_clamp_v", jclv));
    IM3D_TRY(upload_jobs(ctx, "wl_clamp_s", jcls));
    IM3D_TRY(upload_jobs(ctx, "wl_bregman_v", jbrv));
    IM3D_TRY(upload_jobs(ctx, "wl_bregman_s", jbrs));
    IM3D_TRY(upload_jobs(ctx, "wl_div_v", jdvv));
    IM3D_TRY(upload_jobs(ctx, "wl_div_s", jdvs));
    FinalizeJob *fin_res_d = nullptr, *fin_cl_d = nullptr;
    IM3D_TRY(tbuf<FinalizeJob>(ctx, "wl_fin_res", nv, &fin_res_d));
    IM3D_TRY(tbuf<FinalizeJob>(ctx, "wl_fin_clamp", nv, &fin_cl_d));
    IM3D_CUDA(ctx, cudaMemcpyAsync(fin_res_d, fin_res.data(), nv * sizeof(FinalizeJob), cudaMemcpyHostToDevice,
                                   ctx->stream));
    IM3D_CUDA(ctx, cudaMemcpyAsync(fin_cl_d, fin_cl.data(), nv * sizeof(FinalizeJob), cudaMemcpyHostToDevice,
                                   ctx->stream));

    std::vector<WlCount> C(nv);
    std::vector<double> tol(nv), sched_rate(nv);
    std::vector<int> sched_first(nv), init_vars(nv);
    for (int q = 0; q < nv; ++q) {
        tol[q] = V[q].tollerance;
        sched_first[q] = V[q].sched_first;
        sched_rate[q] = V[q].sched_rate;
        init_vars[q] = V[q].init_variables;
    }
    auto split = [&](const std::vector<int>& sel, std::vector<int>& a, std::vector<int>& b) {
        a.clear();
        b.clear();
        for (int q : sel) (vecrow[q] ? a : b).push_back(q);
    };
    const size_t smem_k4 = k_win_smem<T, 4, S>(), smem_k2 = k_win_smem<T, 2, S>();
    const size_t smem_s4 = s_win_smem<T, 4, S>(), smem_s2 = s_win_smem<T, 2, S>();
    const dim3 blk_k(kKwT, kKwR), blk_s(TW, TY);
    std::vector<int> act, sv, ss;
    // a volume whose loop would not start (maxiter < 1) returns its initial level set
    for (int q = 0; q < nv; ++q)
        if (!(tol[q] > p->tol) || p->maxiter < 1) {
            C[q].done = true;
            IM3D_CUDA(ctx, cudaMemcpyAsync(vols[ids[q]].phi_out, V[q].phi, V[q].n * sizeof(T), cudaMemcpyDefault,
                                           ctx->stream));
        }
    IM3D_TRY(sync(ctx));
    for (int q = 0; q < nv; ++q)
        if (C[q].done && latency_ms)
            latency_ms[ids[q]] =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    for (int t = 1;; ++t) {
        act.clear();
        for (int q = 0; q < nv; ++q)
            if (!C[q].done) act.push_back(q);
        if (act.empty()) break;
        // stage 1-5: Heaviside, the four convolutions, fitting terms, forcing term
        IM3D_TRY((wl_launch<KHeav, kKwT * kKwR, 3>(ctx, jk, act, nullptr, blk_k, smem_k4, "conv_k_heaviside")));
        IM3D_TRY((wl_launch<SJ4, TW * TY, 2>(ctx, js4, act, nullptr, blk_s, smem_s4, "conv_s_j4")));
        if constexpr (sizeof(T) == 4)
            IM3D_TRY((wl_launch<FitM, 32 * kMarchJB, MarchMinB<S>::v>(ctx, jfm, act, nullptr, dim3(32, kMarchJB), 0,
                                                                       "conv_i_fit")));
        else
            IM3D_TRY((wl_launch<FitW, TW * TY, 1>(ctx, jfw, act, nullptr, blk_s, fit_win_smem<T, S>(), "conv_i_fit")));
        IM3D_TRY((wl_launch<SJ2, TW * TY, 3>(ctx, js2, act, nullptr, blk_s, smem_s2, "conv_s_j2")));
        IM3D_TRY((wl_launch<KRhs, kKwT * kKwR, 3>(ctx, jr, act, nullptr, blk_k, smem_k2, "conv_k_rhs")));

        // the Poisson step: rb_solve for every volume, the half-sweeps of all unconverged
        // volumes in one launch, a residual check for each volume when its schedule
        // (next_check) asks for one
        const int maxs = std::max(p->gs_max_sweeps, 1);
        const int every = std::max(p->gs_check_every, 0);
        for (int q : act) {
            WlCount& c = C[q];
            c.s = 0;
            c.s_prev = 0;
            c.r_prev = -1;
            c.rate_used = 0;
            c.beff2 = -1;
            c.rel = -1;
            c.conv = false;
            c.next = every > 0 ? every : (sched_first[q] > 0 ? sched_first[q] : 4);
        }
        const int pfs = prof_begin(ctx, "poisson_solve");
        // the volumes solve in subgroups whose solve state (u and b_eff, colour-packed)
        // fits in L2 together, so that consecutive half-sweeps re-read it from L2 as a
        // single volume's do; one launch per half-sweep covers the subgroup
        std::vector<std::vector<int>> sub;
        size_t sub_bytes = 0;
        for (int q : act) {
            const size_t b = (size_t)V[q].npk2 * 2 * sizeof(T);
            if (sub.empty() || sub_bytes + b > kSolveGroupBytes) {
                sub.emplace_back();
                sub_bytes = 0;
            }
            sub.back().push_back(q);
            sub_bytes += b;
        }
        // one subgroup's solves on the context `sc` (its stream): the half-sweeps of its
        // unconverged volumes in one launch each, a residual check of each volume on its
        // own schedule; the volumes of a subgroup have consecutive indices, so their
        // control blocks are one range
        auto solve_group = [&](im3d_ctx* sc, const std::vector<int>& grp) -> int {
            std::vector<int> solving = grp, due, flags, still;
            const int q0 = grp.front(), q1 = grp.back() + 1;
            while (!solving.empty()) {
                int k = maxs;
                for (int q : solving) k = std::min(k, std::min(C[q].next, maxs) - C[q].s);
                k = std::max(k, 1);
                for (int i = 0; i < k; ++i)
                    for (int c = 0; c < 2; ++c) {
                        if (neu)
                            IM3D_TRY((wl_launch<RbN, 128, 1>(sc, jrn[c], solving, nullptr, kBlkVec, 0, "rb_half", true)));
                        else
                            IM3D_TRY((wl_launch<RbD, 128, RB_MINB>(sc, jrd[c], solving, nullptr, kBlkVec, 0, "rb_half",
                                                                   true)));
                    }
                due.clear();
                flags.clear();
                for (int q : solving) {
                    C[q].s += k;
                    if (C[q].s >= C[q].next || C[q].s == maxs) {
                        due.push_back(q);
                        flags.push_back(C[q].beff2 < 0 ? 1 : 0);
                    }
                }
                IM3D_TRY((wl_launch<Res, 256, 4>(sc, jres, due, flags.data(), kBlkVec, 0, "rb_residual")));
                IM3D_TRY(wl_finalize(sc, fin_res_d, due, flags.data(), 1, SUM_RES2));
                IM3D_CUDA(sc, cudaMemcpyAsync(ctx->wl_ctrl_h + q0, ctrl + q0, (q1 - q0) * sizeof(Ctrl),
                                              cudaMemcpyDeviceToHost, sc->stream));
                IM3D_CUDA(sc, cudaStreamSynchronize(sc->stream));
                still.clear();
                for (int q : solving) {
                    WlCount& c = C[q];
                    const bool checked = c.s >= c.next || c.s == maxs;
                    if (checked) {
                        ++c.checks;
                        const Ctrl& cb = ctx->wl_ctrl_h[q];
                        if (c.beff2 < 0) c.beff2 = cb.sum[SUM_BEFF2];
                        const double rr = cb.sum[SUM_RES2];
                        const double r = c.beff2 > 0 ? std::sqrt(rr) / std::sqrt(c.beff2) : std::sqrt(rr);
                        c.rel = r;
                        if (r <= p->gs_rel_res_tol) {
                            c.conv = true;
                            continue;
                        }
                        if (c.s >= maxs) continue;  // not converged
                        c.next = next_check(c.s, r, c.s_prev, c.r_prev, p->gs_rel_res_tol, every, sched_rate[q],
                                            &c.rate_used);
                        if (c.next > maxs) c.next = maxs;
                        c.s_prev = c.s;
                        c.r_prev = r;
                    }
                    still.push_back(q);
                }
                solving.swap(still);
            }
            return IM3D_OK;
        };
        // the subgroups run concurrently on the worker streams, each after the forcing
        // terms are written (so a worker's residual round trips overlap the others'
        // sweeps); the loop's stream then waits for all of them
        const int nw = std::min<int>(streams, (int)sub.size());
        IM3D_CUDA(ctx, cudaEventRecord(ctx->wl_ev[0], ctx->stream));
        std::atomic<int> next_sub(0);
        std::vector<int> wst(nw, IM3D_OK);
        auto work = [&](int w) {
            im3d_ctx* wc = ctx->workers[w];
            cudaSetDevice(wc->device);
            wc->err.clear();
            if (cudaStreamWaitEvent(wc->stream, ctx->wl_ev[0], 0) != cudaSuccess) {
                wst[w] = fail(wc, IM3D_ERR_CUDA, "cannot order a worker stream after the forcing terms");
                return;
            }
            for (int g = next_sub++; g < (int)sub.size(); g = next_sub++) {
                wst[w] = solve_group(wc, sub[g]);
                if (wst[w] != IM3D_OK) break;
            }
            cudaEventRecord(wc->wl_ev[1], wc->stream);
        };
        {
            std::vector<std::thread> pool;
            for (int w = 1; w < nw; ++w) pool.emplace_back(work, w);
            work(0);
            for (auto& th : pool) th.join();
        }
        cudaSetDevice(ctx->device);
        for (int w = 0; w < nw; ++w) {
            ctx->launches += ctx->workers[w]->launches;
            ctx->workers[w]->launches = 0;
            if (wst[w] != IM3D_OK) return fail(ctx, wst[w], ctx->workers[w]->err);
            IM3D_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->workers[w]->wl_ev[1], 0));
        }
        prof_end(ctx, pfs);
        for (int q : act) {
            WlCount& c = C[q];
            const double rate = c.rate_used > 0 ? c.rate_used : sched_rate[q];
            sched_first[q] = c.conv ? c.s : 0;
            sched_rate[q] = c.conv ? rate : 0;
            if (!c.conv) c.not_conv++;
            c.total_sweeps += c.s;
            c.last_sweeps = c.s;
            c.last_rel = c.rel;
        }

        // clamp and tolerance, then the Bregman update and div(d - b)
        split(act, sv, ss);
        IM3D_TRY((wl_launch<ClV, 256, 4>(ctx, jclv, sv, nullptr, kBlkVec, 0, "clamp_tol")));
        IM3D_TRY((wl_launch<ClS, 256, 1>(ctx, jcls, ss, nullptr, kBlkVol, 0, "clamp_tol_columns")));
        IM3D_TRY(wl_finalize(ctx, fin_cl_d, act, nullptr, 2, SUM_DPHI2));
        IM3D_CUDA(ctx, cudaMemcpyAsync(ctx->wl_ctrl_h, ctrl, nv * sizeof(Ctrl), cudaMemcpyDeviceToHost, ctx->stream));
        IM3D_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
        std::vector<int> upd;
        for (int q : act) {
            if (init_vars[q]) {
                IM3D_CUDA(ctx, cudaMemsetAsync(V[q].divdb, 0, V[q].n * sizeof(T), ctx->stream));
                IM3D_CUDA(ctx, cudaMemsetAsync(V[q].b3, 0, 3 * V[q].n * sizeof(T), ctx->stream));
                init_vars[q] = 0;
            } else {
                upd.push_back(q);
            }
        }
        split(upd, sv, ss);
        IM3D_TRY((wl_launch<BrV, 256, 2>(ctx, jbrv, sv, nullptr, kBlkVec, 0, "bregman")));
        IM3D_TRY((wl_launch<BrS, 256, 1>(ctx, jbrs, ss, nullptr, kBlkVol, 0, "bregman_columns")));
        IM3D_TRY((wl_launch<DvV, 256, 3>(ctx, jdvv, sv, nullptr, kBlkVec, 0, "div")));
        IM3D_TRY((wl_launch<DvS, 256, 1>(ctx, jdvs, ss, nullptr, kBlkVol, 0, "div_columns")));
        if (cudaEventSynchronize(ctx->ev[3]) != cudaSuccess) IM3D_TRY(sync(ctx));
        for (int q : act) {
            const Ctrl& cb = ctx->wl_ctrl_h[q];
            tol[q] = std::sqrt(V[q].hhh * cb.sum[SUM_DPHI2]) / std::sqrt(V[q].hhh * cb.sum[SUM_PHIOLD2]);
            C[q].iterations = t;
            if (!(tol[q] > p->tol) || t + 1 > p->maxiter) C[q].done = true;
        }
        // volumes that finished: their result goes out now (latency)
        bool any = false;
        for (int q : act) any = any || C[q].done;
        if (any) {
            for (int q : act) {
                if (!C[q].done) continue;
                const im3d_volume_desc& dsc = vols[ids[q]];
                IM3D_CUDA(ctx, cudaMemcpyAsync(dsc.phi_out, V[q].phi, V[q].n * sizeof(T), cudaMemcpyDefault,
                                               ctx->stream));
            }
            IM3D_TRY(sync(ctx));
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start)
                                  .count();
            for (int q : act)
                if (C[q].done && latency_ms) latency_ms[ids[q]] = ms;
        }
    }
    if (stats) {
        for (int q = 0; q < nv; ++q) {
            im3d_rsfe_stats& st = stats[ids[q]];
            std::memset(&st, 0, sizeof(st));
            st.iterations = C[q].iterations;
            st.last_tol = tol[q];
            st.total_sweeps = C[q].total_sweeps;
            st.last_sweeps = C[q].last_sweeps;
            st.last_rel_res = C[q].last_rel;
            st.last_ls_err = -1;
            st.not_converged = C[q].not_conv;
            st.residual_checks = C[q].checks;
        }
    }
    return IM3D_OK;
}

// Work-list batch: groups of up to kMaxListVols volumes, largest first.
template <typename T>
int rsfe_apply_worklist(im3d_ctx* ctx, int nvol, const im3d_volume_desc* vols, const im3d_rsfe_params* p,
                        int nh, int streams, im3d_rsfe_stats* stats, double* latency_ms)
{
    std::vector<int> order(nvol);
    for (int v = 0; v < nvol; ++v) order[v] = v;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)vols[a].nx * vols[a].ny * vols[a].nz > (long long)vols[b].nx * vols[b].ny * vols[b].nz;
    });
    const auto t0 = std::chrono::steady_clock::now();
    for (int g0 = 0; g0 < nvol; g0 += kMaxListVols) {
        const std::vector<int> ids(order.begin() + g0, order.begin() + std::min(nvol, g0 + kMaxListVols));
        if (nh == 19) IM3D_TRY((worklist_group<T, 9>(ctx, ids, vols, p, streams, stats, latency_ms, t0)));
        else IM3D_TRY((worklist_group<T, 12>(ctx, ids, vols, p, streams, stats, latency_ms, t0)));
    }
    return IM3D_OK;
}

// Batch of independent volumes: a queue ordered largest first, drained by `streams`
// host workers, each owning a worker context (stream + buffers) of the same device.
template <typename T>
int rsfe_apply_batched(im3d_ctx* ctx, int nvol, const im3d_volume_desc* vols,
                       const im3d_rsfe_params* p, int streams, im3d_rsfe_stats* stats,
                       double* latency_ms)
{
    if (nvol < 0 || (nvol > 0 && !vols) || !p) return fail(ctx, IM3D_ERR_INVALID_ARG, "bad batch");
    if (nvol == 0) return IM3D_OK;
    if (streams <= 0) streams = 4;
    if (streams > 32) streams = 32;
    if (ctx->batch_mode == IM3D_BATCH_WORKLIST) {
        // the work list runs valid volumes only (the stream queue, the default, reports
        // each bad volume and segments the others)
        int st = check_params(ctx, p);
        for (int v = 0; v < nvol && st == IM3D_OK; ++v) {
            if (!vols[v].myim || !vols[v].phi_out)
                st = fail(ctx, IM3D_ERR_INVALID_ARG, "volume " + std::to_string(v) + ": myim and phi_out are required");
            else
                st = check_dims(ctx, vols[v].nx, vols[v].ny, vols[v].nz, vols[v].hx, vols[v].hy, vols[v].hz);
        }
        int nh = 0;
        if (st != IM3D_OK) return st;
        if (!worklist_eligible<T>(p, nvol, vols, &nh))
            return fail(ctx, IM3D_ERR_UNSUPPORTED, "the work-list batch needs a residual solve with omega 1, "
                                                   "19 or 25 Gaussian taps on every axis and no "
                                                   "connected-component extraction");
        return rsfe_apply_worklist<T>(ctx, nvol, vols, p, nh, streams, stats, latency_ms);
    }
    if (streams > nvol) streams = nvol;
    IM3D_TRY(ensure_workers(ctx, streams));
    std::vector<int> order(nvol);
    for (int v = 0; v < nvol; ++v) order[v] = v;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)vols[a].nx * vols[a].ny * vols[a].nz > (long long)vols[b].nx * vols[b].ny * vols[b].nz;
    });
    std::atomic<int> next(0);
    std::vector<int> status(nvol, IM3D_OK);
    std::vector<std::string> errs(nvol);
    const auto t0 = std::chrono::steady_clock::now();
    auto work = [&](int wid) {
        im3d_ctx* w = ctx->workers[wid];
        w->prof = ctx->prof;
        cudaSetDevice(w->device);
        for (int q = next++; q < nvol; q = next++) {
            const int v = order[q];
            const im3d_volume_desc& dsc = vols[v];
            im3d_rsfe_stats st;
            w->err.clear();
            status[v] = rsfe_apply<T>(w, static_cast<const T*>(dsc.myim), static_cast<const T*>(dsc.init),
                                      dsc.nx, dsc.ny, dsc.nz, dsc.hx, dsc.hy, dsc.hz, p,
                                      static_cast<T*>(dsc.phi_out), nullptr, nullptr, nullptr, &st);
            if (status[v] != IM3D_OK) errs[v] = w->err;
            if (stats) stats[v] = st;
            if (latency_ms)
                latency_ms[v] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    };
    std::vector<std::thread> pool;
    for (int wid = 1; wid < streams; ++wid) pool.emplace_back(work, wid);
    work(0);
    for (auto& t : pool) t.join();
    cudaSetDevice(ctx->device);
    for (int wid = 0; wid < streams; ++wid) {
        im3d_ctx* w = ctx->workers[wid];
        ctx->launches += w->launches;
        w->launches = 0;
        if (ctx->prof) {
            prof_resolve(w);
            for (auto& kv : w->prof_acc) {
                bool found = false;
                for (auto& mine : ctx->prof_acc)
                    if (mine.first == kv.first) {
                        mine.second.ms += kv.second.ms;
                        mine.second.count += kv.second.count;
                        found = true;
                    }
                if (!found) ctx->prof_acc.push_back(kv);
            }
            w->prof_acc.clear();
        }
    }
    for (int v = 0; v < nvol; ++v)
        if (status[v] != IM3D_OK) {
            ctx->err = "volume " + std::to_string(v) + ": " + errs[v];
            return status[v];
        }
    return IM3D_OK;
}

int enter(im3d_ctx* ctx)
{
    if (!ctx) return IM3D_ERR_INVALID_ARG;
    ctx->err.clear();
    IM3D_CUDA(ctx, cudaSetDevice(ctx->device));
    return IM3D_OK;
}

}  // namespace

#if IM3D_UNIT != 2
// ------------------------------------------------- shared with the other units
cudaStream_t im3d_ctx_stream(im3d_ctx* ctx) { return ctx->stream; }
int im3d_ctx_device(im3d_ctx* ctx) { return ctx->device; }
std::string& im3d_ctx_error_ref(im3d_ctx* ctx) { return ctx->err; }

// ====================================================================== C ABI
#endif

extern "C" {

#if IM3D_UNIT != 2
int im3d_ctx_create(int device, im3d_ctx** out)
{
    if (!out) return IM3D_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return IM3D_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return IM3D_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
        cudaGetLastError();
        return IM3D_ERR_NO_DEVICE;
    }
    im3d_ctx* ctx = new im3d_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->ctrl_d, sizeof(Ctrl)) != cudaSuccess ||
        cudaMallocHost(&ctx->ctrl_h, sizeof(Ctrl)) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return IM3D_ERR_CUDA;
    }
    for (int q = 0; q < 3; ++q) cudaEventCreate(&ctx->ev[q]);
    cudaEventCreateWithFlags(&ctx->ev[3], cudaEventDisableTiming);
    for (auto& e : ctx->wl_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    ctx->stream = ctx->own_stream;
    ctx->num_sms = prop.multiProcessorCount;
    *out = ctx;
    return IM3D_OK;
}

int im3d_ctx_destroy(im3d_ctx* ctx)
{
    if (!ctx) return IM3D_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (im3d_ctx* w : ctx->workers) im3d_ctx_destroy(w);
    for (im3d_ctx* v : ctx->vols) im3d_ctx_destroy(v);
    ctx->vols.clear();
    if (ctx->wl_ctrl_h) cudaFreeHost(ctx->wl_ctrl_h);
    ctx->workers.clear();
    cudaSetDevice(ctx->device);
    for (auto& kv : ctx->bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    if (ctx->ctrl_d) cudaFree(ctx->ctrl_d);
    if (ctx->ctrl_h) cudaFreeHost(ctx->ctrl_h);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : ctx->wl_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return IM3D_OK;
}

const char* im3d_ctx_last_error(const im3d_ctx* ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }

int im3d_ctx_set_stream(im3d_ctx* ctx, void* stream)
{
    if (!ctx) return IM3D_ERR_INVALID_ARG;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return IM3D_OK;
}

int64_t im3d_ctx_launch_count(const im3d_ctx* ctx) { return ctx ? ctx->launches : 0; }

int im3d_ctx_set_option(im3d_ctx* ctx, int option, int64_t value)
{
    if (!ctx) return IM3D_ERR_INVALID_ARG;
    if (value < 0) return fail(ctx, IM3D_ERR_INVALID_ARG, "option values are non negative");
    switch (option) {
    case IM3D_OPT_FIT_CHUNKS:
        ctx->ifit_chunks = value > 0x7fffffff ? 0x7fffffff : (int)value;
        return IM3D_OK;
    case IM3D_OPT_DEVICE_MEMORY_LIMIT:
        ctx->mem_limit = (size_t)value;
        for (im3d_ctx* w : ctx->workers) w->mem_limit = (size_t)value;
        return IM3D_OK;
    case IM3D_OPT_BATCH_MODE:
        if (value > IM3D_BATCH_WORKLIST) return fail(ctx, IM3D_ERR_INVALID_ARG, "unknown batch mode");
        ctx->batch_mode = (int)value;
        return IM3D_OK;
    case IM3D_OPT_TILE_LOADS:
        if (value > 1) return fail(ctx, IM3D_ERR_INVALID_ARG, "IM3D_OPT_TILE_LOADS is 0 or 1");
        ctx->tile_loads = (int)value;
        for (im3d_ctx* w : ctx->workers) w->tile_loads = (int)value;
        return IM3D_OK;
    default:
        return fail(ctx, IM3D_ERR_INVALID_ARG, "unknown option " + std::to_string(option));
    }
}

int im3d_ctx_set_observer(im3d_ctx* ctx, int every, int with_state, im3d_rsfe_observer cb, void* user)
{
    if (!ctx) return IM3D_ERR_INVALID_ARG;
    if (cb && every <= 0) return fail(ctx, IM3D_ERR_INVALID_ARG, "the observer needs every > 0");
    ctx->obs = cb;
    ctx->obs_user = user;
    ctx->obs_every = cb ? every : 0;
    ctx->obs_state = with_state ? 1 : 0;
    return IM3D_OK;
}

int im3d_ctx_set_warm_start(im3d_ctx* ctx, im3d_unet* net, int mode, double lr)
{
    if (!ctx) return IM3D_ERR_INVALID_ARG;
    if (mode != IM3D_WS_OFF && mode != IM3D_WS_PREDICT && mode != IM3D_WS_TRAIN)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "unknown warm-start mode");
    if (mode == IM3D_WS_TRAIN && !(lr > 0)) return fail(ctx, IM3D_ERR_INVALID_ARG, "training needs lr > 0");
    if (net && im3d::unet::net_device(net) != ctx->device)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "the network lives on another device");
    ctx->ws_net = mode == IM3D_WS_OFF ? nullptr : net;
    ctx->ws_mode = net ? mode : IM3D_WS_OFF;
    ctx->ws_lr = lr;
    return IM3D_OK;
}

int im3d_ctx_set_resume(im3d_ctx* ctx, const im3d_rsfe_checkpoint* from, int element_size)
{
    if (!ctx) return IM3D_ERR_INVALID_ARG;
    if (!from) {
        ctx->resume = false;
        return IM3D_OK;
    }
    if (element_size != 4 && element_size != 8)
        return fail(ctx, IM3D_ERR_INVALID_ARG, "element_size must be 4 or 8");
    ctx->resume = true;
    ctx->resume_from = *from;
    ctx->resume_esize = element_size;
    return IM3D_OK;
}

int im3d_ctx_set_profiling(im3d_ctx* ctx, int on)
{
    if (!ctx) return IM3D_ERR_INVALID_ARG;
    ctx->prof = on == 2 ? 2 : (on != 0 ? 1 : 0);
    return IM3D_OK;
}

int im3d_ctx_profile(im3d_ctx* ctx, char* names, int names_cap, double* ms, int64_t* counts,
                     int max_entries, int reset)
{
    if (!ctx) return -IM3D_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return -IM3D_ERR_CUDA;
    }
    prof_resolve(ctx);
    int n = 0;
    std::string all;
    for (auto& kv : ctx->prof_acc) {
        if (n >= max_entries) break;
        if (ms) ms[n] = kv.second.ms;
        if (counts) counts[n] = kv.second.count;
        all += kv.first;
        all += '\n';
        ++n;
    }
    if (names && names_cap > 0) {
        std::strncpy(names, all.c_str(), (size_t)names_cap - 1);
        names[names_cap - 1] = 0;
    }
    if (reset) ctx->prof_acc.clear();
    return n;
}

void im3d_rsfe_params_default(im3d_rsfe_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // rsfe_splitbregman_imp.hxx:25-41
    p->tol = 1.e-5;
    p->sigma = 3;
    p->lamda = 5.e-2;
    p->lamda1 = 1.e-5;
    p->lamda2 = 1.e-5;
    p->beta = 100.;
    p->nu = 1.;
    p->dt = 1;
    p->epsilon = 1.e-3;
    p->a0 = 0.;
    p->b0 = 1.;
    p->ls_tol = 0;
    p->edge_detector_sigma = 0;
    p->maxiter = 100;
    p->ls_steps = 5;
    p->bc = IM3D_BC_DEFAULT;
    p->gaussian_pixel_approach = 0;
    p->init_variables = 0;
    // extensions
    p->sweep = IM3D_SWEEP_LEXICOGRAPHIC;
    p->gs_rel_res_tol = 0;
    p->omega = 1.0;
    p->gs_max_sweeps = 1000;
    p->gs_check_every = 0;
    // connected-component extraction (rsfe_splitbregman_imp.hxx:32-33, 40)
    p->cc_init_pixel_x = -1;
    p->cc_init_pixel_y = -1;
    p->cc_init_pixel_z = -1;
    p->alpha = (p->a0 + p->b0) / 2.;
    p->auto_extract_conn_comp = 0;
    p->auto_extract_conn_comp_freq = 0;
    p->cc_binary_output = 1;
    p->cc_init_variables = 1;
    p->conv_cyclic = 0;
    p->reserved_ = 0;
}
#endif  // generic entry points

#define IM3D_ENTRY(...)                \
    do {                               \
        int s_ = enter(ctx);           \
        if (s_ != IM3D_OK) return s_;  \
        return __VA_ARGS__;            \
    } while (0)

#if IM3D_UNIT != 2
int im3d_gauss_filter_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny, int nz,
                          double hx, double hy, double hz, double sigma, double radius,
                          int pixel_approach)
{
    IM3D_ENTRY(gauss_filter<double>(ctx, in, out, nx, ny, nz, hx, hy, hz, sigma, radius, pixel_approach));
}

int im3d_connected_component_f64(im3d_ctx* ctx, const double* img, double* res, int nx, int ny,
                                 int nz, const double* init, int i, int j, int k, double threshold,
                                 int full_connected, int binary_output, int* passes)
{
    IM3D_ENTRY(connected_component_op<double>(ctx, img, res, nx, ny, nz, init, i, j, k, threshold,
                                              full_connected, binary_output, passes));
}

int im3d_gauss_filter_cyclic_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny,
                                 int nz, double hx, double hy, double hz, double sigma,
                                 double radius, int pixel_approach)
{
    IM3D_ENTRY(gauss_filter<double>(ctx, in, out, nx, ny, nz, hx, hy, hz, sigma, radius,
                                    pixel_approach, 1));
}

int im3d_poisson_sweeps_f64(im3d_ctx* ctx, double* res, const double* b, int nx, int ny, int nz,
                            double hx, double hy, double hz, double dt, double bc, int bc_type,
                            int sweep_order, int sweeps)
{
    IM3D_ENTRY(poisson_sweeps<double>(ctx, res, b, nx, ny, nz, hx, hy, hz, dt, bc, bc_type, sweep_order, sweeps));
}

int im3d_poisson_solve_f64(im3d_ctx* ctx, double* u, const double* b, int nx, int ny, int nz,
                           double hx, double hy, double hz, double dt, double bc, int bc_type,
                           double rel_res_tol, int max_sweeps, int check_every, double omega,
                           int* sweeps_done, double* rel_res)
{
    IM3D_ENTRY(poisson_solve<double>(ctx, u, b, nx, ny, nz, hx, hy, hz, dt, bc, bc_type, rel_res_tol,
                                     max_sweeps, check_every, omega, sweeps_done, rel_res));
}

int im3d_grad_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny, int nz, double hx,
                  double hy, double hz)
{
    IM3D_ENTRY(grad_op<double>(ctx, in, out, nx, ny, nz, hx, hy, hz));
}

int im3d_div_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny, int nz, double hx,
                 double hy, double hz)
{
    IM3D_ENTRY(div_op<double>(ctx, in, out, nx, ny, nz, hx, hy, hz));
}

int im3d_rsfe_apply_f64(im3d_ctx* ctx, const double* myim, const double* init, int nx, int ny,
                        int nz, double hx, double hy, double hz, const im3d_rsfe_params* p,
                        double* phi_out, double* u_out, double* f1_out, double* f2_out,
                        im3d_rsfe_stats* stats)
{
    IM3D_ENTRY(rsfe_apply<double>(ctx, myim, init, nx, ny, nz, hx, hy, hz, p, phi_out, u_out, f1_out,
                                  f2_out, stats));
}

int im3d_rsfe_apply_batched_f64(im3d_ctx* ctx, int nvol, const im3d_volume_desc* vols,
                                const im3d_rsfe_params* p, int streams, im3d_rsfe_stats* stats,
                                double* latency_ms)
{
    IM3D_ENTRY(rsfe_apply_batched<double>(ctx, nvol, vols, p, streams, stats, latency_ms));
}
#endif  // FP64 entry points

#if IM3D_UNIT != 1
int im3d_gauss_filter_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny, int nz,
                          double hx, double hy, double hz, double sigma, double radius,
                          int pixel_approach)
{
    IM3D_ENTRY(gauss_filter<float>(ctx, in, out, nx, ny, nz, hx, hy, hz, sigma, radius, pixel_approach));
}

int im3d_connected_component_f32(im3d_ctx* ctx, const float* img, float* res, int nx, int ny,
                                 int nz, const float* init, int i, int j, int k, double threshold,
                                 int full_connected, int binary_output, int* passes)
{
    IM3D_ENTRY(connected_component_op<float>(ctx, img, res, nx, ny, nz, init, i, j, k, threshold,
                                             full_connected, binary_output, passes));
}

int im3d_gauss_filter_cyclic_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny,
                                 int nz, double hx, double hy, double hz, double sigma,
                                 double radius, int pixel_approach)
{
    IM3D_ENTRY(gauss_filter<float>(ctx, in, out, nx, ny, nz, hx, hy, hz, sigma, radius,
                                   pixel_approach, 1));
}

int im3d_poisson_sweeps_f32(im3d_ctx* ctx, float* res, const float* b, int nx, int ny, int nz,
                            double hx, double hy, double hz, double dt, double bc, int bc_type,
                            int sweep_order, int sweeps)
{
    IM3D_ENTRY(poisson_sweeps<float>(ctx, res, b, nx, ny, nz, hx, hy, hz, dt, bc, bc_type, sweep_order, sweeps));
}

int im3d_poisson_solve_f32(im3d_ctx* ctx, float* u, const float* b, int nx, int ny, int nz,
                           double hx, double hy, double hz, double dt, double bc, int bc_type,
                           double rel_res_tol, int max_sweeps, int check_every, double omega,
                           int* sweeps_done, double* rel_res)
{
    IM3D_ENTRY(poisson_solve<float>(ctx, u, b, nx, ny, nz, hx, hy, hz, dt, bc, bc_type, rel_res_tol,
                                    max_sweeps, check_every, omega, sweeps_done, rel_res));
}

int im3d_gauss_filter_f32_noalloc(const float* in, float* out, int nx, int ny, int nz,
                                  double hx, double hy, double hz, double sigma, double radius,
                                  int pixel_approach, void* stream)
{
    return gauss_filter_noalloc(in, out, nx, ny, nz, hx, hy, hz, sigma, radius, pixel_approach,
                                (cudaStream_t)stream);
}

int im3d_grad_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny, int nz, double hx,
                  double hy, double hz)
{
    IM3D_ENTRY(grad_op<float>(ctx, in, out, nx, ny, nz, hx, hy, hz));
}

int im3d_div_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny, int nz, double hx,
                 double hy, double hz)
{
    IM3D_ENTRY(div_op<float>(ctx, in, out, nx, ny, nz, hx, hy, hz));
}

int im3d_rsfe_apply_f32(im3d_ctx* ctx, const float* myim, const float* init, int nx, int ny, int nz,
                        double hx, double hy, double hz, const im3d_rsfe_params* p, float* phi_out,
                        float* u_out, float* f1_out, float* f2_out, im3d_rsfe_stats* stats)
{
    IM3D_ENTRY(rsfe_apply<float>(ctx, myim, init, nx, ny, nz, hx, hy, hz, p, phi_out, u_out, f1_out,
                                 f2_out, stats));
}

int im3d_rsfe_apply_batched_f32(im3d_ctx* ctx, int nvol, const im3d_volume_desc* vols,
                                const im3d_rsfe_params* p, int streams, im3d_rsfe_stats* stats,
                                double* latency_ms)
{
    IM3D_ENTRY(rsfe_apply_batched<float>(ctx, nvol, vols, p, streams, stats, latency_ms));
}
#endif  // FP32 entry points

}  // extern "C"

/*
 * im3d_b200.h -- C ABI of the B200 (sm_100a) backend for 3dimagetoolkit's
 * RSFE Split-Bregman level-set segmentation path.
 *
 * Every entry point returns an int status (IM3D_OK = 0). No C++ types, no torch
 * types cross this boundary: plain pointers, sizes and POD structs only.
 *
 * Volumes follow the reference's image3d layout (header/image3d_imp.hxx:142-153):
 * element (i, j, k) of an nx x ny x nz volume sits at index (i*ny + j)*nz + k, so k
 * is the contiguous axis. Spacings are hx, hy, hz.
 *
 * Pointer arguments may be host memory (pageable or pinned) or device memory of
 * the context's device; the library asks the CUDA runtime which one each pointer
 * is and stages host buffers through device buffers that the context owns. All
 * calls on one context are serialised on the context's stream and return after
 * the results are in the caller's buffers.
 *
 * Status codes map to the reference's WARNING behaviour: the reference prints a
 * WARNING and returns (e.g. image3d_imp.hxx:221-225, rsfe_splitbregman_imp.hxx:957-960);
 * here the call returns a non-zero status and im3d_ctx_last_error() holds the text.
 */
#ifndef IM3D_B200_H
#define IM3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IM3D_OK 0
#define IM3D_ERR_INVALID_ARG 1   /* bad size, spacing or parameter */
#define IM3D_ERR_UNSUPPORTED 2   /* 2-D volumes (nz == 1) and dims < 3: not on this backend */
#define IM3D_ERR_NOT_CONVERGED 3 /* a sweep cap was hit before the requested tolerance */
#define IM3D_ERR_CUDA 4          /* a CUDA runtime call failed (text in last_error) */
#define IM3D_ERR_OOM 5           /* device allocation failed */
#define IM3D_ERR_NO_DEVICE 6     /* no usable sm_100 device */
#define IM3D_ERR_TOO_LARGE 7     /* volume above the fixed scratch of a no-allocation entry point */
#define IM3D_ERR_NONFINITE 8     /* an input volume holds NaN or Inf (the reference's debug build
                                    traps such values as floating-point exceptions,
                                    exceptions.hxx:25-35; here the call refuses them) */

/* Boundary condition selector. The reference keeps bc_type private
 * (rsfe_splitbregman.hxx:108); its constructor sets bc = NEU but installs
 * DirGaussSeidel (rsfe_splitbregman_imp.hxx:33-35), so an untouched instance solves
 * with Dirichlet value 0. IM3D_BC_DEFAULT reproduces that; NEU and DIR reproduce
 * set_bc(NEU) / set_bc(DIR) (rsfe_splitbregman_imp.hxx:1294-1322). */
#define IM3D_BC_DEFAULT 0
#define IM3D_BC_NEU 1
#define IM3D_BC_DIR 2

/* Order of the Gauss-Seidel point updates inside one sweep.
 * LEXICOGRAPHIC reproduces lapl::DirGaussSeidel / lapl::NeuGaussSeidel exactly
 * (poisson_imp.hxx:340-429 / 23-336): every point sees new values at its minus
 * neighbours and old values at its plus neighbours. REDBLACK updates the points
 * with even (i+j+k) first, then the odd ones, with the same per-point formula. */
#define IM3D_SWEEP_LEXICOGRAPHIC 0
#define IM3D_SWEEP_REDBLACK 1

/* Parameters of segm::rsfe_splitbregman<T> (rsfe_splitbregman.hxx:99-894).
 * im3d_rsfe_params_default() fills the reference constructor's values
 * (rsfe_splitbregman_imp.hxx:25-41). Field names are the reference's. */
typedef struct im3d_rsfe_params {
    double tol;                 /* outer stop: ||phi-phiold||_L2/||phiold||_L2 <= tol (1e-5) */
    double sigma;               /* Gaussian std-dev of the fitting kernel (3) */
    double lamda;               /* Bregman weight (5e-2) */
    double lamda1;              /* inside fitting weight (1e-5) */
    double lamda2;              /* outside fitting weight (1e-5) */
    double beta;                /* edge detector g = 1/(1+beta|grad u0|^2) (100) */
    double nu;                  /* TV weight (1) */
    double dt;                  /* pseudo time step of the unsteady Poisson step (1) */
    double epsilon;             /* Heaviside width (1e-3) */
    double a0;                  /* lower level-set value (0) */
    double b0;                  /* upper level-set value (1) */
    double ls_tol;              /* relative-change stop of the sweep loop, 0 = off (0) */
    double edge_detector_sigma; /* pre-blur of u0 for the edge detector, 0 = none (0) */
    /* extensions with no reference counterpart */
    double gs_rel_res_tol;      /* >0: each outer iteration solves (1/dt - Lap) u = u_old/dt + rhs
                                   to this relative residual instead of running ls_steps sweeps */
    double omega;               /* over-relaxation factor of the residual solve (1 = Gauss-Seidel) */
    int32_t maxiter;            /* outer iteration cap (100) */
    int32_t ls_steps;           /* sweeps per outer iteration (5) */
    int32_t bc;                 /* IM3D_BC_* (IM3D_BC_DEFAULT) */
    int32_t gaussian_pixel_approach; /* build the Gaussian with unit spacing (0) */
    int32_t init_variables;     /* the first iteration resets b and div(d-b) instead of the
                                   Bregman update: the reference's private flag, which starts
                                   false and which an extraction raises (0) */
    int32_t sweep;              /* IM3D_SWEEP_* used by the ls_steps sweeps (LEXICOGRAPHIC) */
    int32_t gs_max_sweeps;      /* sweep cap of the residual solve (1000) */
    int32_t gs_check_every;     /* residual every this many sweeps; 0 = predicted from the
                                   observed contraction rate (0) */
    /* automatic connected-component extraction inside the loop: the automatic case of
     * extract_connected_component (rsfe_splitbregman_imp.hxx:448-536), run after cut_phi
     * at every outer iteration t with t % auto_extract_conn_comp_freq == 0 (:1809) */
    double cc_init_pixel_x;     /* seed in physical coordinates, cell floor(x / hx) (-1) */
    double cc_init_pixel_y;     /* (-1) */
    double cc_init_pixel_z;     /* (-1) */
    double alpha;               /* level of phi whose inside is white: the black-and-white
                                   threshold is (alpha - a0) / (b0 - a0) ((a0 + b0) / 2) */
    int32_t auto_extract_conn_comp;      /* extraction on (0) */
    int32_t auto_extract_conn_comp_freq; /* every this many outer iterations, 0 = never (0) */
    int32_t cc_binary_output;   /* phi becomes the 0/1 component (1) or keeps its values on
                                   the component and outside the threshold (0) */
    int32_t cc_init_variables;  /* reset b and div(d-b) after an extraction (1) */
    /* the convolution plug-in (set_cv, rsfe_splitbregman_imp.hxx:836-842): 0 =
     * acyclic_fftw_convolution (zero boundary, the constructor's choice), 1 =
     * cyclic_fftw_convolution (periodic boundary) */
    int32_t conv_cyclic;
    int32_t reserved_;
} im3d_rsfe_params;

typedef struct im3d_rsfe_stats {
    double last_tol;      /* ||phi-phiold||_L2/||phiold||_L2 of the last outer iteration */
    double last_rel_res;  /* relative residual at the end of the last solve (residual mode) */
    double last_ls_err;   /* relative change of the last sweep (ls_tol mode) */
    double setup_ms;      /* device time of the set-up (filters, k*1, k*u0, edge detector) */
    double loop_ms;       /* device time of the outer loop */
    int64_t total_sweeps; /* sweeps over all outer iterations */
    int32_t iterations;   /* outer iterations run */
    int32_t last_sweeps;  /* sweeps of the last outer iteration */
    int32_t not_converged;/* outer iterations whose solve hit gs_max_sweeps */
    int32_t residual_checks; /* residual evaluations of the Poisson solves (residual mode) */
    int32_t ws_used;      /* solves started from the learned warm start (IM3D_WS_PREDICT) */
    int32_t ws_rejected;  /* solves where it lost to the previous iterate */
    double ws_loss;       /* mean training loss over the solves (IM3D_WS_TRAIN) */
} im3d_rsfe_stats;

typedef struct im3d_ctx im3d_ctx;

/* Context: one per host thread; owns a stream, device buffers and cached plans. */
int im3d_ctx_create(int device, im3d_ctx** out);
int im3d_ctx_destroy(im3d_ctx* ctx);
const char* im3d_ctx_last_error(const im3d_ctx* ctx);
/* Run subsequent calls on an external cudaStream_t (NULL = the context's own). */
int im3d_ctx_set_stream(im3d_ctx* ctx, void* cuda_stream);
/* Count of kernel launches the context issued since creation (instrumentation). */
int64_t im3d_ctx_launch_count(const im3d_ctx* ctx);

/* Context options (no counterpart in the reference), set with im3d_ctx_set_option:
 *  IM3D_OPT_FIT_CHUNKS           chunks of planes along i of the FP32 fitting stage;
 *                                0 (default) = the cost model's choice. Every choice
 *                                gives bit-identical results.
 *  IM3D_OPT_DEVICE_MEMORY_LIMIT  bytes of device buffers the context may hold; a call
 *                                that would need more returns IM3D_ERR_OOM before it
 *                                allocates (0, the default, = no limit). For callers that
 *                                share the GPU under a memory budget.
 *  IM3D_OPT_BATCH_MODE           how im3d_rsfe_apply_batched_* runs its volumes:
 *                                IM3D_BATCH_AUTO (default) and IM3D_BATCH_STREAMS = the
 *                                stream queue (the faster on B200: each volume's state stays
 *                                in L2 across its stages and sweeps); IM3D_BATCH_WORKLIST =
 *                                the work list, IM3D_ERR_UNSUPPORTED where it cannot run.
 *  IM3D_OPT_TILE_LOADS           1 (default): the FP32 Heaviside pass moves whole rows
 *                                with the Tensor Memory Accelerator where the volume allows
 *                                it (nz a multiple of 8 and at most 256, 16-byte aligned
 *                                buffers, 19 or 25 taps); 0: the register-window kernel
 *                                everywhere. Both give bit-identical results.
 * Returns IM3D_ERR_INVALID_ARG for an unknown option or a negative value. */
#define IM3D_OPT_FIT_CHUNKS 1
#define IM3D_OPT_DEVICE_MEMORY_LIMIT 2
#define IM3D_OPT_BATCH_MODE 3
#define IM3D_BATCH_AUTO 0
#define IM3D_BATCH_STREAMS 1
#define IM3D_BATCH_WORKLIST 2
#define IM3D_OPT_TILE_LOADS 4
int im3d_ctx_set_option(im3d_ctx* ctx, int option, int64_t value);
/* Per-stage device timing: with profiling on, each launch of the loop's kernels is
 * bracketed by CUDA events on the launching stream. im3d_ctx_profile() synchronises,
 * writes up to max_entries stage names ('\n'-separated into names), total ms and
 * launch counts, returns the number of stages (negative status on error) and clears
 * the totals when reset != 0. on == 2 times only each Poisson solve as a whole (stage
 * "poisson_solve", warm start included), with no events between the launches inside it,
 * so that they keep their overlap. No counterpart in the reference (it has no timers). */
int im3d_ctx_set_profiling(im3d_ctx* ctx, int on);
int im3d_ctx_profile(im3d_ctx* ctx, char* names, int names_cap, double* ms, int64_t* counts,
                     int max_entries, int reset);

/* Reference constructor defaults (rsfe_splitbregman_imp.hxx:25-41) plus the
 * extension defaults documented in im3d_rsfe_params. */
void im3d_rsfe_params_default(im3d_rsfe_params* p);

/* Gaussian filtering with zero boundary:
 * conv::filtering<T>::build_gaussian_filter(f, sigma, radius, pixel_approach)
 * (convolution_imp.hxx:22-91) followed by conv::acyclic_fftw_convolution(out, in)
 * (convolution_imp.hxx:535-653). The result is the linear convolution with the
 * normalised kernel, cropped to the input size; computed here as three 1-D passes. */
int im3d_gauss_filter_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny, int nz,
                          double hx, double hy, double hz, double sigma, double radius,
                          int pixel_approach);
int im3d_gauss_filter_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny, int nz,
                          double hx, double hy, double hz, double sigma, double radius,
                          int pixel_approach);

/* The same Gaussian with conv::cyclic_fftw_convolution (convolution_imp.hxx:657-754,
 * filter built by build_freq_filters' cyclic part, :406-528): the volume is taken as
 * periodic (the reference periodises it over a grid of the volume's size, repeated
 * until it covers the kernel), so each axis pass is the circular convolution
 * out[a] = sum_t w[t] in[(a - t) mod n]. */
int im3d_gauss_filter_cyclic_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny,
                                 int nz, double hx, double hy, double hz, double sigma,
                                 double radius, int pixel_approach);
int im3d_gauss_filter_cyclic_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny,
                                 int nz, double hx, double hy, double hz, double sigma,
                                 double radius, int pixel_approach);

/* `sweeps` calls of lapl::DirGaussSeidel (bc_type DIR or DEFAULT) or
 * lapl::NeuGaussSeidel (NEU), in place on res (poisson_imp.hxx:340-429, 23-336):
 * res <- (sum of neighbour terms + b + res/dt) * htilde, boundary per bc_type. */
int im3d_poisson_sweeps_f32(im3d_ctx* ctx, float* res, const float* b, int nx, int ny, int nz,
                            double hx, double hy, double hz, double dt, double bc, int bc_type,
                            int sweep_order, int sweeps);
int im3d_poisson_sweeps_f64(im3d_ctx* ctx, double* res, const double* b, int nx, int ny, int nz,
                            double hx, double hy, double hz, double dt, double bc, int bc_type,
                            int sweep_order, int sweeps);

/* Red-black solve of (1/dt - Lap_h) u = u_in/dt + b (u_in = u on entry, held fixed),
 * boundary per bc_type, until ||residual||_2/||b + u_in/dt||_2 <= rel_res_tol (checked
 * every check_every sweeps) or max_sweeps; returns IM3D_ERR_NOT_CONVERGED at the cap. */
int im3d_poisson_solve_f32(im3d_ctx* ctx, float* u, const float* b, int nx, int ny, int nz,
                           double hx, double hy, double hz, double dt, double bc, int bc_type,
                           double rel_res_tol, int max_sweeps, int check_every, double omega,
                           int* sweeps_done, double* rel_res);
int im3d_poisson_solve_f64(im3d_ctx* ctx, double* u, const double* b, int nx, int ny, int nz,
                           double hx, double hy, double hz, double dt, double bc, int bc_type,
                           double rel_res_tol, int max_sweeps, int check_every, double omega,
                           int* sweeps_done, double* rel_res);

/* Gaussian filter that allocates nothing. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code that runs while a host framework owns
 * all device memory through its own pool (a caching allocator or a fixed arena that a
 * second allocator must not fragment), code inside a hard device-memory budget, and
 * code that must not make the allocation calls that can synchronise the device. The
 * caller passes device buffers `in` and `out` (nx*ny*nz floats each, on the current
 * device; pointers of another device return IM3D_ERR_INVALID_ARG) and a cudaStream_t
 * (NULL = the default stream); every call waits for that stream to finish before it
 * returns. It is im3d_gauss_filter_f32 with its two intermediate volumes and its taps
 * held in one file-scope __device__ array of 2 * 2097152 + 387 floats (16 MiB), which
 * every GPU that loads the library keeps until the process exits. Volumes above
 * 2097152 voxels (128^3) return IM3D_ERR_TOO_LARGE, and nx or ny above 65535 return
 * IM3D_ERR_INVALID_ARG, both without touching the GPU. The first call on a device
 * looks the array's device address up (cudaGetSymbolAddress); make that first call
 * before any stream capture. Later calls may be captured into a CUDA graph: on a
 * capturing stream the call returns without waiting, and the caller waits for the
 * graph's launch; otherwise it returns after the stream has finished the filter. Calls
 * share the array, so calls that overlap on the GPU
 * (other threads or streams) race; every call rewrites all of the scratch it reads,
 * so nothing carries over from the previous call. A launch that fails returns
 * IM3D_ERR_CUDA; an error the caller left pending is neither reported nor cleared. */
int im3d_gauss_filter_f32_noalloc(const float* in, float* out, int nx, int ny, int nz,
                                  double hx, double hy, double hz, double sigma, double radius,
                                  int pixel_approach, void* stream);

/* image3d<T>::grad (image3d_imp.hxx:744-889): out holds 3 volumes, component-major. */
int im3d_grad_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny, int nz,
                  double hx, double hy, double hz);
int im3d_grad_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny, int nz,
                  double hx, double hy, double hz);
/* im3d::div (image3d_imp.hxx:948-1384): in holds 3 volumes, component-major. */
int im3d_div_f32(im3d_ctx* ctx, const float* in, float* out, int nx, int ny, int nz,
                 double hx, double hy, double hz);
int im3d_div_f64(im3d_ctx* ctx, const double* in, double* out, int nx, int ny, int nz,
                 double hx, double hy, double hz);

/* segm::rsfe_splitbregman<T>::apply(myim, init) (rsfe_splitbregman_imp.hxx:1547-1995);
 * init == NULL is apply(myim) with the default cube (:1531-1543, :48-95).
 * phi_out receives getoutput() (segmentation.hxx:108-111). u_out (phi after the last
 * solve, before the clamp), f1_out and f2_out (the last iteration's fitting means,
 * :1709-1717) are optional (NULL = not copied). A myim or init holding NaN or Inf
 * returns IM3D_ERR_NONFINITE before the loop starts. */
int im3d_rsfe_apply_f32(im3d_ctx* ctx, const float* myim, const float* init, int nx, int ny,
                        int nz, double hx, double hy, double hz, const im3d_rsfe_params* p,
                        float* phi_out, float* u_out, float* f1_out, float* f2_out,
                        im3d_rsfe_stats* stats);
int im3d_rsfe_apply_f64(im3d_ctx* ctx, const double* myim, const double* init, int nx, int ny,
                        int nz, double hx, double hy, double hz, const im3d_rsfe_params* p,
                        double* phi_out, double* u_out, double* f1_out, double* f2_out,
                        im3d_rsfe_stats* stats);

/* State of the loop after outer iteration t: what rsfe_splitbregman<T> holds between
 * iterations (phi, the Bregman variable b and div(d - b)), plus this backend's
 * residual-schedule state, so that a run resumed from it continues exactly as the
 * uninterrupted run would. Arrays are T (float for _f32, double for _f64) in the
 * image3d layout; b holds 3 volumes, component-major. */
typedef struct im3d_rsfe_checkpoint {
    int32_t t;               /* outer iterations completed */
    int32_t init_variables;  /* the next iteration resets b and div(d-b) (after an extraction) */
    int32_t sched_first;     /* sweeps before the first residual check of the next solve */
    int32_t reserved;
    double sched_rate;       /* contraction rate carried to the next solve */
    double tollerance;       /* ||phi - phiold||_L2 / ||phiold||_L2 of iteration t */
    void* phi;               /* n values */
    void* b;                 /* 3n values (NULL when the observer did not ask for the state) */
    void* divdb;             /* n values (NULL likewise) */
} im3d_rsfe_checkpoint;

/* Per-iteration observer of im3d_rsfe_apply_*: the dumps of the reference's loop
 * (dumpfrequency, rsfe_splitbregman_imp.hxx:1940-1951, which writes phi every
 * dumpfrequency-th iteration except the last) and full-state checkpoints. After
 * outer iteration t, when every > 0, t % every == 0 and t != maxiter, the loop copies
 * phi (and with with_state != 0 also b and div(d-b)) to host memory owned by the
 * context and calls cb(user, &checkpoint); the pointers are valid during the call
 * only. A non-zero return ends the loop after that iteration, as the reference's
 * end_now does (:1659). cb == NULL removes the observer. The other iterations copy
 * nothing. No counterpart as a function in the reference. */
typedef int (*im3d_rsfe_observer)(void* user, const im3d_rsfe_checkpoint* state);
int im3d_ctx_set_observer(im3d_ctx* ctx, int every, int with_state, im3d_rsfe_observer cb,
                          void* user);

/* Resume: the next im3d_rsfe_apply_* call on this context starts from `from` instead
 * of the initial level set (its init argument is then ignored), at outer iteration
 * from->t + 1, with the set-up (filters, edge detector) recomputed from myim. phi, b
 * and divdb must be set (host or device memory holding values of element_size bytes:
 * 4 for the _f32 call, 8 for _f64) and stay valid until that call returns; the
 * struct itself is copied here. The result equals the uninterrupted run's bit for bit.
 * from == NULL cancels a pending resume. The reference can only restart from phi
 * (apply(myim, init) rescales init and zeroes b, :99-170, :1606-1629). */
int im3d_ctx_set_resume(im3d_ctx* ctx, const im3d_rsfe_checkpoint* from, int element_size);

/* ---- Learned warm start of the Poisson step (no counterpart in the reference) ----
 * A 3-level 3-D U-Net (16/32/64 channels, 3x3x3 convolutions, ReLU, 2x2x2 max pooling
 * and transposed convolutions, a 1x1 output layer) maps four fields of an outer
 * iteration -- the forcing term rhs, the previous solve's u, div(d - b) and phi -- to a
 * correction of phi that starts the Gauss-Seidel solve of
 * rsfe_splitbregman_imp.hxx:1768-1785 (poisson_imp.hxx:340-429). Activations are BF16
 * (channels last), filters BF16 with FP32 master copies, accumulation FP32 on the
 * tensor cores (tcgen05). The solve still runs to the requested residual after it. */
typedef struct im3d_unet im3d_unet;

/* A network with He-normal weights from `seed` (the output layer starts at zero, so an
 * untrained network predicts no correction), on the context's device. */
int im3d_unet_create(im3d_ctx* ctx, uint64_t seed, im3d_unet** out);
int im3d_unet_destroy(im3d_unet* net);
/* Parameters as FP32, in this order per 3x3x3 layer (e1a, e1b, e2a, e2b, e3a, e3b,
 * d2a, d2b, d1a, d1b): W[cout][cin][27] (tap = 9 dz + 3 dy + dx over the (i, j, k)
 * offsets -1..1), bias[cout]; then the transposed convolutions up2 (64 -> 32) and up1
 * (32 -> 16): U[8][cin][cout] (child o = 4 di + 2 dj + dk), bias[cout]; then the 1x1
 * output layer: w[16], bias[1]. */
int64_t im3d_unet_param_count(const im3d_unet* net);
int im3d_unet_get_params(im3d_ctx* ctx, im3d_unet* net, float* host, int64_t count);
int im3d_unet_set_params(im3d_ctx* ctx, im3d_unet* net, const float* host, int64_t count);
/* Forward pass of nsamp samples: x holds nsamp x 4 FP32 volumes [s][field][nx][ny][nz]
 * (host or device), y receives nsamp FP32 volumes. nx, ny: multiples of 4; nz, nz/2,
 * nz/4 multiples of 16 that are at most 128 or multiples of 128. */
int im3d_unet_forward(im3d_ctx* ctx, im3d_unet* net, const float* x, int nsamp, int nx, int ny, int nz,
                      float* y);
/* One training step on (x, target): forward, mean squared error, backward (BF16
 * tensor-core data and weight gradients), Adam with learning rate lr (lr = 0: no
 * update). *loss (may be NULL) receives the loss of the forward pass, grads (host, may
 * be NULL) the FP32 gradient of every parameter in the order above. */
int im3d_unet_train_step(im3d_ctx* ctx, im3d_unet* net, const float* x, const float* target, int nsamp, int nx,
                         int ny, int nz, double lr, double* loss, float* grads);
/* One 3x3x3 convolution (zero padding, stride 1) on the tensor cores, as the network's
 * layers run it: x BF16 channels-last (c_pitch channels per voxel, the cin used ones
 * from c_off), w FP32 [cout][cin][27], bias FP32 [cout] or NULL, out FP32 channels-last
 * [voxel][cout]; cin, cout in {16, 32, 64}; all pointers device memory. */
int im3d_conv3d_bf16(im3d_ctx* ctx, const uint16_t* x, int c_pitch, int c_off, int cin, const float* w,
                     const float* bias, int cout, int nsamp, int nx, int ny, int nz, float* out);

/* The warm start inside im3d_rsfe_apply_f32 when gs_rel_res_tol > 0:
 *  IM3D_WS_PREDICT  before each solve the network's correction is added to phi; the
 *                   solve starts from it when its residual is below the previous
 *                   iterate's, and from the previous iterate otherwise;
 *  IM3D_WS_TRAIN    after each solve the network takes one training step (learning
 *                   rate lr) on that solve's fields and its solution (the pairs the
 *                   plain solver generates); the solve itself is the plain one.
 * net == NULL or mode IM3D_WS_OFF removes it. The network must stay alive while set. */
#define IM3D_WS_OFF 0
#define IM3D_WS_PREDICT 1
#define IM3D_WS_TRAIN 2
int im3d_ctx_set_warm_start(im3d_ctx* ctx, im3d_unet* net, int mode, double lr);

/* Connected component of the thresholded image, as
 * image3d<T>::connected_component (image3d_imp.hxx:1694-2120):
 *  - init == NULL: the component containing cell (i, j, k) (:1694-1758). The seed is
 *    moved off the faces (to 1..dim-2; k = 0 when nz == 1); if the image is below
 *    the pivot there, the component is taken in the negative black-and-white image.
 *  - init != NULL: the cells connected to the cells where init != 0 and the image is
 *    at or above the pivot (:1761-1798); i, j, k are ignored.
 * The black-and-white image is 1 where img >= pivot = min + (max - min) * threshold
 * (im_to_black_and_white, :1592-1623; a threshold outside [0, 1] becomes 0.5, as in
 * the reference, and the WARNING is left in im3d_ctx_last_error with status OK).
 * Only cells off the faces spread the component (to their 6 face neighbours, 26 with
 * full_connected; 4 / 8 in 2-D). res receives 1 on the component and 0 elsewhere,
 * or, with binary_output == 0, cc_not_binary_output (:1801-1817):
 * (res + negative b&w) * (img - min) + min. img, init and res are device or host
 * buffers in the image3d layout; nx, ny >= 2 and nz >= 1. `passes` (may be NULL)
 * receives the number of whole-volume propagation passes run. */
int im3d_connected_component_f32(im3d_ctx* ctx, const float* img, float* res, int nx, int ny,
                                 int nz, const float* init, int i, int j, int k, double threshold,
                                 int full_connected, int binary_output, int* passes);
int im3d_connected_component_f64(im3d_ctx* ctx, const double* img, double* res, int nx, int ny,
                                 int nz, const double* init, int i, int j, int k, double threshold,
                                 int full_connected, int binary_output, int* passes);

/* A batch of independent volumes of uneven sizes. No counterpart
 * in the reference, which segments one image per apply(). Each descriptor holds the
 * caller's buffers (host or device, T = float for _f32, double for _f64), the size
 * and the spacing. */
typedef struct im3d_volume_desc {
    const void* myim;   /* image to segment */
    const void* init;   /* initial level set, NULL = the default cube */
    void* phi_out;      /* receives getoutput() */
    int32_t nx, ny, nz, reserved;
    double hx, hy, hz;
} im3d_volume_desc;

/* Segments nvol volumes with the same parameters, in one of two ways
 * (IM3D_OPT_BATCH_MODE; the stream queue by default):
 *  - the work list: groups of up to 64 volumes, largest first, advance their outer
 *    iterations together; each convolution, clamp, Bregman and div stage is ONE
 *    launch over the blocks of every volume of the group, and the Poisson solves run
 *    in L2-sized subgroups of volumes (one launch per half-sweep and per residual
 *    check of a subgroup) on `streams` concurrent worker streams (0 = 4). Runs when
 *    the Poisson step is solved to a residual (gs_rel_res_tol > 0, omega 1), the
 *    Gaussian has 19 or 25 taps on every axis of every volume and no
 *    connected-component extraction is asked for.
 *  - the stream queue: volumes are taken largest first from a shared queue by
 *    `streams` workers (0 = 4), each running whole segmentations on its own CUDA
 *    stream with its own device buffers, so small volumes overlap on the GPU.
 * Both give every volume the result of its own im3d_rsfe_apply_* call, bit for bit.
 * stats and latency_ms (either may be NULL) receive nvol entries: the statistics of
 * each volume and the time from the start of the call to that volume's result.
 * Returns the first non-OK status. */
int im3d_rsfe_apply_batched_f32(im3d_ctx* ctx, int nvol, const im3d_volume_desc* vols,
                                const im3d_rsfe_params* p, int streams, im3d_rsfe_stats* stats,
                                double* latency_ms);
int im3d_rsfe_apply_batched_f64(im3d_ctx* ctx, int nvol, const im3d_volume_desc* vols,
                                const im3d_rsfe_params* p, int streams, im3d_rsfe_stats* stats,
                                double* latency_ms);

#ifdef __cplusplus
}
#endif

#endif /* IM3D_B200_H */

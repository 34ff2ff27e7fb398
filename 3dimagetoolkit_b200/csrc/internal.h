// internal.h -- what the translation units of libim3d_b200.so share beyond the C ABI:
// the context's stream, device and error text for the learned warm start (unet.cu),
// and the network entry points the segmentation loop (im3d_b200.cu) calls.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/im3d_b200.h"

cudaStream_t im3d_ctx_stream(im3d_ctx* ctx);
int im3d_ctx_device(im3d_ctx* ctx);
std::string& im3d_ctx_error_ref(im3d_ctx* ctx);

namespace im3d {
namespace unet {

// Forward pass of nsamp samples of 4 FP32 fields ([s][f][D][H][W], device) into y
// ([s][D][H][W], FP32, device), on stream st.
int net_forward_fields(im3d_unet* n, cudaStream_t st, const float* x, int nsamp, int D, int H, int W, float* y,
                       std::string& err);
// One training step (forward, mean squared error against target -- weighted by wt when
// not NULL --, backward, Adam with learning rate lr when lr > 0); *loss receives the
// loss, grads_host (may be NULL) the parameter gradients.
int net_train_fields(im3d_unet* n, cudaStream_t st, const float* x, const float* target, const float* wt, int nsamp,
                     int D, int H, int W, double lr, double* loss, float* grads_host, std::string& err);
int net_device(const im3d_unet* n);
// kernels the network code has launched in this process (instrumentation)
long long launch_total();

}  // namespace unet
}  // namespace im3d

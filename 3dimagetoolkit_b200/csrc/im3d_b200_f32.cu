// im3d_b200_f32.cu -- the FP32 entry points of im3d_b200.cu, compiled in their own
// translation unit without -fmad=false: the FP32 kernels may contract multiply-adds,
// while the FP64 path (unit 1) keeps the reference's operations.
#define IM3D_UNIT 2
#include "im3d_b200.cu"

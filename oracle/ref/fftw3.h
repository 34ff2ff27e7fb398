/*
 * fftw3.h -- the subset of the FFTW3 API that the reference headers call
 * (convolution_imp.hxx:222-233, 280-282, 386-402, 535-653, 657-757), declared here
 * so that the reference's own convolution code compiles without FFTW.
 *
 * TEST INFRASTRUCTURE ONLY: this header and fft_shim.cpp exist to build the
 * reference (oracle/_ref) as a CPU checker. Nothing in the product links them.
 *
 * FFTW3 itself is absent from this machine and from the reference tree (the
 * reference finds it with CMake's find_library, no version pinned). The transform
 * implemented behind these names is the unnormalised DFT that FFTW documents:
 *   out[k] = sum_j in[j] * exp(sign * 2*pi*i * j*k / n), sign = FFTW_FORWARD (-1)
 * or FFTW_BACKWARD (+1), applied along each axis of a row-major n0 x n1 x n2 array.
 */
#ifndef IM3D_ORACLE_FFTW3_SHIM_H
#define IM3D_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct im3d_fft_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);

#ifdef __cplusplus
}
#endif

#endif

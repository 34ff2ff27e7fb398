/*
 * im3d_oracle.h -- CPU restatement (FP64) of 3dimagetoolkit's RSFE Split-Bregman
 * segmentation path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU results are compared with.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * The product (3dimagetoolkit_b200/) never links or calls anything here.
 *
 * Every function states the reference file:line it restates. Volumes use the
 * reference's image3d layout: (i, j, k) at (i*ny + j)*nz + k, k contiguous.
 * The parameter and statistics structs are the ones the product's C ABI uses.
 */
#ifndef IM3D_ORACLE_H
#define IM3D_ORACLE_H

#include <stddef.h>

#include "../include/im3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Normalised 1-D Gaussian taps of conv::filtering<T>::build_gaussian_filter. */
int orc_gauss_taps(double sigma, double radius, double h, double* taps, int cap);
void orc_gauss_filter(const double* in, double* out, int nx, int ny, int nz, double hx,
                      double hy, double hz, double sigma, double radius, int pixel_approach);
void orc_gauss_filter_cyclic(const double* in, double* out, int nx, int ny, int nz, double hx,
                             double hy, double hz, double sigma, double radius,
                             int pixel_approach);
void orc_gauss_filter_mode(const double* in, double* out, int nx, int ny, int nz, double hx,
                           double hy, double hz, double sigma, double radius,
                           int pixel_approach, int cyclic);
void orc_grad(const double* in, double* out3, int nx, int ny, int nz, double hx, double hy,
              double hz);
void orc_div(const double* in3, double* out, int nx, int ny, int nz, double hx, double hy,
             double hz);
void orc_poisson_sweeps(double* res, const double* b, int nx, int ny, int nz, double hx,
                        double hy, double hz, double dt, double bc, int bc_type, int order,
                        int sweeps);
int orc_poisson_solve(double* u, const double* b, int nx, int ny, int nz, double hx, double hy,
                      double hz, double dt, double bc, int bc_type, double rel_res_tol,
                      int max_sweeps, int check_every, double omega, int* sweeps_done,
                      double* rel_res);
double orc_im_to_bw(const double* img, size_t n, double threshold, int negative,
                    unsigned char* bw);
void orc_cc_grow(unsigned char* res, const unsigned char* bw, int nx, int ny, int nz, int full);
int orc_connected_component(const double* img, double* res, int nx, int ny, int nz,
                            const double* init, int i, int j, int k, double threshold,
                            int full_connected, int binary_output);
int orc_poisson_solve_sched(double* u, const double* b, int nx, int ny, int nz, double hx,
                            double hy, double hz, double dt, double bc, int bc_type,
                            double rel_res_tol, int max_sweeps, int check_every, double omega,
                            int first_check, double rate_hint, int* sweeps_done,
                            double* rel_res, double* rate_out, int* checks);
int orc_rsfe_apply(const double* myim, const double* init, int nx, int ny, int nz, double hx,
                   double hy, double hz, const im3d_rsfe_params* p, double* phi_out,
                   double* u_out, double* f1_out, double* f2_out, im3d_rsfe_stats* stats);

#ifdef __cplusplus
}
#endif

#endif

/*
 * b200.hxx -- glue between the header-only C++ API (im3d/, conv/, lapl/, segm/) and
 * the C ABI of the B200 backend (im3d_b200.h, libim3d_b200.so).
 *
 * One process-wide backend context per host thread is created on first use on the
 * device named by the IM3D_DEVICE environment variable (default 0). Only T = float and
 * T = double reach the GPU; other element types fail to compile where a GPU routine
 * is called.
 */
#ifndef IM3D_B200_HXX
#define IM3D_B200_HXX

#include <cstdlib>
#include <iostream>
#include <string>

#include "../im3d_b200.h"

namespace im3d
{
namespace b200
{

/* The calling thread's backend context (NULL when no usable device exists). */
inline im3d_ctx* context ()
{
    thread_local struct Holder
    {
        im3d_ctx* ctx = nullptr;
        bool tried = false;
        ~Holder()
        {
            if (ctx) im3d_ctx_destroy (ctx);
        }
    } h;
    if (!h.tried)
    {
        h.tried = true;
        const char* env = std::getenv ("IM3D_DEVICE");
        const int dev = env ? std::atoi (env) : 0;
        if (im3d_ctx_create (dev, &h.ctx) != IM3D_OK) h.ctx = nullptr;
    }
    return h.ctx;
}

/* Prints the reference-style WARNING for a failed backend call; true when it failed. */
inline bool failed (int status, char const* where)
{
    if (status == IM3D_OK) return false;
    im3d_ctx* c = context();
    std::clog << "WARNING::" << where << ": "
              << (c ? im3d_ctx_last_error (c) : "no usable B200 device") << std::endl;
    return true;
}

template <typename T>
struct ops;

template <>
struct ops<float>
{
    static int gauss (im3d_ctx* c, float const* in, float* out, int x, int y, int z, double hx,
                      double hy, double hz, double s, double r, int gpa, int cyc = 0)
    {
        return cyc ? im3d_gauss_filter_cyclic_f32 (c, in, out, x, y, z, hx, hy, hz, s, r, gpa)
                   : im3d_gauss_filter_f32 (c, in, out, x, y, z, hx, hy, hz, s, r, gpa);
    }
    static int sweeps (im3d_ctx* c, float* res, float const* b, int x, int y, int z, double hx,
                       double hy, double hz, double dt, double bc, int bct, int order, int n)
    {
        return im3d_poisson_sweeps_f32 (c, res, b, x, y, z, hx, hy, hz, dt, bc, bct, order, n);
    }
    static int grad (im3d_ctx* c, float const* in, float* out, int x, int y, int z, double hx,
                     double hy, double hz)
    {
        return im3d_grad_f32 (c, in, out, x, y, z, hx, hy, hz);
    }
    static int div (im3d_ctx* c, float const* in, float* out, int x, int y, int z, double hx,
                    double hy, double hz)
    {
        return im3d_div_f32 (c, in, out, x, y, z, hx, hy, hz);
    }
    static int apply (im3d_ctx* c, float const* u0, float const* init, int x, int y, int z,
                      double hx, double hy, double hz, im3d_rsfe_params const* p, float* phi,
                      im3d_rsfe_stats* st)
    {
        return im3d_rsfe_apply_f32 (c, u0, init, x, y, z, hx, hy, hz, p, phi, nullptr, nullptr,
                                    nullptr, st);
    }
    static int cc (im3d_ctx* c, float const* img, float* res, int x, int y, int z,
                   float const* init, int i, int j, int k, double thr, int full, int bin)
    {
        return im3d_connected_component_f32 (c, img, res, x, y, z, init, i, j, k, thr, full, bin,
                                             nullptr);
    }
};

template <>
struct ops<double>
{
    static int gauss (im3d_ctx* c, double const* in, double* out, int x, int y, int z,
                      double hx, double hy, double hz, double s, double r, int gpa, int cyc = 0)
    {
        return cyc ? im3d_gauss_filter_cyclic_f64 (c, in, out, x, y, z, hx, hy, hz, s, r, gpa)
                   : im3d_gauss_filter_f64 (c, in, out, x, y, z, hx, hy, hz, s, r, gpa);
    }
    static int sweeps (im3d_ctx* c, double* res, double const* b, int x, int y, int z,
                       double hx, double hy, double hz, double dt, double bc, int bct, int order,
                       int n)
    {
        return im3d_poisson_sweeps_f64 (c, res, b, x, y, z, hx, hy, hz, dt, bc, bct, order, n);
    }
    static int grad (im3d_ctx* c, double const* in, double* out, int x, int y, int z, double hx,
                     double hy, double hz)
    {
        return im3d_grad_f64 (c, in, out, x, y, z, hx, hy, hz);
    }
    static int div (im3d_ctx* c, double const* in, double* out, int x, int y, int z, double hx,
                    double hy, double hz)
    {
        return im3d_div_f64 (c, in, out, x, y, z, hx, hy, hz);
    }
    static int apply (im3d_ctx* c, double const* u0, double const* init, int x, int y, int z,
                      double hx, double hy, double hz, im3d_rsfe_params const* p, double* phi,
                      im3d_rsfe_stats* st)
    {
        return im3d_rsfe_apply_f64 (c, u0, init, x, y, z, hx, hy, hz, p, phi, nullptr, nullptr,
                                    nullptr, st);
    }
    static int cc (im3d_ctx* c, double const* img, double* res, int x, int y, int z,
                   double const* init, int i, int j, int k, double thr, int full, int bin)
    {
        return im3d_connected_component_f64 (c, img, res, x, y, z, init, i, j, k, thr, full, bin,
                                             nullptr);
    }
};

} // namespace b200
} // namespace im3d

#endif

/*
 * ref_capi.cpp -- C entry points over the reference's OWN headers (compiled from
 * the reference tree by oracle/Makefile, with the headless interface, GetPot and
 * FFTW shims in this directory). TEST INFRASTRUCTURE ONLY: it pins the C
 * restatement (im3d_oracle.c) and serves as the timed CPU baseline.
 *
 * Nothing here re-implements the algorithm: each entry point instantiates the
 * reference's templates and calls them. Two public plug-in points of the reference
 * are used to observe or swap the Poisson step, exactly as a user could:
 *   - rsfe_splitbregman<T>::set_cv (rsfe_splitbregman_imp.hxx:836-842) installs a
 *     wrapper around conv::acyclic_fftw_convolution that keeps k*1, k*u0 and the
 *     last iteration's num = k*(H u0) and den = k*H, from which f1 and f2 are formed
 *     with the reference's own expressions (rsfe_splitbregman_imp.hxx:1709-1717);
 *   - rsfe_splitbregman<T>::set_onestep_poisson (:845-852) installs a wrapper that
 *     calls lapl::DirGaussSeidel / lapl::NeuGaussSeidel (or, for the red-black and
 *     residual modes, the restated sweeps of im3d_oracle.c) and keeps the result of
 *     the last call, which is u (phi after the solve, before cut_phi).
 */
#include "rsfe_splitbregman.hxx"

#include "../im3d_oracle.h"

#include <chrono>
#include <cstring>
#include <vector>

// fft_shim.cpp: wall seconds spent in fftw_execute and its call count
extern "C" void im3d_fft_shim_totals(double* seconds, long long* calls);

namespace {

typedef im3d::image3d<double> img;

void to_img(img& dst, const double* src, int nx, int ny, int nz, double hx, double hy,
            double hz)
{
    dst.setdim (nx, ny, nz);
    dst.seth (hx, hy, hz);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                dst (i, j, k) = src[ ( (size_t) i * ny + j) * nz + k];
}

void from_img(double* dst, img const& src)
{
    const int nx = src.getdimx(), ny = src.getdimy(), nz = src.getdimz();
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                dst[ ( (size_t) i * ny + j) * nz + k] = src (i, j, k);
}

struct Recorder
{
    int conv_calls = 0;
    int setup_convs = 2;  // k*1 and k*u0; a third when edge_detector_sigma != 0
    img kones, kmyim, num, den, u;
    // Poisson plug-in selection
    int mode = 0;     // 0 reference Dir, 1 reference Neu, 2 red-black sweep, 3 residual solve
    int bc_type = IM3D_BC_DIR;
    double rel_res_tol = 0, omega = 1;
    int max_sweeps = 1000, check_every = 0;
    int sched_first = 0;
    double sched_rate = 0;
    int checks = 0;
    long long sweeps = 0;
    int last_sweeps = 0;
    double last_rel = -1;
    int not_converged = 0;
    std::vector<double> stamps;  // wall clock (s) at the end of each Poisson step
    std::vector<double> marks;   // sweeps run up to the end of each Poisson step
    std::vector<double> solve_s; // wall seconds inside each Poisson step
    std::vector<double> fft_s;   // FFT wall seconds (fft_shim.cpp) up to the end of each step
};

Recorder g_rec;
std::vector<double> g_last_stamps, g_last_marks, g_last_solve, g_last_fft;
double g_apply_start = 0, g_apply_end = 0;

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// set_bc takes the class's private enum bc_type by value; the enum is deduced from
// the public member's signature instead of being named.
template <typename E>
void call_with_enum (segm::rsfe_splitbregman<double>& a,
                     void (segm::rsfe_splitbregman<double>::*f) (E const), int v)
{
    (a.*f) (static_cast<E> (v) );
}

void record_conv (img const& result);

void rec_conv (img& result, img const& factor)
{
    conv::acyclic_fftw_convolution (result, factor);
    record_conv (result);
}

void rec_conv_cyclic (img& result, img const& factor)
{
    conv::cyclic_fftw_convolution (result, factor);
    record_conv (result);
}

void record_conv (img const& result)
{
    const int c = g_rec.conv_calls++;
    if (c == 0) g_rec.kones = result;
    else if (c == 1) g_rec.kmyim = result;
    else if (c >= g_rec.setup_convs)
    {
        const int r = (c - g_rec.setup_convs) % 4;
        if (r == 0) g_rec.num = result;
        else if (r == 1) g_rec.den = result;
    }
}

void rec_poisson (img& res, img const& b, double const& dt, double const& bc, img const& input)
{
    const double t_enter = now_s();
    const int nx = res.getdimx(), ny = res.getdimy(), nz = res.getdimz();
    if (g_rec.mode == 0)
    {
        lapl::DirGaussSeidel (res, b, dt, bc, input);
        g_rec.sweeps++;
    }
    else if (g_rec.mode == 1)
    {
        lapl::NeuGaussSeidel (res, b, dt, bc, input);
        g_rec.sweeps++;
    }
    else
    {
        std::vector<double> r ( (size_t) nx * ny * nz), bb ( (size_t) nx * ny * nz);
        from_img (r.data(), res);
        from_img (bb.data(), b);
        if (g_rec.mode == 2)
        {
            orc_poisson_sweeps (r.data(), bb.data(), nx, ny, nz, res.gethx(), res.gethy(),
                                res.gethz(), dt, bc, g_rec.bc_type, IM3D_SWEEP_REDBLACK, 1);
            g_rec.sweeps++;
        }
        else
        {
            int sw = 0;
            double rel = -1, rate = 0;
            // the residual schedule carries over from the previous solve of this apply
            int st = orc_poisson_solve_sched (r.data(), bb.data(), nx, ny, nz, res.gethx(),
                                              res.gethy(), res.gethz(), dt, bc, g_rec.bc_type,
                                              g_rec.rel_res_tol, g_rec.max_sweeps,
                                              g_rec.check_every, g_rec.omega, g_rec.sched_first,
                                              g_rec.sched_rate, &sw, &rel, &rate, &g_rec.checks);
            g_rec.sched_first = st == IM3D_OK ? sw : 0;
            g_rec.sched_rate = st == IM3D_OK ? rate : 0;
            if (st != IM3D_OK) g_rec.not_converged++;
            g_rec.sweeps += sw;
            g_rec.last_sweeps = sw;
            g_rec.last_rel = rel;
        }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k)
                    res (i, j, k) = r[ ( (size_t) i * ny + j) * nz + k];
    }
    g_rec.u = res;
    g_rec.stamps.push_back(now_s() );
    g_rec.marks.push_back( (double) g_rec.sweeps);
    g_rec.solve_s.push_back(g_rec.stamps.back() - t_enter);
    double fft_seconds = 0;
    im3d_fft_shim_totals(&fft_seconds, nullptr);
    g_rec.fft_s.push_back(fft_seconds);
}

}  // namespace

extern "C" {

/* conv::filtering<double>::build_gaussian_filter + acyclic_fftw_convolution */
int ref_gauss_filter (const double* in, double* out, int nx, int ny, int nz, double hx,
                      double hy, double hz, double sigma, double radius, int pixel_approach)
{
    img f, r;
    to_img (f, in, nx, ny, nz, hx, hy, hz);
    conv::filtering<double>::build_gaussian_filter (f, sigma, radius, pixel_approach != 0);
    conv::acyclic_fftw_convolution (r, f);
    from_img (out, r);
    return 0;
}

/* conv::filtering<double>::build_gaussian_filter + cyclic_fftw_convolution */
int ref_gauss_filter_cyclic (const double* in, double* out, int nx, int ny, int nz, double hx,
                             double hy, double hz, double sigma, double radius,
                             int pixel_approach)
{
    img f, r;
    to_img (f, in, nx, ny, nz, hx, hy, hz);
    conv::filtering<double>::build_gaussian_filter (f, sigma, radius, pixel_approach != 0);
    conv::cyclic_fftw_convolution (r, f);
    from_img (out, r);
    return 0;
}

/* conv::filtering<double>::build_gaussian_filter + direct_convolution */
int ref_gauss_filter_direct (const double* in, double* out, int nx, int ny, int nz, double hx,
                             double hy, double hz, double sigma, double radius,
                             int pixel_approach)
{
    img f, r;
    to_img (f, in, nx, ny, nz, hx, hy, hz);
    conv::filtering<double>::build_gaussian_filter (f, sigma, radius, pixel_approach != 0);
    conv::direct_convolution (r, f);
    from_img (out, r);
    return 0;
}

/* image3d<double>::connected_component: the seeded overload (image3d_imp.hxx:1694-1758)
 * when init == NULL, else the overload taking an initial image (:1761-1798) */
int ref_connected_component (const double* in, double* out, int nx, int ny, int nz,
                             const double* init, int i, int j, int k, double threshold,
                             int full_connected, int binary_output)
{
    img f, r;
    to_img (f, in, nx, ny, nz, 1., 1., 1.);
    if (init)
    {
        img s;
        to_img (s, init, nx, ny, nz, 1., 1., 1.);
        f.connected_component (r, s, threshold, full_connected != 0, binary_output != 0);
    }
    else
    {
        f.connected_component (r, (uint) i, (uint) j, (uint) k, threshold, full_connected != 0,
                               binary_output != 0);
    }
    from_img (out, r);
    return 0;
}

/* the FFTW shim itself, for checking it against numpy.fft */
int ref_fft3d (const double* in_interleaved, double* out_interleaved, int n0, int n1, int n2,
               int sign)
{
    size_t n = (size_t) n0 * n1 * n2;
    fftw_complex* in = (fftw_complex*) fftw_malloc (sizeof (fftw_complex) * n);
    fftw_complex* out = (fftw_complex*) fftw_malloc (sizeof (fftw_complex) * n);
    std::memcpy (in, in_interleaved, sizeof (fftw_complex) * n);
    fftw_plan p = fftw_plan_dft_3d (n0, n1, n2, in, out, sign, FFTW_ESTIMATE);
    fftw_execute (p);
    fftw_destroy_plan (p);
    std::memcpy (out_interleaved, out, sizeof (fftw_complex) * n);
    fftw_free (in);
    fftw_free (out);
    return 0;
}

/* image3d<double>::grad; out is component-major (3 volumes) */
int ref_grad (const double* in, double* out3, int nx, int ny, int nz, double hx, double hy,
              double hz)
{
    img f;
    to_img (f, in, nx, ny, nz, hx, hy, hz);
    std::vector<img> g;
    f.grad (g);
    size_t n = (size_t) nx * ny * nz;
    for (int c = 0; c < 3; ++c) from_img (out3 + c * n, g[c]);
    return 0;
}

/* im3d::div of 3 component-major volumes */
int ref_div (const double* in3, double* out, int nx, int ny, int nz, double hx, double hy,
             double hz)
{
    size_t n = (size_t) nx * ny * nz;
    std::vector<img> f (3);
    for (int c = 0; c < 3; ++c) to_img (f[c], in3 + c * n, nx, ny, nz, hx, hy, hz);
    img r;
    im3d::div (r, f);
    from_img (out, r);
    return 0;
}

/* `sweeps` calls of lapl::DirGaussSeidel (neu == 0) or lapl::NeuGaussSeidel */
int ref_gs (double* res, const double* b, int nx, int ny, int nz, double hx, double hy,
            double hz, double dt, double bc, int neu, int sweeps)
{
    img r, bb;
    to_img (r, res, nx, ny, nz, hx, hy, hz);
    to_img (bb, b, nx, ny, nz, hx, hy, hz);
    for (int s = 0; s < sweeps; ++s)
    {
        if (neu) lapl::NeuGaussSeidel (r, bb, dt, bc);
        else lapl::DirGaussSeidel (r, bb, dt, bc);
    }
    from_img (res, r);
    return 0;
}

/* image3d<double>::change_range_of_intensity(max, min) */
int ref_change_range (double* data, int nx, int ny, int nz, double mx, double mn)
{
    img f;
    to_img (f, data, nx, ny, nz, 1, 1, 1);
    f.change_range_of_intensity (mx, mn);
    from_img (data, f);
    return 0;
}

/* segm::rsfe_splitbregman<double>::apply with the parameters of p set through the
 * reference's own setters. init == NULL runs apply(myim) (cube initial contour). */
int ref_rsfe_apply (const double* myim, const double* init, int nx, int ny, int nz, double hx,
                    double hy, double hz, const im3d_rsfe_params* p, double* phi_out,
                    double* u_out, double* f1_out, double* f2_out, im3d_rsfe_stats* stats,
                    int verbosity)
{
    img u0, phi0;
    to_img (u0, myim, nx, ny, nz, hx, hy, hz);
    if (init) to_img (phi0, init, nx, ny, nz, hx, hy, hz);

    g_rec = Recorder();
    g_rec.setup_convs = p->edge_detector_sigma != 0 ? 3 : 2;

    segm::rsfe_splitbregman<double> algo;
    algo.set_verbosity (verbosity != 0);
    algo.set_getpotfile ("");
    algo.set_onthego (false);
    algo.set_maxiter (p->maxiter);
    algo.set_tol (p->tol);
    algo.set_sigma (p->sigma);
    algo.set_lamda (p->lamda);
    algo.set_lamda1 (p->lamda1);
    algo.set_lamda2 (p->lamda2);
    algo.set_beta (p->beta);
    algo.set_nu (p->nu);
    algo.set_dt (p->dt);
    algo.set_epsilon (p->epsilon);
    algo.set_b0 (p->b0);
    algo.set_a0 (p->a0);
    // in the residual mode the plug-in is the whole solve of an outer iteration, so the
    // reference's sweep loop (:1771-1785) must call it exactly once
    const bool solve_mode = p->gs_rel_res_tol > 0;
    algo.set_ls_steps (solve_mode ? 1 : p->ls_steps);
    algo.set_ls_tol (solve_mode ? 0 : p->ls_tol);
    algo.set_edge_detector_sigma (p->edge_detector_sigma);
    algo.set_gaussian_pixel_approach (p->gaussian_pixel_approach != 0);
    // automatic connected-component extraction (public setters, :903-1022, 1380-1415)
    algo.set_alpha (p->alpha);
    algo.set_auto_extract_conn_comp (p->auto_extract_conn_comp != 0);
    algo.set_auto_extract_conn_comp_freq ( (uint) p->auto_extract_conn_comp_freq);
    if (p->cc_init_pixel_x >= 0) algo.set_cc_init_pixel_x (p->cc_init_pixel_x);
    if (p->cc_init_pixel_y >= 0) algo.set_cc_init_pixel_y (p->cc_init_pixel_y);
    if (p->cc_init_pixel_z >= 0) algo.set_cc_init_pixel_z (p->cc_init_pixel_z);
    algo.set_cc_binary_output (p->cc_binary_output != 0);
    algo.set_cc_init_variables (p->cc_init_variables != 0);
    // bc_type is private to the class (rsfe_splitbregman.hxx:108); its values are
    // NEU = 1, DIR = 2, and set_bc takes it by value, so the call goes through
    // the parameter's own type.
    if (p->bc == IM3D_BC_NEU || p->bc == IM3D_BC_DIR)
    {
        call_with_enum (algo, &segm::rsfe_splitbregman<double>::set_bc, p->bc);
    }
    algo.set_cv (conv::filtering<double> (p->conv_cyclic ? rec_conv_cyclic : rec_conv) );

    const bool neu = p->bc == IM3D_BC_NEU;
    g_rec.bc_type = neu ? IM3D_BC_NEU : IM3D_BC_DIR;
    if (p->gs_rel_res_tol > 0)
    {
        g_rec.mode = 3;
        g_rec.rel_res_tol = p->gs_rel_res_tol;
        g_rec.max_sweeps = p->gs_max_sweeps;
        g_rec.check_every = p->gs_check_every;
        g_rec.omega = p->omega;
    }
    else if (p->sweep == IM3D_SWEEP_REDBLACK)
    {
        g_rec.mode = 2;
    }
    else
    {
        g_rec.mode = neu ? 1 : 0;
    }
    algo.set_onestep_poisson (lapl::unsteady_poisson_functor<double> (rec_poisson) );

    g_apply_start = now_s();
    if (init) algo.apply (u0, phi0);
    else algo.apply (u0);
    g_apply_end = now_s();
    g_last_stamps = g_rec.stamps;
    g_last_marks = g_rec.marks;
    g_last_solve = g_rec.solve_s;
    g_last_fft = g_rec.fft_s;

    img phi = algo.getoutput();
    if (phi_out) from_img (phi_out, phi);
    if (u_out) from_img (u_out, g_rec.u);
    const size_t n = (size_t) nx * ny * nz;
    if (f1_out || f2_out)
    {
        // rsfe_splitbregman_imp.hxx:1709-1717, in the reference's operation order
        img f1 = g_rec.num / g_rec.den;
        img num = g_rec.num, den = g_rec.den;
        num -= g_rec.kmyim;
        den -= g_rec.kones;
        num /= den;
        if (f1_out) from_img (f1_out, f1);
        if (f2_out) from_img (f2_out, num);
    }
    (void) n;
    if (stats)
    {
        std::memset (stats, 0, sizeof (*stats) );
        stats->iterations = (g_rec.conv_calls - g_rec.setup_convs) / 4;
        stats->total_sweeps = g_rec.sweeps;
        stats->last_sweeps = g_rec.last_sweeps;
        stats->last_rel_res = g_rec.last_rel;
        stats->not_converged = g_rec.not_converged;
        stats->residual_checks = g_rec.checks;
    }
    g_rec = Recorder();
    return 0;
}

/* Timing of the last ref_rsfe_apply: out[0] = start of apply, out[1..n] = wall time
 * at the end of each outer iteration's Poisson step, out[n+1] = end of apply.
 * Returns n + 2 (the number of values written, at most cap). */
int ref_last_timeline (double* out, int cap)
{
    int n = 0;
    if (n < cap) out[n++] = g_apply_start;
    for (double t : g_last_stamps)
        if (n < cap) out[n++] = t;
    if (n < cap) out[n++] = g_apply_end;
    return n;
}

/* Sweeps of the last ref_rsfe_apply: out[n] = sweeps run up to the end of the n-th
 * outer iteration's Poisson step. Returns the number of values written. */
int ref_last_sweep_marks (double* out, int cap)
{
    int n = 0;
    for (double m : g_last_marks)
        if (n < cap) out[n++] = m;
    return n;
}

/* Per outer iteration of the last ref_rsfe_apply: solve[n] = wall seconds inside its
 * Poisson step, fft[n] = wall seconds spent in FFTs (since the library loaded) up to
 * the end of that step. Returns the number of iterations written. */
int ref_last_step_profile (double* solve, double* fft, int cap)
{
    int n = 0;
    for (; n < (int) g_last_solve.size() && n < cap; ++n)
    {
        solve[n] = g_last_solve[n];
        fft[n] = g_last_fft[n];
    }
    return n;
}

}  // extern "C"

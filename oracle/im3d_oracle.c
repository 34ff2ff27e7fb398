/*
 * im3d_oracle.c -- CPU restatement (FP64) of the RSFE Split-Bregman path of
 * 3dimagetoolkit. TEST INFRASTRUCTURE ONLY: the checker, never the product.
 *
 * Restated from (paths relative to the reference project):
 *   header/convolution_imp.hxx   build_gaussian_filter :22-91, acyclic conv :535-653
 *   header/poisson_imp.hxx       NeuGaussSeidel :23-336, DirGaussSeidel :340-429
 *   header/image3d_imp.hxx       grad :744-889, div :948-1384, norms :1388-1511,
 *                                change_range_of_intensity :1628-1636
 *   header/rsfe_splitbregman_imp.hxx  ctor :25-41, cube init :48-95, init :99-170,
 *                                heaviside :174-192, edge_detect :196-316,
 *                                cut_phi :320-339, shrink :343-365, apply :1547-1995
 *
 * The Gaussian convolution is written as three 1-D passes with the per-axis
 * normalised taps. This is the same linear convolution the reference evaluates
 * with a zero-padded FFT: the reference's kernel is exp(-|d|^2/2s^2) normalised by
 * its L1 norm, which factors into the product of three normalised 1-D kernels, and
 * its padded length dim+Nh-1 leaves no circular wrap inside [0, dim).
 *
 * Reductions are summed per i-plane and then in plane order, so results do not
 * depend on the number of OpenMP threads.
 */
#include "im3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, k) (((size_t)(i) * ny + (j)) * nz + (k))

/* convolution_imp.hxx:36-80: Nh = ceil(2*radius*sigma/h) made odd, shift = Nh/2,
 * g[t] = exp(-(t-shift)^2 h^2 / (2 sigma^2)); normalised to unit sum per axis. */
int orc_gauss_taps(double sigma, double radius, double h, double* taps, int cap)
{
    int nh = (int)ceil(2 * radius * sigma / h);
    if (nh % 2 == 0) nh++;
    if (nh > cap) return -1;
    int shift = (int)floor((double)nh / 2.);
    double s = 0;
    for (int t = 0; t < nh; ++t) {
        double d = (double)(t - shift);
        taps[t] = exp(-d * d * h * h / (2 * sigma * sigma));
        s += taps[t];
    }
    for (int t = 0; t < nh; ++t) taps[t] /= s;
    return nh;
}

/* One axis of the separable filter: zero outside the volume, or with `cyclic` the
 * circular convolution out[a] = sum_t w[t] in[(a - t) mod len]. */
static void conv_axis(const double* in, double* out, int nx, int ny, int nz, int axis,
                      const double* w, int nh, int cyclic)
{
    const int shift = nh / 2;
    const int len = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const size_t stride = axis == 0 ? (size_t)ny * nz : (axis == 1 ? (size_t)nz : 1);
    #pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int pos = axis == 0 ? i : (axis == 1 ? j : k);
                const double* base = in + IDX(i, j, k) - (size_t)pos * stride;
                double acc = 0;
                for (int t = 0; t < nh; ++t) {
                    int q = pos - (t - shift);
                    if (cyclic) q = ((q % len) + len) % len;
                    if (q >= 0 && q < len) acc += w[t] * base[(size_t)q * stride];
                }
                out[IDX(i, j, k)] = acc;
            }
}

/* build_gaussian_filter (convolution_imp.hxx:22-91) + acyclic_fftw_convolution
 * (:535-653): result = linear convolution with the normalised Gaussian, zero outside
 * the volume, cropped to [0,dim). pixel_approach uses unit spacing for the taps. */
void orc_gauss_filter_mode(const double* in, double* out, int nx, int ny, int nz, double hx,
                           double hy, double hz, double sigma, double radius,
                           int pixel_approach, int cyclic)
{
    double wx[4096], wy[4096], wz[4096];
    double gx = pixel_approach ? 1. : hx, gy = pixel_approach ? 1. : hy,
           gz = pixel_approach ? 1. : hz;
    int nhx = orc_gauss_taps(sigma, radius, gx, wx, 4096);
    int nhy = orc_gauss_taps(sigma, radius, gy, wy, 4096);
    int nhz = nz == 1 ? 1 : orc_gauss_taps(sigma, radius, gz, wz, 4096);
    if (nz == 1) wz[0] = 1.;
    size_t n = (size_t)nx * ny * nz;
    double* tmp = (double*)malloc(n * sizeof(double));
    conv_axis(in, out, nx, ny, nz, 2, wz, nhz, cyclic);
    conv_axis(out, tmp, nx, ny, nz, 1, wy, nhy, cyclic);
    conv_axis(tmp, out, nx, ny, nz, 0, wx, nhx, cyclic);
    free(tmp);
}

void orc_gauss_filter(const double* in, double* out, int nx, int ny, int nz, double hx,
                      double hy, double hz, double sigma, double radius, int pixel_approach)
{
    orc_gauss_filter_mode(in, out, nx, ny, nz, hx, hy, hz, sigma, radius, pixel_approach, 0);
}

/* build_gaussian_filter + cyclic_fftw_convolution (convolution_imp.hxx:406-528,
 * 657-754): the reference periodises the volume over a grid of its own size (repeated
 * until it covers the kernel) and multiplies by the DFT of the wrapped kernel, which
 * is the circular convolution of each axis with the normalised taps. */
void orc_gauss_filter_cyclic(const double* in, double* out, int nx, int ny, int nz, double hx,
                             double hy, double hz, double sigma, double radius,
                             int pixel_approach)
{
    orc_gauss_filter_mode(in, out, nx, ny, nz, hx, hy, hz, sigma, radius, pixel_approach, 1);
}

/* image3d<T>::grad, 3-D branch (image3d_imp.hxx:750-838): central differences
 * inside, second-order one-sided differences on the faces. */
void orc_grad(const double* f, double* out3, int nx, int ny, int nz, double hx, double hy,
              double hz)
{
    size_t n = (size_t)nx * ny * nz;
    double* g0 = out3;
    double* g1 = out3 + n;
    double* g2 = out3 + 2 * n;
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t p = IDX(i, j, k);
                if (i == 0)
                    g0[p] = (4 * f[IDX(1, j, k)] - 3 * f[IDX(0, j, k)] - f[IDX(2, j, k)]) / (2. * hx);
                else if (i == nx - 1)
                    g0[p] = (3 * f[IDX(nx - 1, j, k)] - 4 * f[IDX(nx - 2, j, k)] +
                             f[IDX(nx - 3, j, k)]) / (2. * hx);
                else
                    g0[p] = (f[IDX(i + 1, j, k)] - f[IDX(i - 1, j, k)]) / (2. * hx);
                if (j == 0)
                    g1[p] = (4 * f[IDX(i, 1, k)] - 3 * f[IDX(i, 0, k)] - f[IDX(i, 2, k)]) / (2. * hy);
                else if (j == ny - 1)
                    g1[p] = (3 * f[IDX(i, ny - 1, k)] - 4 * f[IDX(i, ny - 2, k)] +
                             f[IDX(i, ny - 3, k)]) / (2. * hy);
                else
                    g1[p] = (f[IDX(i, j + 1, k)] - f[IDX(i, j - 1, k)]) / (2. * hy);
                if (k == 0)
                    g2[p] = (4 * f[IDX(i, j, 1)] - 3 * f[IDX(i, j, 0)] - f[IDX(i, j, 2)]) / (2. * hz);
                else if (k == nz - 1)
                    g2[p] = (3 * f[IDX(i, j, nz - 1)] - 4 * f[IDX(i, j, nz - 2)] +
                             f[IDX(i, j, nz - 3)]) / (2. * hz);
                else
                    g2[p] = (f[IDX(i, j, k + 1)] - f[IDX(i, j, k - 1)]) / (2. * hz);
            }
}

/* One axis term of im3d::div: which stencil applies depends on the position class
 * of the point along that axis (0 low face, 1 inside, 2 high face). */
static double div_term(const double* f, size_t p, size_t stride, int pos, int len, double h)
{
    if (pos == 0)
        return (4 * f[p + stride] - 3 * f[p] - f[p + 2 * stride]) / (2. * h);
    if (pos == len - 1)
        return (3 * f[p] - 4 * f[p - stride] + f[p - 2 * stride]) / (2. * h);
    return (f[p + stride] - f[p - stride]) / (2. * h);
}

/* im3d::div, 3-D branch (image3d_imp.hxx:1060-1380). Faces, edges and corners use
 * the one-sided stencil of grad per axis; two quirks of the reference are kept:
 *  - face i = X-1 with j, k inside (:1091-1099): the x term is ((3f-4f+f)/2)*hx
 *    (written `/ 2.* (hx)`), equal to the intended /(2 hx) only when hx = 1;
 *  - edge j = 0, k = Z-1 with i inside (:1203-1213): the z term reads Z-2 twice,
 *    (3 f[Z-1] - 4 f[Z-2] + f[Z-2]) / (2 hz). */
void orc_div(const double* in3, double* out, int nx, int ny, int nz, double hx, double hy,
             double hz)
{
    size_t n = (size_t)nx * ny * nz;
    const double* f0 = in3;
    const double* f1 = in3 + n;
    const double* f2 = in3 + 2 * n;
    const size_t sx = (size_t)ny * nz, sy = nz, sz = 1;
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t p = IDX(i, j, k);
                int cx = i == 0 ? 0 : (i == nx - 1 ? 2 : 1);
                int cy = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
                int cz = k == 0 ? 0 : (k == nz - 1 ? 2 : 1);
                double tx, tz;
                if (cx == 2 && cy == 1 && cz == 1)
                    tx = (3 * f0[p] - 4 * f0[p - sx] + f0[p - 2 * sx]) / 2. * (hx);
                else
                    tx = div_term(f0, p, sx, i, nx, hx);
                double ty = div_term(f1, p, sy, j, ny, hy);
                if (cx == 1 && cy == 0 && cz == 2)
                    tz = (3 * f2[p] - 4 * f2[p - sz] + f2[p - sz]) / (2. * hz);
                else
                    tz = div_term(f2, p, sz, k, nz, hz);
                out[p] = tx + ty + tz;
            }
}

/* ---------------------------------------------------------------- Gauss-Seidel */

typedef struct {
    int nx, ny, nz;
    double ihx2, ihy2, ihz2; /* 1/h^2 as (h*h) divisors are applied below */
    double hx, hy, hz, dt, bc;
    int neu;
} gs_geom;

/* Neighbour terms of one point (poisson_imp.hxx:340-429 for Dirichlet interior
 * points; :23-336 for Neumann, where a boundary axis reads the one inside neighbour
 * and the flux bc*h scaled by the oblique normal 1, 1/sqrt2, 1/sqrt3 for a face, an
 * edge, a corner). Returns the update value (sum + b + res/dt) * htilde; `self`
 * is the value used for the res/dt term. */
static double gs_point(const gs_geom* g, const double* r, const double* b, int i, int j,
                       int k, double self, double* htilde_out)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    size_t p = IDX(i, j, k);
    const double hx = g->hx, hy = g->hy, hz = g->hz, dt = g->dt;
    if (!g->neu) {
        double htilde = 1. / (1. / dt + 2. / (hx * hx) + 2. / (hy * hy) + 2. / (hz * hz));
        *htilde_out = htilde;
        return ((r[IDX(i + 1, j, k)] + r[IDX(i - 1, j, k)]) / (hx * hx) +
                (r[IDX(i, j + 1, k)] + r[IDX(i, j - 1, k)]) / (hy * hy) +
                (r[IDX(i, j, k + 1)] + r[IDX(i, j, k - 1)]) / (hz * hz) + b[p] + self / dt) *
               htilde;
    }
    int cx = i == 0 ? 0 : (i == nx - 1 ? 2 : 1);
    int cy = j == 0 ? 0 : (j == ny - 1 ? 2 : 1);
    int cz = k == 0 ? 0 : (k == nz - 1 ? 2 : 1);
    int nb = (cx != 1) + (cy != 1) + (cz != 1);
    double nrm = 1.;
    if (nb == 2) { nrm = 1.; nrm /= sqrt(2.); }
    if (nb == 3) { nrm = 1.; nrm /= sqrt(3.); }
    double bcn = nb == 1 ? g->bc : nrm * g->bc;
    double tx, ty, tz;
    if (cx == 1) tx = (r[IDX(i + 1, j, k)] + r[IDX(i - 1, j, k)]) / (hx * hx);
    else if (cx == 0) tx = (r[IDX(1, j, k)] - bcn * hx) / (hx * hx);
    else tx = (r[IDX(nx - 2, j, k)] + bcn * hx) / (hx * hx);
    if (cy == 1) ty = (r[IDX(i, j + 1, k)] + r[IDX(i, j - 1, k)]) / (hy * hy);
    else if (cy == 0) ty = (r[IDX(i, 1, k)] - bcn * hy) / (hy * hy);
    else ty = (r[IDX(i, ny - 2, k)] + bcn * hy) / (hy * hy);
    if (cz == 1) tz = (r[IDX(i, j, k + 1)] + r[IDX(i, j, k - 1)]) / (hz * hz);
    else if (cz == 0) tz = (r[IDX(i, j, 1)] - bcn * hz) / (hz * hz);
    else tz = (r[IDX(i, j, nz - 2)] + bcn * hz) / (hz * hz);
    double htilde = 1. / (1. / dt + (cx == 1 ? 2. : 1.) / (hx * hx) +
                          (cy == 1 ? 2. : 1.) / (hy * hy) + (cz == 1 ? 2. : 1.) / (hz * hz));
    *htilde_out = htilde;
    return (tx + ty + tz + b[p] + self / dt) * htilde;
}

static void dir_set_boundary(double* r, int nx, int ny, int nz, double bc)
{
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) r[IDX(0, j, k)] = r[IDX(nx - 1, j, k)] = bc;
    for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nx; ++i) r[IDX(i, 0, k)] = r[IDX(i, ny - 1, k)] = bc;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) r[IDX(i, j, 0)] = r[IDX(i, j, nz - 1)] = bc;
}

static void make_geom(gs_geom* g, int nx, int ny, int nz, double hx, double hy, double hz,
                      double dt, double bc, int bc_type)
{
    g->nx = nx; g->ny = ny; g->nz = nz;
    g->hx = hx; g->hy = hy; g->hz = hz;
    g->dt = dt; g->bc = bc;
    g->neu = bc_type == IM3D_BC_NEU;
}

/* `sweeps` in-place sweeps of DirGaussSeidel / NeuGaussSeidel. order 0 is the
 * reference's lexicographic order (Dir: i, j, k; Neu: k, j, i -- both give every
 * point new minus-neighbours and old plus-neighbours); order 1 is red-black. */
void orc_poisson_sweeps(double* res, const double* b, int nx, int ny, int nz, double hx,
                        double hy, double hz, double dt, double bc, int bc_type, int order,
                        int sweeps)
{
    gs_geom g;
    make_geom(&g, nx, ny, nz, hx, hy, hz, dt, bc, bc_type);
    int lo = g.neu ? 0 : 1;
    int hix = g.neu ? nx : nx - 1, hiy = g.neu ? ny : ny - 1, hiz = g.neu ? nz : nz - 1;
    double ht;
    for (int s = 0; s < sweeps; ++s) {
        if (!g.neu) dir_set_boundary(res, nx, ny, nz, bc);
        if (order == IM3D_SWEEP_LEXICOGRAPHIC) {
            if (!g.neu) {
                for (int i = lo; i < hix; ++i)
                    for (int j = lo; j < hiy; ++j)
                        for (int k = lo; k < hiz; ++k)
                            res[IDX(i, j, k)] = gs_point(&g, res, b, i, j, k, res[IDX(i, j, k)], &ht);
            } else {
                for (int k = lo; k < hiz; ++k)
                    for (int j = lo; j < hiy; ++j)
                        for (int i = lo; i < hix; ++i)
                            res[IDX(i, j, k)] = gs_point(&g, res, b, i, j, k, res[IDX(i, j, k)], &ht);
            }
        } else {
            for (int color = 0; color < 2; ++color) {
                #pragma omp parallel for schedule(static) private(ht)
                for (int i = lo; i < hix; ++i)
                    for (int j = lo; j < hiy; ++j)
                        for (int k = lo + ((i + j + lo + color) & 1); k < hiz; k += 2)
                            res[IDX(i, j, k)] = gs_point(&g, res, b, i, j, k, res[IDX(i, j, k)], &ht);
            }
        }
    }
}

/* Squared residual of (1/dt - Lap) u = uin/dt + b over the unknowns, and the squared
 * norm of uin/dt + b; the residual at p is (gs(p) - u_p)/htilde_p. */
static void solve_residual(const gs_geom* g, const double* u, const double* uin,
                           const double* b, double* rr, double* bb)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    int lo = g->neu ? 0 : 1;
    int hix = g->neu ? nx : nx - 1, hiy = g->neu ? ny : ny - 1, hiz = g->neu ? nz : nz - 1;
    double* prr = (double*)calloc(nx, sizeof(double));
    double* pbb = (double*)calloc(nx, sizeof(double));
    #pragma omp parallel for schedule(static)
    for (int i = lo; i < hix; ++i) {
        double sr = 0, sb = 0, ht;
        for (int j = lo; j < hiy; ++j)
            for (int k = lo; k < hiz; ++k) {
                size_t p = IDX(i, j, k);
                double v = gs_point(g, u, b, i, j, k, uin[p], &ht);
                double r = (v - u[p]) / ht;
                double e = b[p] + uin[p] / g->dt;
                sr += r * r;
                sb += e * e;
            }
        prr[i] = sr;
        pbb[i] = sb;
    }
    double sr = 0, sb = 0;
    for (int i = 0; i < nx; ++i) { sr += prr[i]; sb += pbb[i]; }
    free(prr);
    free(pbb);
    *rr = sr;
    *bb = sb;
}

/* Next residual check: a fixed interval when check_every > 0; otherwise
 * ceil(log(tol/r_s)/log(rate)) sweeps later, clamped to [1, 32], with
 * rate = (r_s/r_prev)^(1/(s - s_prev)) once two residuals are known, else the rate
 * carried over from the previous solve (rate_hint in (0, 1)), else 4 sweeps later. */
static int next_check(int s, double r_s, int s_prev, double r_prev, double tol, int check_every,
                      double rate_hint, double* rate_used)
{
    if (check_every > 0) return s + check_every;
    double rate;
    if (s_prev > 0 && r_prev > r_s && r_s > 0) rate = pow(r_s / r_prev, 1.0 / (double)(s - s_prev));
    else if (rate_hint > 0 && rate_hint < 1 && r_s > 0) rate = rate_hint;
    else return s + 4;
    *rate_used = rate;
    double need = log(tol / r_s) / log(rate);
    int step = 32;
    if (need == need && need < 32.0) step = (int)ceil(need);
    if (step < 1) step = 1;
    return s + step;
}

/* Red-black solve of (1/dt - Lap) u = uin/dt + b with uin = u on entry held fixed
 * (the converged form of one unsteady step; the reference's single sweep is its
 * first Gauss-Seidel iterate). Residual checked on the schedule of next_check; the
 * first check comes after first_check sweeps (0: after 4). rate_out (may be NULL)
 * receives the last contraction rate the schedule used (rate_hint if none). */
int orc_poisson_solve_sched(double* u, const double* b, int nx, int ny, int nz, double hx,
                            double hy, double hz, double dt, double bc, int bc_type,
                            double rel_res_tol, int max_sweeps, int check_every, double omega,
                            int first_check, double rate_hint, int* sweeps_done,
                            double* rel_res, double* rate_out, int* checks)
{
    gs_geom g;
    make_geom(&g, nx, ny, nz, hx, hy, hz, dt, bc, bc_type);
    size_t n = (size_t)nx * ny * nz;
    if (!g.neu) dir_set_boundary(u, nx, ny, nz, bc);
    double* uin = (double*)malloc(n * sizeof(double));
    memcpy(uin, u, n * sizeof(double));
    int lo = g.neu ? 0 : 1;
    int hix = g.neu ? nx : nx - 1, hiy = g.neu ? ny : ny - 1, hiz = g.neu ? nz : nz - 1;
    if (check_every < 0) check_every = 0;
    if (max_sweeps < 1) max_sweeps = 1;
    int s = 0, conv = 0, s_prev = 0;
    int next = check_every > 0 ? check_every : (first_check > 0 ? first_check : 4);
    double rel = -1, r_prev = -1, rate_used = 0;
    while (s < max_sweeps) {
        for (int color = 0; color < 2; ++color) {
            #pragma omp parallel for schedule(static)
            for (int i = lo; i < hix; ++i) {
                double ht;
                for (int j = lo; j < hiy; ++j)
                    for (int k = lo + ((i + j + lo + color) & 1); k < hiz; k += 2) {
                        size_t p = IDX(i, j, k);
                        double v = gs_point(&g, u, b, i, j, k, uin[p], &ht);
                        u[p] = omega == 1. ? v : u[p] + omega * (v - u[p]);
                    }
            }
        }
        ++s;
        if (s >= next || s == max_sweeps) {
            double rr, bb;
            solve_residual(&g, u, uin, b, &rr, &bb);
            if (checks) ++*checks;
            rel = bb > 0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
            if (rel <= rel_res_tol) { conv = 1; break; }
            next = next_check(s, rel, s_prev, r_prev, rel_res_tol, check_every, rate_hint, &rate_used);
            if (next > max_sweeps) next = max_sweeps;
            s_prev = s;
            r_prev = rel;
        }
    }
    free(uin);
    if (sweeps_done) *sweeps_done = s;
    if (rel_res) *rel_res = rel;
    if (rate_out) *rate_out = rate_used > 0 ? rate_used : rate_hint;
    return conv ? IM3D_OK : IM3D_ERR_NOT_CONVERGED;
}

int orc_poisson_solve(double* u, const double* b, int nx, int ny, int nz, double hx, double hy,
                      double hz, double dt, double bc, int bc_type, double rel_res_tol,
                      int max_sweeps, int check_every, double omega, int* sweeps_done,
                      double* rel_res)
{
    return orc_poisson_solve_sched(u, b, nx, ny, nz, hx, hy, hz, dt, bc, bc_type, rel_res_tol,
                                   max_sweeps, check_every, omega, 0, 0.0, sweeps_done, rel_res,
                                   NULL, NULL);
}

/* ------------------------------------------------------------------- the loop */

static double sum_sq_diff(const double* a, const double* b, size_t n, int nx)
{
    size_t plane = n / nx;
    double* part = (double*)calloc(nx, sizeof(double));
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        double s = 0;
        for (size_t q = (size_t)i * plane; q < (size_t)(i + 1) * plane; ++q) {
            double d = b ? a[q] - b[q] : a[q];
            s += d * d;
        }
        part[i] = s;
    }
    double s = 0;
    for (int i = 0; i < nx; ++i) s += part[i];
    free(part);
    return s;
}

static double vmin(const double* a, size_t n)
{
    double m = a[0];
    for (size_t q = 0; q < n; ++q) if (m > a[q]) m = a[q];
    return m;
}

static double vmax(const double* a, size_t n)
{
    double m = a[0];
    for (size_t q = 0; q < n; ++q) if (m < a[q]) m = a[q];
    return m;
}

/* rsfe_splitbregman<T>::apply(myim, init) (rsfe_splitbregman_imp.hxx:1547-1995). */
/* ------------------------------------------------------------ connected component */

/* image3d<T>::im_to_black_and_white (image3d_imp.hxx:1592-1623): 1 where the image is
 * at or above pivot = min + (max - min) * threshold (0 with `negative`), a threshold
 * outside [0, 1] replaced by 0.5. Returns the pivot. */
double orc_im_to_bw(const double* img, size_t n, double threshold, int negative,
                    unsigned char* bw)
{
    if (threshold > 1 || threshold < 0) threshold = 0.5;
    const double mx = vmax(img, n), mn = vmin(img, n);
    const double pivot = mn + (mx - mn) * threshold;
    for (size_t q = 0; q < n; ++q) bw[q] = img[q] < pivot ? (unsigned char)(negative != 0)
                                                          : (unsigned char)(negative == 0);
    return pivot;
}

/* The growth loop of connected_component (image3d_imp.hxx:1821-2120). The reference
 * repeats eight octant sweeps (four in 2-D) in which every set cell with
 * 1 <= i <= nx-2, 1 <= j <= ny-2 and (nz == 1 or 1 <= k <= nz-2) copies bw into its
 * forward face neighbours (and, with full_connected, the forward edge and corner
 * neighbours of that octant), until a sweep changes nothing. The set cells always lie
 * inside bw, so a copy only turns cells on, and the fixed point is the set of bw
 * cells reachable from the initial cells through cells off the faces: 6-connected
 * (4 in 2-D), or 26-connected (8) with full_connected. This computes that fixed point
 * with a work list. */
void orc_cc_grow(unsigned char* res, const unsigned char* bw, int nx, int ny, int nz, int full)
{
    const size_t n = (size_t)nx * ny * nz;
    size_t* list = (size_t*)malloc((n + 1) * sizeof(size_t));
    size_t head = 0, tail = 0;
    const int two_d = nz == 1;
#define SPREADS(i, j, k) ((i) >= 1 && (i) <= nx - 2 && (j) >= 1 && (j) <= ny - 2 && \
                          (two_d || ((k) >= 1 && (k) <= nz - 2)))
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                if (res[IDX(i, j, k)] && SPREADS(i, j, k)) list[tail++] = IDX(i, j, k);
    while (head < tail) {
        const size_t c = list[head++];
        const int k = (int)(c % nz), j = (int)((c / nz) % ny), i = (int)(c / ((size_t)nz * ny));
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = (two_d ? 0 : -1); dk <= (two_d ? 0 : 1); ++dk) {
                    const int nz_ = (di != 0) + (dj != 0) + (dk != 0);
                    if (nz_ == 0 || (!full && nz_ != 1)) continue;
                    const int a = i + di, b = j + dj, e = k + dk;
                    const size_t q = IDX(a, b, e);
                    if (res[q] || !bw[q]) continue;
                    res[q] = 1;
                    if (SPREADS(a, b, e)) list[tail++] = q;
                }
    }
#undef SPREADS
    free(list);
}

/* image3d<T>::connected_component (image3d_imp.hxx:1694-1817): seeded by cell
 * (i, j, k) moved off the faces (:1700-1736; in the negative image when the seed is
 * below the pivot, :1740-1745) when init == NULL, else by init != 0 inside bw
 * (:1761-1798); then the growth above, and with binary_output == 0
 * cc_not_binary_output (:1801-1817). */
int orc_connected_component(const double* img, double* res, int nx, int ny, int nz,
                            const double* init, int i, int j, int k, double threshold,
                            int full_connected, int binary_output)
{
    const size_t n = (size_t)nx * ny * nz;
    unsigned char* bw = (unsigned char*)malloc(n);
    unsigned char* r = (unsigned char*)calloc(n, 1);
    orc_im_to_bw(img, n, threshold, 0, bw);
    if (!init) {
        unsigned I = (unsigned)i, J = (unsigned)j, K = (unsigned)k;
        if (I == 0) ++I;
        if (J == 0) ++J;
        if (I >= (unsigned)nx - 1) I = nx - 2;
        if (J >= (unsigned)ny - 1) J = ny - 2;
        if (nz == 1) {
            K = 0;
        } else {
            if (K == 0) ++K;
            if (K >= (unsigned)nz - 1) K = nz - 2;
        }
        if (bw[IDX(I, J, K)] == 0) orc_im_to_bw(img, n, threshold, 1, bw);
        r[IDX(I, J, K)] = 1;
    } else {
        for (size_t q = 0; q < n; ++q) r[q] = (unsigned char)(init[q] != 0 && bw[q]);
    }
    orc_cc_grow(r, bw, nx, ny, nz, full_connected);
    for (size_t q = 0; q < n; ++q) res[q] = (double)r[q];
    if (!binary_output) {
        const double mn = vmin(img, n);
        orc_im_to_bw(img, n, threshold, 1, bw);
        for (size_t q = 0; q < n; ++q) {
            double v = res[q];
            v += (double)bw[q];
            v *= img[q] - mn;
            v += mn;
            res[q] = v;
        }
    }
    free(bw);
    free(r);
    return IM3D_OK;
}

/* extract_connected_component, automatic case (rsfe_splitbregman_imp.hxx:448-536):
 * seed cell floor(cc_init_pixel / h); nothing happens when it is outside the volume or
 * below the (alpha - a0)/(b0 - a0) threshold of phi; otherwise phi becomes its
 * connected component (threshold 0.5, face connectivity), rescaled to [a0, b0] by
 * change_range_of_intensity(b0, a0). Returns 1 when phi was replaced. */
static int extract_cc(double* phi, int nx, int ny, int nz, double hx, double hy, double hz,
                      const im3d_rsfe_params* p)
{
    const size_t n = (size_t)nx * ny * nz;
    const int i = (int)floor(p->cc_init_pixel_x / hx);
    const int j = (int)floor(p->cc_init_pixel_y / hy);
    const int k = (int)floor(p->cc_init_pixel_z / hz);
    if (i < 0 || j < 0 || (nz != 1 && k < 0)) return 0;
    const unsigned I = (unsigned)i, J = (unsigned)j, K = (unsigned)k;
    if (I > (unsigned)nx - 1 || J > (unsigned)ny - 1 || (nz != 1 && K > (unsigned)nz - 1)) return 0;
    unsigned char* bw = (unsigned char*)malloc(n);
    orc_im_to_bw(phi, n, (p->alpha - p->a0) / (p->b0 - p->a0), 0, bw);
    const int white = bw[IDX(I, J, K)] != 0;
    free(bw);
    if (!white) return 0;
    double* cc = (double*)malloc(n * sizeof(double));
    orc_connected_component(phi, cc, nx, ny, nz, NULL, (int)I, (int)J, (int)K, 0.5, 0,
                            p->cc_binary_output);
    /* phi = cc; change_range_of_intensity(b0, a0) (image3d_imp.hxx:1628-1636) */
    const double mn = vmin(cc, n);
    for (size_t q = 0; q < n; ++q) cc[q] -= mn;
    const double sc = vmax(cc, n) / (p->b0 - p->a0);
    for (size_t q = 0; q < n; ++q) {
        cc[q] /= sc;
        cc[q] += p->a0;
    }
    memcpy(phi, cc, n * sizeof(double));
    free(cc);
    return 1;
}

int orc_rsfe_apply(const double* u0, const double* init, int nx, int ny, int nz, double hx,
                   double hy, double hz, const im3d_rsfe_params* p, double* phi_out,
                   double* u_out, double* f1_out, double* f2_out, im3d_rsfe_stats* stats)
{
    if (nx < 3 || ny < 3 || nz < 3) return IM3D_ERR_UNSUPPORTED;
    const size_t n = (size_t)nx * ny * nz;
    double* phi = phi_out;
    double* phiold = (double*)malloc(n * sizeof(double));
    double* kones = (double*)malloc(n * sizeof(double));
    double* kmyim = (double*)malloc(n * sizeof(double));
    double* g = (double*)malloc(n * sizeof(double));
    double* divdb = (double*)calloc(n, sizeof(double));
    double* bb = (double*)calloc(3 * n, sizeof(double));
    double* d = (double*)malloc(3 * n * sizeof(double));
    double* num = (double*)malloc(n * sizeof(double));
    double* den = (double*)malloc(n * sizeof(double));
    double* f1 = (double*)malloc(n * sizeof(double));
    double* f2 = (double*)malloc(n * sizeof(double));
    double* kr1 = (double*)malloc(n * sizeof(double));
    double* kr2 = (double*)malloc(n * sizeof(double));
    double* aux = (double*)malloc(n * sizeof(double));
    const double a0 = p->a0, b0 = p->b0;

    /* initial level set: initialize_phi_with_init (:99-170) or the cube (:48-95) */
    if (init) {
        memcpy(phi, init, n * sizeof(double));
    } else {
        int ix = (int)(nx * 0.33), iy = (int)(ny * 0.33), iz = (int)(nz * 0.33);
        int fx = (int)(nx * (1 - 0.33)), fy = (int)(ny * (1 - 0.33)), fz = (int)(nz * (1 - 0.33));
        for (size_t q = 0; q < n; ++q) phi[q] = a0;
        for (int i = ix; i < fx; ++i)
            for (int j = iy; j < fy; ++j)
                for (int k = iz; k < fz; ++k) phi[IDX(i, j, k)] = b0;
    }
    /* change_range_of_intensity(b0, a0) (image3d_imp.hxx:1628-1636) */
    {
        double mn = vmin(phi, n);
        for (size_t q = 0; q < n; ++q) phi[q] -= mn;
        double mx = vmax(phi, n);
        double sc = mx / (b0 - a0);
        for (size_t q = 0; q < n; ++q) { phi[q] /= sc; phi[q] += a0; }
    }

    /* kones = K*1, kmyim = K*u0 (:1648-1651) */
    for (size_t q = 0; q < n; ++q) aux[q] = 1.;
    orc_gauss_filter_mode(aux, kones, nx, ny, nz, hx, hy, hz, p->sigma, 3, p->gaussian_pixel_approach, p->conv_cyclic);
    orc_gauss_filter_mode(u0, kmyim, nx, ny, nz, hx, hy, hz, p->sigma, 3, p->gaussian_pixel_approach, p->conv_cyclic);

    /* edge_detect, GRAD branch (:196-316): optional pre-blur, |grad u0|^2, then
     * g = nu / (lamda (1 + beta |grad u0|^2)) in the reference's operation order */
    {
        const double* src = u0;
        if (p->edge_detector_sigma != 0) {
            orc_gauss_filter_mode(u0, aux, nx, ny, nz, hx, hy, hz, p->edge_detector_sigma, 3,
                             p->gaussian_pixel_approach, p->conv_cyclic);
            src = aux;
        }
        orc_grad(src, d, nx, ny, nz, hx, hy, hz);
        for (size_t q = 0; q < n; ++q) {
            double a = d[q] * d[q];
            a += d[n + q] * d[n + q];
            a += d[2 * n + q] * d[2 * n + q];
            a *= p->beta;
            a += 1.;
            double r = 1.;
            r /= a;
            r /= p->lamda;
            r *= p->nu;
            g[q] = r;
        }
    }

    const double center = (a0 + b0) / 2.;
    const double M_PI_ = 3.14159265358979323846;
    double tollerance = 1000;
    int init_variables = p->init_variables;
    int t;
    long long total_sweeps = 0;
    int last_sweeps = 0, not_conv = 0;
    double last_rel = -1, last_ls_err = -1;
    const int bc_type = p->bc;
    /* chosen_bc (:1735-1743): NEU -> 0, DIR -> a0; the constructor default is NEU */
    const double chosen_bc = (bc_type == IM3D_BC_DIR) ? a0 : 0.;
    const int neu = bc_type == IM3D_BC_NEU;
    int sched_first = 0;     /* residual schedule carried between Poisson solves */
    int checks = 0;
    double sched_rate = 0;

    for (t = 1; tollerance > p->tol && t <= p->maxiter; ++t) {
        memcpy(phiold, phi, n * sizeof(double));
        /* set_heaviside (:174-192) */
        for (size_t q = 0; q < n; ++q) {
            double H = 0.5 * (1. + 2. / M_PI_ * atan((phi[q] - center) / (p->epsilon)));
            aux[q] = H * u0[q];
            f1[q] = H;
        }
        orc_gauss_filter_mode(aux, num, nx, ny, nz, hx, hy, hz, p->sigma, 3, p->gaussian_pixel_approach, p->conv_cyclic);
        orc_gauss_filter_mode(f1, den, nx, ny, nz, hx, hy, hz, p->sigma, 3, p->gaussian_pixel_approach, p->conv_cyclic);
        /* f1, f2 (:1709-1717) */
        for (size_t q = 0; q < n; ++q) {
            f1[q] = num[q] / den[q];
            double nm = num[q] - kmyim[q];
            double dn = den[q] - kones[q];
            f2[q] = nm / dn;
        }
        /* kr2 = K*(lamda1 f1 - lamda2 f2), kr1 = K*(lamda1 f1^2 - lamda2 f2^2) (:1720-1729) */
        for (size_t q = 0; q < n; ++q) aux[q] = f1[q] * p->lamda1 - f2[q] * p->lamda2;
        orc_gauss_filter_mode(aux, kr2, nx, ny, nz, hx, hy, hz, p->sigma, 3, p->gaussian_pixel_approach, p->conv_cyclic);
        for (size_t q = 0; q < n; ++q) {
            double a = f1[q];
            a *= a;
            a *= p->lamda1;
            double b2 = f2[q];
            b2 *= b2;
            b2 *= p->lamda2;
            a -= b2;
            aux[q] = a;
        }
        orc_gauss_filter_mode(aux, kr1, nx, ny, nz, hx, hy, hz, p->sigma, 3, p->gaussian_pixel_approach, p->conv_cyclic);
        if (f1_out) memcpy(f1_out, f1, n * sizeof(double));
        if (f2_out) memcpy(f2_out, f2, n * sizeof(double));
        /* forcing term (:1750-1761) */
        for (size_t q = 0; q < n; ++q) {
            double r = kr2[q];
            r *= u0[q];
            r *= 2;
            double a = p->lamda1 - p->lamda2;
            a *= u0[q];
            a *= u0[q];
            a *= kones[q];
            r -= a;
            r -= kr1[q];
            r /= p->lamda;
            r -= divdb[q];
            kr2[q] = r;
        }
        /* the Poisson step (:1768-1785) */
        if (p->gs_rel_res_tol > 0) {
            int sw = 0;
            double rel = -1, rate = 0;
            /* the schedule of each solve starts from the previous one: first check
             * after as many sweeps as it needed, its contraction rate as the first
             * prediction */
            int st = orc_poisson_solve_sched(phi, kr2, nx, ny, nz, hx, hy, hz, p->dt, chosen_bc,
                                             neu ? IM3D_BC_NEU : IM3D_BC_DIR, p->gs_rel_res_tol,
                                             p->gs_max_sweeps, p->gs_check_every, p->omega,
                                             sched_first, sched_rate, &sw, &rel, &rate, &checks);
            sched_first = st == IM3D_OK ? sw : 0;
            sched_rate = st == IM3D_OK ? rate : 0;
            if (st != IM3D_OK) not_conv++;
            total_sweeps += sw;
            last_sweeps = sw;
            last_rel = rel;
        } else {
            double ls_err = p->ls_tol ? 1000. : -1.;
            int s;
            for (s = 0; s < p->ls_steps || ls_err > p->ls_tol; ++s) {
                if (p->ls_tol != 0) memcpy(aux, phi, n * sizeof(double));
                orc_poisson_sweeps(phi, kr2, nx, ny, nz, hx, hy, hz, p->dt, chosen_bc,
                                   neu ? IM3D_BC_NEU : IM3D_BC_DIR, p->sweep, 1);
                if (p->ls_tol != 0 && s >= p->ls_steps - 1)
                    ls_err = sqrt(sum_sq_diff(phi, aux, n, nx)) / sqrt(sum_sq_diff(aux, NULL, n, nx));
                if (s > 100000) break;
            }
            total_sweeps += s;
            last_sweeps = s;
            last_ls_err = ls_err;
        }
        if (u_out) memcpy(u_out, phi, n * sizeof(double));
        /* cut_phi (:320-339) */
        for (size_t q = 0; q < n; ++q) {
            if (phi[q] < a0) phi[q] = a0;
            else if (phi[q] > b0) phi[q] = b0;
        }
        /* automatic connected-component extraction (:1809-1812) */
        if (p->auto_extract_conn_comp && p->auto_extract_conn_comp_freq != 0 &&
            t % p->auto_extract_conn_comp_freq == 0) {
            if (extract_cc(phi, nx, ny, nz, hx, hy, hz, p) && p->cc_init_variables) init_variables = 1;
        }
        /* tolerance (:1832): normL2(phi - phiold)/normL2(phiold) */
        tollerance = sqrt(hx * hy * hz * sum_sq_diff(phi, phiold, n, nx)) /
                     sqrt(hx * hy * hz * sum_sq_diff(phiold, NULL, n, nx));
        if (init_variables) {
            memset(divdb, 0, n * sizeof(double));
            memset(bb, 0, 3 * n * sizeof(double));
            init_variables = 0;
        } else {
            /* d = grad(phi); b += d; d = shrink(b, g); b -= d; d -= b; divdb = div(d)
             * (:1868-1932, shrink :343-365) */
            orc_grad(phi, d, nx, ny, nz, hx, hy, hz);
            for (size_t q = 0; q < 3 * n; ++q) bb[q] += d[q];
            for (int c = 0; c < 3; ++c)
                for (size_t q = 0; q < n; ++q) {
                    double v = bb[c * n + q];
                    double sgn = (double)((int)(v > 0.) - (int)(v < 0.));
                    double m = fabs(v) - g[q];
                    d[c * n + q] = sgn * ((m < 0.) ? 0. : m); /* std::max(m, 0) */
                }
            for (size_t q = 0; q < 3 * n; ++q) {
                bb[q] -= d[q];
                d[q] -= bb[q];
            }
            orc_div(d, divdb, nx, ny, nz, hx, hy, hz);
        }
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->iterations = t - 1;
        stats->last_tol = tollerance;
        stats->total_sweeps = total_sweeps;
        stats->last_sweeps = last_sweeps;
        stats->last_rel_res = last_rel;
        stats->last_ls_err = last_ls_err;
        stats->not_converged = not_conv;
        stats->residual_checks = checks;
    }
    free(phiold); free(kones); free(kmyim); free(g); free(divdb); free(bb); free(d);
    free(num); free(den); free(f1); free(f2); free(kr1); free(kr2); free(aux);
    return IM3D_OK;
}

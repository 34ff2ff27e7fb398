/*
 * fft_shim.cpp -- FP64 complex DFT behind the FFTW3 names declared in fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU checker's build of the reference).
 *
 * Written from the DFT definition and two published algorithms:
 *  - mixed-radix Cooley-Tukey (decimation in time, recursive, out of place) for
 *    lengths whose prime factors are all <= 7;
 *  - Bluestein's chirp-z identity jk = (j^2 + k^2 - (k-j)^2)/2 for every other
 *    length, turning a length-n DFT into a circular convolution of power-of-two
 *    length m >= 2n-1 (evaluated with the radix-2 path above).
 * Twiddles are computed directly with cos/sin of an exactly reduced angle (no
 * recurrences), so the transform is accurate to a few ulp times log2(n).
 * A 3-D transform is three batches of 1-D transforms (axis 2 is contiguous),
 * parallel over lines with OpenMP, as FFTW's threaded planner would run it.
 */
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

typedef std::complex<double> cplx;

struct Plan1D {
    int n = 0;
    int sign = -1;
    bool bluestein = false;
    std::vector<int> factors;  // Cooley-Tukey radices, product = n
    std::vector<cplx> tw;      // tw[e] = exp(sign*2*pi*i*e/n), e in [0, n)
    // Bluestein state
    int m = 0;
    std::vector<cplx> chirp;   // c[k] = exp(sign*i*pi*k^2/n)
    std::vector<cplx> bhat;    // FFT_m of conj(chirp) arranged circularly
    Plan1D* fwd_m = nullptr;   // length-m forward transform
    Plan1D* bwd_m = nullptr;   // length-m backward transform

    ~Plan1D() { delete fwd_m; delete bwd_m; }
};

const double kPi = 3.14159265358979323846264338327950288;

void exec_1d(const Plan1D* p, const cplx* in, cplx* out, cplx* scratch);

bool factorize_small(int n, std::vector<int>& f)
{
    f.clear();
    int r = n;
    while (r % 4 == 0) { f.push_back(4); r /= 4; }
    const int primes[] = {2, 3, 5, 7};
    for (int p : primes)
        while (r % p == 0) { f.push_back(p); r /= p; }
    return r == 1;
}

Plan1D* make_plan(int n, int sign);

void init_twiddles(Plan1D* p)
{
    p->tw.resize(p->n);
    for (int e = 0; e < p->n; ++e) {
        double ang = p->sign * 2.0 * kPi * (double)e / (double)p->n;
        p->tw[e] = cplx(std::cos(ang), std::sin(ang));
    }
}

Plan1D* make_plan(int n, int sign)
{
    Plan1D* p = new Plan1D();
    p->n = n;
    p->sign = sign;
    if (n <= 1 || factorize_small(n, p->factors)) {
        if (n <= 1) p->factors.clear();
        init_twiddles(p);
        return p;
    }
    // Bluestein
    p->bluestein = true;
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp.resize(n);
    const long long two_n = 2LL * n;
    for (long long k = 0; k < n; ++k) {
        long long e = (k * k) % two_n;  // exact angle reduction: k^2 mod 2n
        double ang = sign * kPi * (double)e / (double)n;
        p->chirp[k] = cplx(std::cos(ang), std::sin(ang));
    }
    p->fwd_m = make_plan(m, -1);
    p->bwd_m = make_plan(m, +1);
    std::vector<cplx> b(m, cplx(0, 0));
    b[0] = std::conj(p->chirp[0]);
    for (int d = 1; d < n; ++d) {
        b[d] = std::conj(p->chirp[d]);
        b[m - d] = std::conj(p->chirp[d]);
    }
    p->bhat.resize(m);
    std::vector<cplx> scratch(4 * m + 16);
    exec_1d(p->fwd_m, b.data(), p->bhat.data(), scratch.data());
    return p;
}

// Recursive decimation-in-time: out[0..n) = DFT_n of in[0], in[stride], ...
// tw_step maps this sub-transform's twiddle exponent to the root table of size N.
void ct_rec(const Plan1D* p, const cplx* in, cplx* out, int n, long stride, int level,
            long tw_step)
{
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int r = p->factors[level];
    const int m = n / r;
    for (int q = 0; q < r; ++q)
        ct_rec(p, in + q * stride, out + q * m, m, stride * r, level + 1, tw_step * r);
    const int N = p->n;
    cplx t[7];
    cplx y[7];
    for (int k = 0; k < m; ++k) {
        // twiddle the r partial transforms
        for (int q = 0; q < r; ++q) {
            long e = ((long)q * k * tw_step) % N;
            t[q] = out[q * m + k] * p->tw[e];
        }
        // radix-r DFT over q
        for (int s = 0; s < r; ++s) {
            cplx acc(0, 0);
            for (int q = 0; q < r; ++q) {
                long e = ((long)q * s * m * tw_step) % N;  // w_r^(q*s)
                acc += t[q] * p->tw[e];
            }
            y[s] = acc;
        }
        for (int s = 0; s < r; ++s) out[k + s * m] = y[s];
    }
}

void exec_1d(const Plan1D* p, const cplx* in, cplx* out, cplx* scratch)
{
    const int n = p->n;
    if (!p->bluestein) {
        if (n == 1) { out[0] = in[0]; return; }
        ct_rec(p, in, out, n, 1, 0, 1);
        return;
    }
    const int m = p->m;
    cplx* a = scratch;         // m
    cplx* ahat = scratch + m;  // m
    cplx* rest = scratch + 2 * m;
    for (int j = 0; j < n; ++j) a[j] = in[j] * p->chirp[j];
    for (int j = n; j < m; ++j) a[j] = cplx(0, 0);
    exec_1d(p->fwd_m, a, ahat, rest);
    for (int j = 0; j < m; ++j) ahat[j] *= p->bhat[j];
    exec_1d(p->bwd_m, ahat, a, rest);
    const double inv_m = 1.0 / (double)m;
    for (int k = 0; k < n; ++k) out[k] = p->chirp[k] * a[k] * inv_m;
}

}  // namespace

struct im3d_fft_plan_s {
    int n[3];
    int sign;
    cplx* in;
    cplx* out;
    Plan1D* axis[3];
};

static int g_nthreads = 0;

extern "C" {

void* fftw_malloc(size_t n) { return std::malloc(n); }
void fftw_free(void* p) { std::free(p); }

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out,
                           int sign, unsigned flags)
{
    (void)flags;
    im3d_fft_plan_s* p = new im3d_fft_plan_s();
    p->n[0] = n0; p->n[1] = n1; p->n[2] = n2;
    p->sign = sign;
    p->in = reinterpret_cast<cplx*>(in);
    p->out = reinterpret_cast<cplx*>(out);
    for (int a = 0; a < 3; ++a) p->axis[a] = make_plan(p->n[a], sign);
    return p;
}

void fftw_execute(const fftw_plan pc)
{
    im3d_fft_plan_s* p = pc;
    const long n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    const long total = n0 * n1 * n2;
    if (p->out != p->in) std::memcpy(p->out, p->in, sizeof(cplx) * total);
    cplx* data = p->out;
    const long strides[3] = {n1 * n2, n2, 1};
    int nthreads = g_nthreads > 0 ? g_nthreads : omp_get_max_threads();
    for (int a = 2; a >= 0; --a) {
        const long len = p->n[a];
        if (len <= 1) continue;
        const long stride = strides[a];
        const Plan1D* pl = p->axis[a];
        const long lines = total / len;
        const long scratch_len = 4L * (pl->bluestein ? pl->m : len) + 16;
        #pragma omp parallel num_threads(nthreads)
        {
            std::vector<cplx> line(len), res(len), scratch(scratch_len);
            #pragma omp for schedule(static)
            for (long l = 0; l < lines; ++l) {
                // line l: the index with axis a removed, in row-major order
                long base;
                if (a == 2) base = l * len;
                else if (a == 1) base = (l / n2) * (n1 * n2) + (l % n2);
                else base = l;
                for (long t = 0; t < len; ++t) line[t] = data[base + t * stride];
                exec_1d(pl, line.data(), res.data(), scratch.data());
                for (long t = 0; t < len; ++t) data[base + t * stride] = res[t];
            }
        }
    }
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    for (int a = 0; a < 3; ++a) delete p->axis[a];
    delete p;
}

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads; }
void fftw_cleanup_threads(void) {}

}  // extern "C"

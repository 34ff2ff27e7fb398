/*
 * fft_shim.cpp -- FP64 complex DFT behind the FFTW3 names declared in fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU checker's build of the reference, which is also
 * the timed CPU baseline; FFTW itself is not available on this machine).
 *
 * Written from the DFT definition and two published algorithms:
 *  - mixed-radix Cooley-Tukey, decimation in time, recursive and out of place, with
 *    radices 4, 2, 3, 5, 7 (radix 2 and 4 butterflies written out);
 *  - Bluestein's chirp-z identity jk = (j^2 + k^2 - (k-j)^2)/2 for the part of the
 *    length with no factor <= 7, turning that DFT into a circular convolution of
 *    power-of-two length m >= 2p-1 (e.g. 274 = 2 * 137: two length-137 Bluestein
 *    transforms of size 512 under one radix-2 stage).
 * Twiddles are computed directly with cos/sin of an exactly reduced angle (no
 * recurrences), so the transform is accurate to a few ulp times log2(n).
 * A 3-D transform is three batches of 1-D transforms (axis 2 contiguous), parallel
 * over lines with OpenMP, as FFTW's threaded planner would run it.
 *
 * im3d_fft_shim_set_external() hands fftw_execute to another in-place transform: the
 * timed CPU baseline registers scipy's pocketfft there (a tuned multi-threaded FFT, the
 * closest stand-in for FFTW on these hosts), the checker keeps the in-tree transform.
 */
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

typedef std::complex<double> cplx;
const double kPi = 3.14159265358979323846264338327950288;

struct Plan1D {
    int n = 0;
    int sign = -1;
    std::vector<int> factors;  // small radices; their product times `large` is n
    int large = 1;             // cofactor with no prime factor <= 7 (Bluestein)
    std::vector<cplx> tw;      // tw[e] = exp(sign*2*pi*i*e/n), e in [0, n)
    // Bluestein of length `large` (pow2 size m)
    int m = 0;
    std::vector<cplx> chirp;   // exp(sign*i*pi*k^2/large)
    std::vector<cplx> bhat;    // FFT_m of conj(chirp), circular
    Plan1D* fwd_m = nullptr;
    Plan1D* bwd_m = nullptr;
    ~Plan1D() { delete fwd_m; delete bwd_m; }
};

void exec_1d(const Plan1D* p, const cplx* in, long stride, cplx* out, cplx* scratch);

Plan1D* make_plan(int n, int sign)
{
    Plan1D* p = new Plan1D();
    p->n = n;
    p->sign = sign;
    int r = n;
    while (r % 4 == 0) { p->factors.push_back(4); r /= 4; }
    const int primes[] = {2, 3, 5, 7};
    for (int q : primes)
        while (r % q == 0) { p->factors.push_back(q); r /= q; }
    p->large = r;
    p->tw.resize(n);
    for (int e = 0; e < n; ++e) {
        double ang = sign * 2.0 * kPi * (double)e / (double)n;
        p->tw[e] = cplx(std::cos(ang), std::sin(ang));
    }
    if (r > 1) {
        int m = 1;
        while (m < 2 * r - 1) m <<= 1;
        p->m = m;
        p->chirp.resize(r);
        const long long two_r = 2LL * r;
        for (long long k = 0; k < r; ++k) {
            long long e = (k * k) % two_r;  // exact angle reduction: k^2 mod 2r
            double ang = sign * kPi * (double)e / (double)r;
            p->chirp[k] = cplx(std::cos(ang), std::sin(ang));
        }
        p->fwd_m = make_plan(m, -1);
        p->bwd_m = make_plan(m, +1);
        std::vector<cplx> b(m, cplx(0, 0));
        b[0] = std::conj(p->chirp[0]);
        for (int d = 1; d < r; ++d) {
            b[d] = std::conj(p->chirp[d]);
            b[m - d] = std::conj(p->chirp[d]);
        }
        p->bhat.resize(m);
        std::vector<cplx> scratch(4 * m + 64);
        exec_1d(p->fwd_m, b.data(), 1, p->bhat.data(), scratch.data());
    }
    return p;
}

// Length-`large` DFT of in[0], in[stride], ... by Bluestein.
void bluestein(const Plan1D* p, const cplx* in, long stride, cplx* out, cplx* scratch)
{
    const int r = p->large, m = p->m;
    cplx* a = scratch;
    cplx* ahat = scratch + m;
    cplx* rest = scratch + 2 * m;
    for (int j = 0; j < r; ++j) a[j] = in[j * stride] * p->chirp[j];
    for (int j = r; j < m; ++j) a[j] = cplx(0, 0);
    exec_1d(p->fwd_m, a, 1, ahat, rest);
    for (int j = 0; j < m; ++j) ahat[j] *= p->bhat[j];
    exec_1d(p->bwd_m, ahat, 1, a, rest);
    const double inv_m = 1.0 / (double)m;
    for (int k = 0; k < r; ++k) out[k] = p->chirp[k] * (a[k] * inv_m);
}

// out[0..n) = DFT_n of in[0], in[stride], ...; w_n^e = tw[e * tw_step].
void ct_rec(const Plan1D* p, const cplx* in, long stride, cplx* out, int n, int level,
            long tw_step, cplx* scratch)
{
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    if (level == (int)p->factors.size()) {  // n == p->large
        bluestein(p, in, stride, out, scratch);
        return;
    }
    const int r = p->factors[level];
    const int m = n / r;
    for (int q = 0; q < r; ++q)
        ct_rec(p, in + q * stride, stride * r, out + q * m, m, level + 1, tw_step * r, scratch);
    const cplx* tw = p->tw.data();
    const long N = p->n;
    if (r == 2) {
        for (int k = 0; k < m; ++k) {
            const cplx a = out[k];
            const cplx b = out[m + k] * tw[k * tw_step];
            out[k] = a + b;
            out[m + k] = a - b;
        }
        return;
    }
    if (r == 4) {
        // w_4 = exp(sign*i*pi/2) = sign*i
        const double sg = (double)p->sign;
        for (int k = 0; k < m; ++k) {
            const cplx t0 = out[k];
            const cplx t1 = out[m + k] * tw[k * tw_step];
            const cplx t2 = out[2 * m + k] * tw[2 * k * tw_step];
            const cplx t3 = out[3 * m + k] * tw[3 * k * tw_step];
            const cplx s02 = t0 + t2, d02 = t0 - t2, s13 = t1 + t3, d13 = t1 - t3;
            const cplx jd13(-sg * d13.imag(), sg * d13.real());  // (sign*i) * d13
            out[k] = s02 + s13;
            out[m + k] = d02 + jd13;
            out[2 * m + k] = s02 - s13;
            out[3 * m + k] = d02 - jd13;
        }
        return;
    }
    cplx t[7], y[7];
    const long step_r = N / r;  // w_r = tw[step_r]
    for (int k = 0; k < m; ++k) {
        for (int q = 0; q < r; ++q) t[q] = out[q * m + k] * tw[(long)q * k * tw_step];
        for (int s = 0; s < r; ++s) {
            cplx acc = t[0];
            for (int q = 1; q < r; ++q) acc += t[q] * tw[((q * s) % r) * step_r];
            y[s] = acc;
        }
        for (int s = 0; s < r; ++s) out[k + s * m] = y[s];
    }
}

void exec_1d(const Plan1D* p, const cplx* in, long stride, cplx* out, cplx* scratch)
{
    ct_rec(p, in, stride, out, p->n, 0, 1, scratch);
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
static double g_exec_seconds = 0;  // wall time spent in fftw_execute since the library loaded
static long long g_exec_calls = 0;
// An external in-place 3-D transform (unnormalised, sign as FFTW's) that serves
// fftw_execute instead of the in-tree one when set (the CPU baseline registers a tuned
// library's FFT here; the checker keeps the in-tree transform).
typedef int (*im3d_fft_external_fn)(int n0, int n1, int n2, void* data, int sign);
static im3d_fft_external_fn g_external = nullptr;

static void execute_3d(im3d_fft_plan_s* p);

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
    const double t0 = omp_get_wtime();
    if (g_external) {
        const long total = (long)pc->n[0] * pc->n[1] * pc->n[2];
        if (pc->out != pc->in) {
            // out-of-place plan: the transform runs in place on out
            const int nthreads = g_nthreads > 0 ? g_nthreads : omp_get_max_threads();
            #pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long c = 0; c < total; c += 65536)
                std::memcpy(pc->out + c, pc->in + c, sizeof(cplx) * std::min<long>(65536, total - c));
        }
        g_external(pc->n[0], pc->n[1], pc->n[2], pc->out, pc->sign);
    } else {
        execute_3d(pc);
    }
    g_exec_seconds += omp_get_wtime() - t0;
    ++g_exec_calls;
}

/* Serve fftw_execute with an external transform (NULL: the in-tree one again). */
void im3d_fft_shim_set_external(im3d_fft_external_fn fn) { g_external = fn; }

/* Wall seconds spent in fftw_execute and the number of its calls since the library
 * loaded (the CPU baseline's FFT share of an outer iteration). */
void im3d_fft_shim_totals(double* seconds, long long* calls)
{
    if (seconds) *seconds = g_exec_seconds;
    if (calls) *calls = g_exec_calls;
}

}  // extern "C"

static void execute_3d(im3d_fft_plan_s* p)
{
    const long n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    const long total = n0 * n1 * n2;
    if (p->out != p->in) std::memcpy(p->out, p->in, sizeof(cplx) * total);
    cplx* data = p->out;
    const long strides[3] = {n1 * n2, n2, 1};
    const int nthreads = g_nthreads > 0 ? g_nthreads : omp_get_max_threads();
    // Axis 2 lines are contiguous. For axes 1 and 0, lines that are neighbours along
    // the contiguous axis are transformed together in tiles of B, so every gathered
    // cache line serves B transforms.
    const int B = 8;
    for (int a = 2; a >= 0; --a) {
        const long len = p->n[a];
        if (len <= 1) continue;
        const long stride = strides[a];
        const Plan1D* pl = p->axis[a];
        const long scratch_len = 4L * (pl->m > 0 ? pl->m : 1) + 64;
        // tiles: (outer, inner start); inner runs along the contiguous axis
        const long inner = a == 2 ? 1 : (a == 1 ? n2 : n1 * n2);
        const long outer = a == 2 ? n0 * n1 : (a == 1 ? n0 : 1);
        const long tiles_in = a == 2 ? 1 : (inner + B - 1) / B;
        const long ntiles = outer * tiles_in;
        #pragma omp parallel num_threads(nthreads)
        {
            std::vector<cplx> tile(len * B), res(len), scratch(scratch_len);
            #pragma omp for schedule(static)
            for (long tI = 0; tI < ntiles; ++tI) {
                const long o = tI / tiles_in;
                if (a == 2) {
                    cplx* line = data + o * len;
                    exec_1d(pl, line, 1, res.data(), scratch.data());
                    std::memcpy(line, res.data(), sizeof(cplx) * len);
                    continue;
                }
                const long i0 = (tI % tiles_in) * B;
                const int nb = (int)std::min<long>(B, inner - i0);
                const long base = (a == 1 ? o * n1 * n2 : 0) + i0;
                for (long t = 0; t < len; ++t)
                    for (int b = 0; b < nb; ++b) tile[t * B + b] = data[base + t * stride + b];
                for (int b = 0; b < nb; ++b) {
                    exec_1d(pl, tile.data() + b, B, res.data(), scratch.data());
                    for (long t = 0; t < len; ++t) tile[t * B + b] = res[t];
                }
                for (long t = 0; t < len; ++t)
                    for (int b = 0; b < nb; ++b) data[base + t * stride + b] = tile[t * B + b];
            }
        }
    }
}

extern "C" {

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

// kernels.cuh -- sm_100a kernels of the RSFE Split-Bregman path, templated on the
// arithmetic type T (float or double).
//
// Reference routines restated here (paths relative to the reference project):
//   Gaussian filter      header/convolution_imp.hxx:22-91, :535-653
//   Heaviside            header/rsfe_splitbregman_imp.hxx:174-192
//   fitting terms + rhs  header/rsfe_splitbregman_imp.hxx:1700-1761
//   Gauss-Seidel         header/poisson_imp.hxx:23-336 (Neumann), :340-429 (Dirichlet)
//   clamp, tolerance     header/rsfe_splitbregman_imp.hxx:320-339, :1832
//   grad, div            header/image3d_imp.hxx:744-889, :948-1384
//   shrink, Bregman      header/rsfe_splitbregman_imp.hxx:343-365, :1868-1932
//   edge detector        header/rsfe_splitbregman_imp.hxx:196-316 (GRAD branch)
#pragma once

#include <type_traits>

#include "common.cuh"

namespace im3d {

constexpr int NH_MAX = 129;  // largest Gaussian support handled by the conv kernels

// ------------------------------------------------------------------ Heaviside
// H(x) = 1/2 (1 + 2/pi atan(x/eps)) and 1 - H(x) = H(-x), both to full relative
// precision: the smaller of the two is atan(1/|y|)/pi for |y| >= 1 (no cancellation
// against 1/2), the larger is 1 minus it. With eps = 1e-3 the smaller value reaches
// ~3e-4 and the fitting terms divide by its convolution, so FP32 needs this form.
template <typename T>
__device__ __forceinline__ void heaviside_pair(T phi, T center, T inv_eps, T& H, T& Hb)
{
    const T inv_pi = T(0.318309886183790671537767526745028724);
    const T x = (phi - center) * inv_eps;
    const T y = fabs(x);
    T small;
    if (y >= T(1)) small = atan(T(1) / y) * inv_pi;
    else small = T(0.5) - atan(y) * inv_pi;
    const T large = T(1) - small;
    if (x > T(0)) { H = large; Hb = small; }
    else { H = small; Hb = large; }
}

// ------------------------------------------------------------ loaders/storers
template <typename T, int N>
struct LdVec {
    const Vec<T, N>* p;
    Dims d;
    __device__ __forceinline__ Vec<T, N> operator()(int i, int j, int k) const
    {
        return p[d.idx(i, j, k)];
    }
};

template <typename T, int N>
struct StVec {
    Vec<T, N>* p;
    Dims d;
    __device__ __forceinline__ void operator()(int i, int j, int k, const Vec<T, N>& v) const
    {
        p[d.idx(i, j, k)] = v;
    }
};

template <typename T>
struct LdScalar {
    const T* p;
    Dims d;
    __device__ __forceinline__ Vec<T, 1> operator()(int i, int j, int k) const
    {
        Vec<T, 1> r;
        r.v[0] = ld_g(p + d.idx(i, j, k));
        return r;
    }
};

template <typename T>
struct LdOne {
    __device__ __forceinline__ Vec<T, 1> operator()(int, int, int) const
    {
        Vec<T, 1> r;
        r.v[0] = T(1);
        return r;
    }
};

template <typename T>
struct StScalar {
    T* p;
    Dims d;
    __device__ __forceinline__ void operator()(int i, int j, int k, const Vec<T, 1>& v) const
    {
        p[d.idx(i, j, k)] = v.v[0];
    }
};

// Stage-1 input: (H u0, H, Hb u0, Hb) from phi and u0.
template <typename T>
struct LdHeaviside {
    const T* phi;
    const T* u0;
    Dims d;
    T center, inv_eps;
    __device__ __forceinline__ Vec<T, 4> operator()(int i, int j, int k) const
    {
        const long long q = d.idx(i, j, k);
        T H, Hb;
        heaviside_pair(ld_g(phi + q), center, inv_eps, H, Hb);
        const T u = ld_g(u0 + q);
        Vec<T, 4> r;
        r.v[0] = H * u;
        r.v[1] = H;
        r.v[2] = Hb * u;
        r.v[3] = Hb;
        return r;
    }
};

// Forcing term of the Poisson step (rsfe_splitbregman_imp.hxx:1750-1761), from
// (kr2, kr1) = K * (l1 f1 - l2 f2, l1 f1^2 - l2 f2^2), in the reference's order:
//   r = kr2*u0*2 - (l1-l2)*u0*u0*kones - kr1, r /= lamda, r -= divdb.
// mode 0: natural rhs. mode 1: colour-packed rhs and colour-packed copy of phi.
// mode 2: colour-packed b_eff = rhs + phi/dt, packed phi, and sum b_eff^2.
// Dirichlet: the packed phi takes the boundary value on the faces.
template <typename T>
struct StRhs {
    const T* u0;
    const T* kones;  // NULL when lamda1 == lamda2 (the term is exactly zero)
    const T* divdb;
    const T* phi;
    T* out;      // natural rhs (mode 0) or packed rhs / b_eff (modes 1, 2)
    T* upk;      // packed phi (modes 1, 2)
    double* beff2;
    Dims d;
    T l12, lamda, inv_dt, bc;
    int mode, dirichlet;
    __device__ __forceinline__ void operator()(int i, int j, int k, const Vec<T, 2>& v) const
    {
        const long long q = d.idx(i, j, k);
        const T u = ld_g(u0 + q);
        T r = v.v[0];
        r *= u;
        r *= T(2);
        if (kones) {
            T a = l12;
            a *= u;
            a *= u;
            a *= ld_g(kones + q);
            r -= a;
        }
        r -= v.v[1];
        r /= lamda;
        r -= ld_g(divdb + q);
        if (mode == 0) {
            out[q] = r;
            return;
        }
        const int c = (i + j + k) & 1;
        const long long pq = d.pidx(i, j, k) + (c ? d.npk() : 0);
        T ph = ld_g(phi + q);
        const bool face = i == 0 || j == 0 || k == 0 || i == d.nx - 1 || j == d.ny - 1 ||
                          k == d.nz - 1;
        if (dirichlet && face) ph = bc;
        upk[pq] = ph;
        out[pq] = mode == 2 ? r + ph * inv_dt : r;
    }
};

// ------------------------------------------------------- separable convolution
// out = sum_t w[t] x[p + t - S], symmetric taps (w[t] == w[nh-1-t]), zero outside.
template <typename T, int N>
__device__ __forceinline__ Vec<T, N> tap_sum(const Vec<T, N>* x, int stride, const T* w, int nh)
{
    const int S = nh >> 1;
    Vec<T, N> acc;
#pragma unroll
    for (int q = 0; q < N; ++q) acc.v[q] = w[S] * x[S * stride].v[q];
    for (int t = 0; t < S; ++t) {
        const Vec<T, N> a = x[t * stride];
        const Vec<T, N> b = x[(nh - 1 - t) * stride];
#pragma unroll
        for (int q = 0; q < N; ++q) acc.v[q] = fma(w[t], a.v[q] + b.v[q], acc.v[q]);
    }
    return acc;
}

// Pass along k (contiguous). Block: TK threads along k x RK rows; grid.x over rows
// (i*ny + j), grid.y over k tiles. smem: RK x (TK + 2S) vectors + taps.
template <typename T, int N, int TK, int RK, class Ld, class St>
__global__ void __launch_bounds__(TK* RK) conv_k_kernel(Ld ld, St st, Dims d, const T* __restrict__ taps,
                                                      int nh)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int S = nh >> 1;
    const int W = TK + 2 * S;
    Vec<T, N>* sm = reinterpret_cast<Vec<T, N>*>(smem_raw);
    T* wsm = reinterpret_cast<T*>(sm + RK * W);
    const int tid = threadIdx.y * TK + threadIdx.x;
    for (int t = tid; t < nh; t += TK * RK) wsm[t] = taps[t];
    const long long row = (long long)blockIdx.x * RK + threadIdx.y;
    const bool live = row < (long long)d.nx * d.ny;
    const int i = live ? (int)(row / d.ny) : 0;
    const int j = live ? (int)(row % d.ny) : 0;
    const int k0 = blockIdx.y * TK;
    Vec<T, N>* srow = sm + threadIdx.y * W;
    for (int s = threadIdx.x; s < W; s += TK) {
        const int k = k0 - S + s;
        srow[s] = (live && k >= 0 && k < d.nz) ? ld(i, j, k) : vzero<T, N>();
    }
    __syncthreads();
    const int k = k0 + threadIdx.x;
    if (!live || k >= d.nz) return;
    st(i, j, k, tap_sum<T, N>(srow + threadIdx.x, 1, wsm, nh));
}

// Pass along j (AXIS 1) or i (AXIS 0). Block: TW threads along k x TY along the
// axis; tile TA outputs along the axis x TW along k. grid = (k tiles, axis tiles,
// the third coordinate). smem: (TA + 2S) x TW vectors + taps.
template <typename T, int N, int AXIS, int TW, int TY, int TA, class Ld, class St>
__global__ void __launch_bounds__(TW* TY) conv_s_kernel(Ld ld, St st, Dims d, const T* __restrict__ taps,
                                                      int nh)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int S = nh >> 1;
    const int H = TA + 2 * S;
    Vec<T, N>* sm = reinterpret_cast<Vec<T, N>*>(smem_raw);
    T* wsm = reinterpret_cast<T*>(sm + H * TW);
    const int tid = threadIdx.y * TW + threadIdx.x;
    for (int t = tid; t < nh; t += TW * TY) wsm[t] = taps[t];
    const int k = blockIdx.x * TW + threadIdx.x;
    const int a0 = blockIdx.y * TA;
    const int other = blockIdx.z;
    const int len = AXIS == 0 ? d.nx : d.ny;
    const bool kin = k < d.nz;
    for (int s = threadIdx.y; s < H; s += TY) {
        const int a = a0 - S + s;
        Vec<T, N> v = vzero<T, N>();
        if (kin && a >= 0 && a < len) v = AXIS == 0 ? ld(a, other, k) : ld(other, a, k);
        sm[s * TW + threadIdx.x] = v;
    }
    __syncthreads();
    if (!kin) return;
    for (int o = threadIdx.y; o < TA; o += TY) {
        const int a = a0 + o;
        if (a >= len) break;
        const Vec<T, N> r = tap_sum<T, N>(sm + o * TW + threadIdx.x, TW, wsm, nh);
        if (AXIS == 0) st(a, other, k, r);
        else st(other, a, k, r);
    }
}

// Fused i-axis stage: K_i applied to the four stage-1 fields (H u0, H, Hb u0, Hb)
// completes num, den, numb, denb; then f1 = num/den, f2 = numb/denb, the second
// pair (l1 f1 - l2 f2, l1 f1^2 - l2 f2^2) is formed and K_i is applied to it.
// The reference's f2 = (num - k*u0)/(den - k*1) equals numb/denb by linearity of
// the convolution (k*u0 - num = k*((1-H) u0), k*1 - den = k*(1-H)).
// Tile: TA outputs along i; the first pass covers TA + 2S rows (zero outside the
// volume, which is the zero boundary of the second convolution's input).
template <typename T, int TW, int TY, int TA>
__global__ void __launch_bounds__(TW* TY) conv_i_fit_kernel(const Vec<T, 4>* __restrict__ in,
                                                          Vec<T, 2>* __restrict__ out, T* f1_out,
                                                          T* f2_out, Dims d,
                                                          const T* __restrict__ taps, int nh,
                                                          T l1, T l2)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int S = nh >> 1;
    const int H1 = TA + 4 * S;  // input rows
    const int H2 = TA + 2 * S;  // rows of the second pass's input
    Vec<T, 4>* sin = reinterpret_cast<Vec<T, 4>*>(smem_raw);
    Vec<T, 2>* smid = reinterpret_cast<Vec<T, 2>*>(sin + H1 * TW);
    T* wsm = reinterpret_cast<T*>(smid + H2 * TW);
    const int tid = threadIdx.y * TW + threadIdx.x;
    for (int t = tid; t < nh; t += TW * TY) wsm[t] = taps[t];
    const int k = blockIdx.x * TW + threadIdx.x;
    const int i0 = blockIdx.y * TA;
    const int j = blockIdx.z;
    const bool kin = k < d.nz;
    for (int s = threadIdx.y; s < H1; s += TY) {
        const int i = i0 - 2 * S + s;
        Vec<T, 4> v = vzero<T, 4>();
        if (kin && i >= 0 && i < d.nx) v = in[d.idx(i, j, k)];
        sin[s * TW + threadIdx.x] = v;
    }
    __syncthreads();
    for (int s = threadIdx.y; s < H2; s += TY) {
        const int i = i0 - S + s;
        Vec<T, 2> m = vzero<T, 2>();
        if (kin && i >= 0 && i < d.nx) {
            const Vec<T, 4> c = tap_sum<T, 4>(sin + s * TW + threadIdx.x, TW, wsm, nh);
            const T f1 = c.v[0] / c.v[1];
            const T f2 = c.v[2] / c.v[3];
            m.v[0] = f1 * l1 - f2 * l2;
            m.v[1] = (f1 * f1) * l1 - (f2 * f2) * l2;
            if (f1_out && s >= S && s < S + TA) {
                const long long q = d.idx(i, j, k);
                f1_out[q] = f1;
                f2_out[q] = f2;
            }
        }
        smid[s * TW + threadIdx.x] = m;
    }
    __syncthreads();
    if (!kin) return;
    for (int o = threadIdx.y; o < TA; o += TY) {
        const int i = i0 + o;
        if (i >= d.nx) break;
        out[d.idx(i, j, k)] = tap_sum<T, 2>(smid + o * TW + threadIdx.x, TW, wsm, nh);
    }
}

// ------------------------------------------------------------------ stencils
// One component of image3d::grad at a point with position pos on an axis of length
// len (image3d_imp.hxx:762-838): central inside, one-sided second order on faces.
template <typename T>
__device__ __forceinline__ T grad_term(const T* f, long long p, long long stride, int pos,
                                       int len, double h)
{
    if (pos == 0)
        return (T(4) * f[p + stride] - T(3) * f[p] - f[p + 2 * stride]) / T(2. * h);
    if (pos == len - 1)
        return (T(3) * f[p] - T(4) * f[p - stride] + f[p - 2 * stride]) / T(2. * h);
    return (f[p + stride] - f[p - stride]) / T(2. * h);
}

template <typename T>
__global__ void grad_kernel(const T* __restrict__ f, T* __restrict__ g, Dims d, double hx,
                            double hy, double hz)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long p = d.idx(i, j, k);
    const long long n = d.n();
    g[p] = grad_term(f, p, (long long)d.ny * d.nz, i, d.nx, hx);
    g[n + p] = grad_term(f, p, (long long)d.nz, j, d.ny, hy);
    g[2 * n + p] = grad_term(f, p, 1, k, d.nz, hz);
}

// im3d::div at one point (image3d_imp.hxx:1060-1380) with the reference's two
// stencil quirks: on the face i = X-1 (j, k inside) the x term is
// ((3f - 4f + f)/2)*hx (:1091-1099), and on the edge j = 0, k = Z-1 (i inside) the
// z term reads Z-2 twice (:1203-1213).
template <typename T>
__device__ __forceinline__ T div_point(const T* f0, const T* f1, const T* f2, const Dims& d,
                                       int i, int j, int k, double hx, double hy, double hz)
{
    const long long p = d.idx(i, j, k);
    const long long sx = (long long)d.ny * d.nz, sy = d.nz;
    const int cx = i == 0 ? 0 : (i == d.nx - 1 ? 2 : 1);
    const int cy = j == 0 ? 0 : (j == d.ny - 1 ? 2 : 1);
    const int cz = k == 0 ? 0 : (k == d.nz - 1 ? 2 : 1);
    T tx, tz;
    if (cx == 2 && cy == 1 && cz == 1)
        tx = (T(3) * f0[p] - T(4) * f0[p - sx] + f0[p - 2 * sx]) / T(2.) * T(hx);
    else
        tx = grad_term(f0, p, sx, i, d.nx, hx);
    const T ty = grad_term(f1, p, sy, j, d.ny, hy);
    if (cx == 1 && cy == 0 && cz == 2)
        tz = (T(3) * f2[p] - T(4) * f2[p - 1] + f2[p - 1]) / T(2. * hz);
    else
        tz = grad_term(f2, p, 1, k, d.nz, hz);
    return tx + ty + tz;
}

template <typename T>
__global__ void div_kernel(const T* __restrict__ v, T* __restrict__ out, Dims d, double hx,
                           double hy, double hz)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long n = d.n();
    out[d.idx(i, j, k)] = div_point(v, v + n, v + 2 * n, d, i, j, k, hx, hy, hz);
}

// Edge detector, GRAD branch (rsfe_splitbregman_imp.hxx:220-232, 308-313):
// g = nu / (lamda (1 + beta |grad f|^2)), evaluated in the reference's order.
template <typename T>
__global__ void edge_kernel(const T* __restrict__ f, T* __restrict__ g, Dims d, double hx,
                            double hy, double hz, T beta, T lamda, T nu)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long p = d.idx(i, j, k);
    const T g0 = grad_term(f, p, (long long)d.ny * d.nz, i, d.nx, hx);
    const T g1 = grad_term(f, p, (long long)d.nz, j, d.ny, hy);
    const T g2 = grad_term(f, p, 1, k, d.nz, hz);
    T a = g0 * g0;
    a += g1 * g1;
    a += g2 * g2;
    a *= beta;
    a += T(1);
    T r = T(1);
    r /= a;
    r /= lamda;
    r *= nu;
    g[p] = r;
}

// Clamped level-set value at a point, read from the natural or the packed layout.
template <typename T, bool PACKED>
__device__ __forceinline__ T phi_at(const T* u, const Dims& d, int i, int j, int k, T a0, T b0)
{
    T v;
    if (PACKED) v = u[d.pidx(i, j, k) + (((i + j + k) & 1) ? d.npk() : 0)];
    else v = u[d.idx(i, j, k)];
    if (v < a0) v = a0;
    else if (v > b0) v = b0;
    return v;
}

template <typename T, bool PACKED>
__device__ __forceinline__ T grad_phi(const T* u, const Dims& d, int i, int j, int k, int axis,
                                      double h, T a0, T b0)
{
    const int len = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
    const int pos = axis == 0 ? i : (axis == 1 ? j : k);
    auto at = [&](int o) {
        return axis == 0 ? phi_at<T, PACKED>(u, d, i + o, j, k, a0, b0)
                         : (axis == 1 ? phi_at<T, PACKED>(u, d, i, j + o, k, a0, b0)
                                      : phi_at<T, PACKED>(u, d, i, j, k + o, a0, b0));
    };
    if (pos == 0) return (T(4) * at(1) - T(3) * at(0) - at(2)) / T(2. * h);
    if (pos == len - 1) return (T(3) * at(0) - T(4) * at(-1) + at(-2)) / T(2. * h);
    return (at(1) - at(-1)) / T(2. * h);
}

// After the Poisson step: cut_phi (clamp to [a0, b0]), the tolerance sums
// sum (phi - phiold)^2 and sum phiold^2, and -- unless bregman == 0 -- the
// Split-Bregman update per component c (rsfe_splitbregman_imp.hxx:1868-1906):
//   d = grad(phi)_c; b += d; d = shrink(b, g); b -= d; d -= b
// The new d (= d_new - b_new) goes to dmb for the divergence kernel.
// `phi` holds phiold on entry and the clamped phi on exit (each thread reads and
// writes only its own point there); the neighbours come from u.
template <typename T, bool PACKED>
__global__ void post_solve_kernel(const T* __restrict__ u, T* phi, T* __restrict__ u_out,
                                  T* __restrict__ b3, T* __restrict__ dmb,
                                  const T* __restrict__ g, Dims d, double hx, double hy,
                                  double hz, T a0, T b0, int bregman, double* sums)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    double s_d = 0, s_o = 0;
    if (k < d.nz && j < d.ny) {
        const long long p = d.idx(i, j, k);
        T uv;
        if (PACKED) uv = u[d.pidx(i, j, k) + (((i + j + k) & 1) ? d.npk() : 0)];
        else uv = u[p];
        if (u_out) u_out[p] = uv;
        T v = uv;
        if (v < a0) v = a0;
        else if (v > b0) v = b0;
        const T old = phi[p];
        phi[p] = v;
        const double df = (double)v - (double)old;
        s_d = df * df;
        s_o = (double)old * (double)old;
        if (bregman) {
            const long long n = d.n();
            const T gg = g[p];
            const double hs[3] = {hx, hy, hz};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T dc = grad_phi<T, PACKED>(u, d, i, j, k, c, hs[c], a0, b0);
                T bb = b3[c * n + p];
                bb += dc;
                const T m = fabs(bb) - gg;
                const T sgn = T((int)(bb > T(0)) - (int)(bb < T(0)));
                const T dn = sgn * ((m < T(0)) ? T(0) : m);
                bb -= dn;
                b3[c * n + p] = bb;
                dmb[c * n + p] = dn - bb;
            }
        }
    }
    block_sum2_atomic(s_d, s_o, sums + SUM_DPHI2, sums + SUM_PHIOLD2);
}

// ------------------------------------------------------------- Gauss-Seidel
template <typename T>
struct GsCoef {
    // exact reference form (double): divisions by h*h and dt
    double hx, hy, hz, dt;
    // reciprocal form (float)
    T ihx2, ihy2, ihz2, idt;
    T htilde[8];   // indexed by (cx inside) | (cy inside) << 1 | (cz inside) << 2
    T bcn[4];      // bc scaled by the oblique normal for 1, 2, 3 boundary axes
    double bcnd[4];
    T bc;
    int neu;
};

// One Gauss-Seidel point value (sum of neighbour terms + b + self/dt) * htilde;
// `self_dt` is self/dt (beff mode folds u_in/dt into b and passes 0).
// r(o_i, o_j, o_k) returns the current value of a neighbour.
template <typename T, class R>
__device__ __forceinline__ T gs_value(const GsCoef<T>& c, const Dims& d, int i, int j, int k,
                                      T b, T self, bool use_self, R r)
{
    if (!c.neu) {
        const T sx = r(1, 0, 0) + r(-1, 0, 0);
        const T sy = r(0, 1, 0) + r(0, -1, 0);
        const T sz = r(0, 0, 1) + r(0, 0, -1);
        if (std::is_same<T, double>::value) {
            double acc = sx / (c.hx * c.hx) + sy / (c.hy * c.hy) + sz / (c.hz * c.hz) + b;
            if (use_self) acc = acc + self / c.dt;
            return T(acc * (double)c.htilde[7]);
        } else {
            T acc = sx * c.ihx2 + sy * c.ihy2 + sz * c.ihz2 + b;
            if (use_self) acc += self * c.idt;
            return acc * c.htilde[7];
        }
    }
    const int cx = i == 0 ? 0 : (i == d.nx - 1 ? 2 : 1);
    const int cy = j == 0 ? 0 : (j == d.ny - 1 ? 2 : 1);
    const int cz = k == 0 ? 0 : (k == d.nz - 1 ? 2 : 1);
    const int nb = (cx != 1) + (cy != 1) + (cz != 1);
    const T bcn = c.bcn[nb];
    T tx, ty, tz;
    if (std::is_same<T, double>::value) {
        const double hx = c.hx, hy = c.hy, hz = c.hz;
        tx = cx == 1 ? (r(1, 0, 0) + r(-1, 0, 0)) / (hx * hx)
                     : (cx == 0 ? (r(1, 0, 0) - bcn * hx) / (hx * hx) : (r(-1, 0, 0) + bcn * hx) / (hx * hx));
        ty = cy == 1 ? (r(0, 1, 0) + r(0, -1, 0)) / (hy * hy)
                     : (cy == 0 ? (r(0, 1, 0) - bcn * hy) / (hy * hy) : (r(0, -1, 0) + bcn * hy) / (hy * hy));
        tz = cz == 1 ? (r(0, 0, 1) + r(0, 0, -1)) / (hz * hz)
                     : (cz == 0 ? (r(0, 0, 1) - bcn * hz) / (hz * hz) : (r(0, 0, -1) + bcn * hz) / (hz * hz));
        double acc = (double)tx + ty + tz + b;
        if (use_self) acc = acc + self / c.dt;
        return T(acc * (double)c.htilde[(cx == 1) | ((cy == 1) << 1) | ((cz == 1) << 2)]);
    } else {
        const T hx = T(c.hx), hy = T(c.hy), hz = T(c.hz);
        tx = (cx == 1 ? r(1, 0, 0) + r(-1, 0, 0)
                      : (cx == 0 ? r(1, 0, 0) - bcn * hx : r(-1, 0, 0) + bcn * hx)) * c.ihx2;
        ty = (cy == 1 ? r(0, 1, 0) + r(0, -1, 0)
                      : (cy == 0 ? r(0, 1, 0) - bcn * hy : r(0, -1, 0) + bcn * hy)) * c.ihy2;
        tz = (cz == 1 ? r(0, 0, 1) + r(0, 0, -1)
                      : (cz == 0 ? r(0, 0, 1) - bcn * hz : r(0, 0, -1) + bcn * hz)) * c.ihz2;
        T acc = tx + ty + tz + b;
        if (use_self) acc += self * c.idt;
        return acc * c.htilde[(cx == 1) | ((cy == 1) << 1) | ((cz == 1) << 2)];
    }
}

template <typename T>
__device__ __forceinline__ T gs_htilde(const GsCoef<T>& c, const Dims& d, int i, int j, int k)
{
    if (!c.neu) return c.htilde[7];
    const int ix = !(i == 0 || i == d.nx - 1), iy = !(j == 0 || j == d.ny - 1),
              iz = !(k == 0 || k == d.nz - 1);
    return c.htilde[ix | (iy << 1) | (iz << 2)];
}

// Lexicographic sweep as a hyperplane wavefront: all unknowns with i+j+k = s are
// independent given planes s-1 (already updated) and s+1 (not yet), which is exactly
// the new/old split every point sees in the reference's i, j, k (Dir) or k, j, i (Neu)
// loop. One launch per hyperplane; threads cover (i, j) and derive k = s - i - j.
template <typename T>
__global__ void lex_plane_kernel(T* __restrict__ r, const T* __restrict__ b, Dims d, GsCoef<T> c,
                                 int s, int lo, int i_begin, int j_begin)
{
    const int j = j_begin + blockIdx.x * blockDim.x + threadIdx.x;
    const int i = i_begin + blockIdx.y * blockDim.y + threadIdx.y;
    const int hix = d.nx - lo, hiy = d.ny - lo, hiz = d.nz - lo;
    if (i >= hix || j >= hiy) return;
    const int k = s - i - j;
    if (k < lo || k >= hiz) return;
    const long long p = d.idx(i, j, k);
    auto rd = [&](int oi, int oj, int ok) { return r[d.idx(i + oi, j + oj, k + ok)]; };
    r[p] = gs_value<T>(c, d, i, j, k, b[p], r[p], true, rd);
}

// Dirichlet boundary assignment of DirGaussSeidel (poisson_imp.hxx:366-391).
template <typename T>
__global__ void dir_faces_kernel(T* r, Dims d, T bc)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    if (i == 0 || j == 0 || k == 0 || i == d.nx - 1 || j == d.ny - 1 || k == d.nz - 1)
        r[d.idx(i, j, k)] = bc;
}

// Red-black half sweep on the colour-packed layout: updates colour `color`, reading
// the other colour. Thread per packed (m, j, i). Modes:
//   use_self = 1: reference sweep formula (b + self/dt), b packed rhs;
//   use_self = 0: fixed u_in, b = b_eff packed; omega != 1 over-relaxes.
template <typename T>
__global__ void rb_half_kernel(T* __restrict__ U, const T* __restrict__ B, Dims d, GsCoef<T> c,
                               int color, int use_self, T omega)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= d.ny) return;
    const int k = 2 * m + ((i + j + color) & 1);
    if (k >= d.nz) return;
    const int lo = c.neu ? 0 : 1;
    if (i < lo || j < lo || k < lo || i >= d.nx - lo || j >= d.ny - lo || k >= d.nz - lo) return;
    const long long npk = d.npk();
    T* own = U + (color ? npk : 0);
    const T* oth = U + (color ? 0 : npk);
    const long long pq = d.pidx(i, j, k);
    auto rd = [&](int oi, int oj, int ok) { return oth[d.pidx(i + oi, j + oj, k + ok)]; };
    const T self = (use_self || omega != T(1)) ? own[pq] : T(0);
    T v = gs_value<T>(c, d, i, j, k, B[(color ? npk : 0) + pq], self, use_self != 0, rd);
    if (omega != T(1)) v = self + omega * (v - self);
    own[pq] = v;
}

// FP64 residual of one unknown of (1/dt - Lap) u = b_eff:
//   r = sum of neighbour terms + b_eff - diag * u,  diag = 1/dt + sum_a c_a/h_a^2
// with c_a = 2 inside and 1 on a Neumann face (the same rows the sweep solves).
template <typename T, class R>
__device__ __forceinline__ double gs_residual_fp64(const GsCoef<T>& c, const Dims& d, int i,
                                                   int j, int k, double b, double u, R r)
{
    const double ihx2 = 1.0 / (c.hx * c.hx), ihy2 = 1.0 / (c.hy * c.hy),
                 ihz2 = 1.0 / (c.hz * c.hz);
    if (!c.neu) {
        const double sx = r(1, 0, 0) + r(-1, 0, 0);
        const double sy = r(0, 1, 0) + r(0, -1, 0);
        const double sz = r(0, 0, 1) + r(0, 0, -1);
        const double diag = 1.0 / c.dt + 2.0 * ihx2 + 2.0 * ihy2 + 2.0 * ihz2;
        return sx * ihx2 + sy * ihy2 + sz * ihz2 + b - diag * u;
    }
    const int cx = i == 0 ? 0 : (i == d.nx - 1 ? 2 : 1);
    const int cy = j == 0 ? 0 : (j == d.ny - 1 ? 2 : 1);
    const int cz = k == 0 ? 0 : (k == d.nz - 1 ? 2 : 1);
    const int nb = (cx != 1) + (cy != 1) + (cz != 1);
    const double bcn = c.bcnd[nb];
    const double tx = cx == 1 ? r(1, 0, 0) + r(-1, 0, 0)
                              : (cx == 0 ? r(1, 0, 0) - bcn * c.hx : r(-1, 0, 0) + bcn * c.hx);
    const double ty = cy == 1 ? r(0, 1, 0) + r(0, -1, 0)
                              : (cy == 0 ? r(0, 1, 0) - bcn * c.hy : r(0, -1, 0) + bcn * c.hy);
    const double tz = cz == 1 ? r(0, 0, 1) + r(0, 0, -1)
                              : (cz == 0 ? r(0, 0, 1) - bcn * c.hz : r(0, 0, -1) + bcn * c.hz);
    const double diag = 1.0 / c.dt + (cx == 1 ? 2.0 : 1.0) * ihx2 + (cy == 1 ? 2.0 : 1.0) * ihy2 +
                        (cz == 1 ? 2.0 : 1.0) * ihz2;
    return tx * ihx2 + ty * ihy2 + tz * ihz2 + b - diag * u;
}

// Residual of (1/dt - Lap) u = b_eff on the packed layout over the unknowns,
// accumulated as sum r^2 in FP64 (values read in T, arithmetic in FP64).
template <typename T>
__global__ void rb_residual_kernel(const T* __restrict__ U, const T* __restrict__ B, Dims d,
                                   GsCoef<T> c, double* sums, int want_beff)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    double acc = 0, accb = 0;
    const int lo = c.neu ? 0 : 1;
    const long long npk = d.npk();
    if (j < d.ny) {
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            const int k = 2 * m + ((i + j + color) & 1);
            if (k >= d.nz) continue;
            if (i < lo || j < lo || k < lo || i >= d.nx - lo || j >= d.ny - lo || k >= d.nz - lo)
                continue;
            const T* own = U + (color ? npk : 0);
            const T* oth = U + (color ? 0 : npk);
            const long long pq = d.pidx(i, j, k);
            auto rd = [&](int oi, int oj, int ok) {
                return (double)oth[d.pidx(i + oi, j + oj, k + ok)];
            };
            const double bv = (double)B[(color ? npk : 0) + pq];
            const double r = gs_residual_fp64<T>(c, d, i, j, k, bv, (double)own[pq], rd);
            acc += r * r;
            accb += bv * bv;
        }
    }
    if (want_beff) block_sum2_atomic(acc, accb, sums + SUM_RES2, sums + SUM_BEFF2);
    else block_sum_atomic(acc, sums + SUM_RES2);
}

// sum (a - b)^2 and sum b^2 over n elements (relative change of a sweep)
template <typename T>
__global__ void diff_sums_kernel(const T* __restrict__ a, const T* __restrict__ b, long long n,
                                 double* sums)
{
    double sd = 0, sb = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const double x = (double)a[q] - (double)b[q];
        sd += x * x;
        sb += (double)b[q] * (double)b[q];
    }
    block_sum2_atomic(sd, sb, sums + SUM_A, sums + SUM_B);
}

// natural -> packed copy of a volume (both colours), and back
template <typename T>
__global__ void pack_kernel(const T* __restrict__ src, T* __restrict__ dst, Dims d)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    dst[d.pidx(i, j, k) + (((i + j + k) & 1) ? d.npk() : 0)] = src[d.idx(i, j, k)];
}

template <typename T>
__global__ void unpack_kernel(const T* __restrict__ src, T* __restrict__ dst, Dims d)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    dst[d.idx(i, j, k)] = src[d.pidx(i, j, k) + (((i + j + k) & 1) ? d.npk() : 0)];
}

// packed b_eff = b + u/dt (u packed), with sum b_eff^2; Dirichlet faces of u := bc
template <typename T>
__global__ void make_beff_kernel(const T* __restrict__ b, T* __restrict__ U, T* __restrict__ Beff,
                                 Dims d, T inv_dt, T bc, int dirichlet, double* sums)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    double acc = 0;
    if (k < d.nz && j < d.ny) {
        const long long pq = d.pidx(i, j, k) + (((i + j + k) & 1) ? d.npk() : 0);
        const bool face = i == 0 || j == 0 || k == 0 || i == d.nx - 1 || j == d.ny - 1 ||
                          k == d.nz - 1;
        T u = U[pq];
        if (dirichlet && face) {
            u = bc;
            U[pq] = u;
        }
        const T e = b[d.idx(i, j, k)] + u * inv_dt;
        Beff[pq] = e;
        if (!(dirichlet && face)) acc = (double)e * (double)e;
    }
    block_sum_atomic(acc, sums + SUM_BEFF2);
}

// ------------------------------------------------------------------ utilities
template <typename T>
__global__ void fill_kernel(T* p, long long n, T v)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
        p[q] = v;
}

// min / max of a volume as order-preserving unsigned keys (umax[0] = max, umax[1] = max of -x)
__device__ __forceinline__ unsigned long long order_key(double x)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

template <typename T>
__global__ void minmax_kernel(const T* __restrict__ p, long long n, unsigned long long* umax)
{
    unsigned long long mx = 0, mn = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const double v = (double)p[q];
        const unsigned long long a = order_key(v), b = order_key(-v);
        mx = a > mx ? a : mx;
        mn = b > mn ? b : mn;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, mx, o);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, mn, o);
        mx = a > mx ? a : mx;
        mn = b > mn ? b : mn;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(umax + 0, mx);
        atomicMax(umax + 1, mn);
    }
}

// change_range_of_intensity(max, min) (image3d_imp.hxx:1628-1636) once the minimum
// mn and the shifted maximum are known: x -= mn; x /= s; x += lo
template <typename T>
__global__ void affine_kernel(T* p, long long n, T mn, T s, T lo)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        T x = p[q];
        x -= mn;
        x /= s;
        x += lo;
        p[q] = x;
    }
}

// initialize_phi_with_cube (rsfe_splitbregman_imp.hxx:48-95): a0 outside the box
// [ix, fx) x [iy, fy) x [iz, fz), b0 inside
template <typename T>
__global__ void cube_kernel(T* p, Dims d, int ix, int iy, int iz, int fx, int fy, int fz, T a0,
                            T b0)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const bool in = i >= ix && i < fx && j >= iy && j < fy && k >= iz && k < fz;
    p[d.idx(i, j, k)] = in ? b0 : a0;
}

}  // namespace im3d

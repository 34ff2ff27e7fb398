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
    // one arctangent, of 1/y or y, and selects instead of branches
    const bool big = y >= T(1);
    T arg = y;
    if (big) {
        if constexpr (sizeof(T) == 4) arg = __frcp_rn(y);  // = 1.0f / y, correctly rounded
        else arg = T(1) / y;
    }
    const T at = atan(arg);
    const T small = big ? at * inv_pi : T(0.5) - at * inv_pi;
    const T large = T(1) - small;
    if (x > T(0)) { H = large; Hb = small; }
    else { H = small; Hb = large; }
}

// ------------------------------------------------------------ loaders/storers
// A loader's raw() issues the memory reads of one cell and cook() turns them into the
// staged fields, so that a pass can issue the reads of all its cells before it
// computes any of them; operator() does both.
template <typename T, int N>
struct LdVec {
    const Vec<T, N>* p;
    Dims d;
    typedef Vec<T, N> Raw;
    __device__ __forceinline__ Raw raw(int i, int j, int k) const { return p[d.idx(i, j, k)]; }
    __device__ __forceinline__ Vec<T, N> cook(const Raw& r) const { return r; }
    __device__ __forceinline__ Vec<T, N> operator()(int i, int j, int k) const
    {
        return p[d.idx(i, j, k)];
    }
};

// A storer's pre() issues the reads that its store of cells k0 .. k0+cnt-1 of one row
// needs, early in a pass, and put4() stores those cells; operator() stores one cell.
template <typename T, int N>
struct StVec {
    Vec<T, N>* p;
    Dims d;
    struct Pre {};
    __device__ __forceinline__ Pre pre(int, int, int, int) const { return Pre{}; }
    __device__ __forceinline__ void put4(const Pre&, int i, int j, int k0, const Vec<T, N> (&v)[4],
                                         int cnt) const
    {
        const long long q = d.idx(i, j, k0);
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r < cnt) p[q + r] = v[r];
    }
    __device__ __forceinline__ void operator()(int i, int j, int k, const Vec<T, N>& v) const
    {
        p[d.idx(i, j, k)] = v;
    }
};

template <typename T>
struct LdScalar {
    const T* p;
    Dims d;
    typedef Vec<T, 1> Raw;
    __device__ __forceinline__ Raw raw(int i, int j, int k) const { return (*this)(i, j, k); }
    __device__ __forceinline__ Vec<T, 1> cook(const Raw& r) const { return r; }
    __device__ __forceinline__ Vec<T, 1> operator()(int i, int j, int k) const
    {
        Vec<T, 1> r;
        r.v[0] = ld_g(p + d.idx(i, j, k));
        return r;
    }
};

template <typename T>
struct LdOne {
    typedef Vec<T, 1> Raw;
    __device__ __forceinline__ Raw raw(int i, int j, int k) const { return (*this)(i, j, k); }
    __device__ __forceinline__ Vec<T, 1> cook(const Raw& r) const { return r; }
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
    struct Pre {};
    __device__ __forceinline__ Pre pre(int, int, int, int) const { return Pre{}; }
    __device__ __forceinline__ void put4(const Pre&, int i, int j, int k0, const Vec<T, 1> (&v)[4],
                                         int cnt) const
    {
        const long long q = d.idx(i, j, k0);
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r < cnt) p[q + r] = v[r].v[0];
    }
    __device__ __forceinline__ void operator()(int i, int j, int k, const Vec<T, 1>& v) const
    {
        p[d.idx(i, j, k)] = v.v[0];
    }
};

// four consecutive values from p (16-byte vector reads when they are aligned), zero
// past cnt
template <typename T>
__device__ __forceinline__ void ld4(const T* __restrict__ p, int cnt, T (&o)[4])
{
    if (cnt == 4 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        if constexpr (sizeof(T) == 4) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(p));
            o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
        } else {
            const double2 a = __ldg(reinterpret_cast<const double2*>(p));
            const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
            o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
        }
    } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) o[r] = r < cnt ? ld_g(p + r) : T(0);
    }
}

// two values to p and p+1: one vector store when aligned
template <typename T>
__device__ __forceinline__ void st2(T* p, T a, T b)
{
    if ((reinterpret_cast<uintptr_t>(p) & (2 * sizeof(T) - 1)) == 0) {
        Vec<T, 2> v;
        v.v[0] = a;
        v.v[1] = b;
        *reinterpret_cast<Vec<T, 2>*>(p) = v;
    } else {
        p[0] = a;
        p[1] = b;
    }
}

// Stage-1 input: (H u0, H, Hb u0, Hb) from phi and u0.
template <typename T>
struct LdHeaviside {
    const T* phi;
    const T* u0;
    Dims d;
    T center, inv_eps;
    struct Raw {
        T phi, u;
    };
    __device__ __forceinline__ Raw raw(int i, int j, int k) const
    {
        const long long q = d.idx(i, j, k);
        return Raw{ld_g(phi + q), ld_g(u0 + q)};
    }
    __device__ __forceinline__ Vec<T, 4> cook(const Raw& w) const
    {
        T H, Hb;
        heaviside_pair(w.phi, center, inv_eps, H, Hb);
        Vec<T, 4> r;
        r.v[0] = H * w.u;
        r.v[1] = H;
        r.v[2] = Hb * w.u;
        r.v[3] = Hb;
        return r;
    }
    __device__ __forceinline__ Vec<T, 4> operator()(int i, int j, int k) const { return cook(raw(i, j, k)); }
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
    T inv_lamda;  // FP32 multiplies by it instead of dividing (same value when lamda is a power of two)
    int mode, dirichlet;
    struct Pre {
        T u[4], kn[4], dv[4], ph[4];
    };
    __device__ __forceinline__ Pre pre(int i, int j, int k0, int cnt) const
    {
        Pre w;
        const long long q = d.idx(i, j, k0);
        ld4(u0 + q, cnt, w.u);
        if (kones) ld4(kones + q, cnt, w.kn);
        ld4(divdb + q, cnt, w.dv);
        if (mode != 0) ld4(phi + q, cnt, w.ph);
        return w;
    }
    // the forcing term of one cell, operations as in operator()
    __device__ __forceinline__ T force(const Pre& w, int r, const Vec<T, 2>& v) const
    {
        const T u = w.u[r];
        T f = v.v[0];
        f *= u;
        f *= T(2);
        if (kones) {
            T a = l12;
            a *= u;
            a *= u;
            a *= w.kn[r];
            f -= a;
        }
        f -= v.v[1];
        if constexpr (sizeof(T) == 4) f *= inv_lamda;
        else f /= lamda;
        f -= w.dv[r];
        return f;
    }
    // k0 is even: cells k0, k0+2 have the colour of k0 and packed slots k0/2, k0/2+1,
    // cells k0+1, k0+3 the other colour and the same two slots
    __device__ __forceinline__ void put4(const Pre& w, int i, int j, int k0, const Vec<T, 2> (&v)[4],
                                         int cnt) const
    {
        T f[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) f[r] = force(w, r, v[r]);
        if (mode == 0) {
            T* o = out + d.idx(i, j, k0);
            if (cnt == 4) {
                st2(o, f[0], f[1]);
                st2(o + 2, f[2], f[3]);
            } else {
#pragma unroll
                for (int r = 0; r < 4; ++r)
                    if (r < cnt) o[r] = f[r];
            }
            return;
        }
        const bool face_ij = i == 0 || j == 0 || i == d.nx - 1 || j == d.ny - 1;
        T ph[4], val[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            ph[r] = w.ph[r];
            if (dirichlet && (face_ij || k0 + r == 0 || k0 + r == d.nz - 1)) ph[r] = bc;
            val[r] = mode == 2 ? f[r] + ph[r] * inv_dt : f[r];
        }
        const int c0 = (i + j + k0) & 1;
        const long long base = d.pidx(i, j, k0);
        const long long o0 = base + (c0 ? d.npk() : 0), o1 = base + (c0 ? 0 : d.npk());
        if (cnt == 4) {
            st2(upk + o0, ph[0], ph[2]);
            st2(upk + o1, ph[1], ph[3]);
            st2(out + o0, val[0], val[2]);
            st2(out + o1, val[1], val[3]);
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (r < cnt) {
                    const long long o = ((r & 1) ? o1 : o0) + (r >> 1);
                    upk[o] = ph[r];
                    out[o] = val[r];
                }
            }
        }
    }
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
        if constexpr (sizeof(T) == 4) r *= inv_lamda;
        else r /= lamda;
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

// ------------------------------------------------------------------- cp.async
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
// 16 bytes, or 16 zero bytes when !valid (nothing is read from gmem then)
__device__ __forceinline__ void cp_async16_zfill(void* smem, const void* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

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
        int kk = 0;
        srow[s] = (live && d.halo(k0 - S + s, d.nz, kk)) ? ld(i, j, kk) : vzero<T, N>();
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
        int a = 0;
        Vec<T, N> v = vzero<T, N>();
        if (kin && d.halo(a0 - S + s, len, a)) v = AXIS == 0 ? ld(a, other, k) : ld(other, a, k);
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

// ---- register-window passes for a compile-time half width S (taps 2S+1) ----
// Each thread computes R consecutive outputs along the convolution axis from a
// register window of R + 2S inputs, with the taps in registers and the inputs in
// shared memory as one plane per field; this reads each staged input (R+2S)/R times
// instead of 2S+1 times.
template <typename T, int S, int R>
__device__ __forceinline__ void window_conv(const T (&x)[R + 2 * S], const T (&w)[S + 1],
                                            T (&out)[R])
{
#pragma unroll
    for (int r = 0; r < R; ++r) {
        T acc = w[S] * x[r + S];
#pragma unroll
        for (int t = 0; t < S; ++t) acc = fma(w[t], x[r + t] + x[r + 2 * S - t], acc);
        out[r] = acc;
    }
}

template <typename T, int S>
__device__ __forceinline__ void load_taps(const T* __restrict__ taps, T (&w)[S + 1])
{
#pragma unroll
    for (int t = 0; t <= S; ++t) w[t] = __ldg(taps + t);
}

// Along k (contiguous). Block TKT x RKR threads; each thread R = 4 RG consecutive k of
// one row (RG groups of 4 for the storer); tile RKR rows x R*TKT k. The halo is rounded
// up to SP = 4*ceil(S/4) so that every thread's window starts 16-byte aligned and is
// read with vector loads. Larger RG reads fewer window values per output from shared
// memory and recomputes fewer halo cells; every output is the same sum either way.
template <typename T, int N, int S, int TKT, int RKR, class Ld, class St, int RG = 1>
__device__ __forceinline__ void conv_k_win_body(const uint3 blockIdx, const dim3 gridDim, Ld ld, St st, Dims d,
                                                const T* __restrict__ taps)
{
    constexpr int R = 4 * RG;
    constexpr int TK = TKT * R;
    constexpr int SP = (S + 3) & ~3;
    constexpr int W = TK + 2 * SP;
    constexpr int XW = R + 2 * SP;  // window read by one thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);  // [N][RKR][W]
    const long long row = (long long)blockIdx.x * RKR + threadIdx.y;
    const bool live = row < (long long)d.nx * d.ny;
    const int i = live ? (int)(row / d.ny) : 0;
    const int j = live ? (int)(row % d.ny) : 0;
    const int k0 = blockIdx.y * TK;
    const int kk = k0 + threadIdx.x * R;  // this thread's first output cell (even)
    typename St::Pre pre[RG]{};
    {
        constexpr int NL = (W + TKT - 1) / TKT;
        // all reads first, then the loader's arithmetic (the Heaviside for stage 1)
        typename Ld::Raw rw[NL];
        bool ok[NL];
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int s = threadIdx.x + u * TKT;
            int k = 0;
            ok[u] = s < W && live && d.halo(k0 - SP + s, d.nz, k);
            if (ok[u]) rw[u] = ld.raw(i, j, k);
        }
        // the storer's own reads (the forcing term's fields) go out with them
#pragma unroll
        for (int g = 0; g < RG; ++g)
            if (kk + 4 * g < d.nz && live) pre[g] = st.pre(i, j, kk + 4 * g, min(4, d.nz - kk - 4 * g));
        Vec<T, N> v[NL];
#pragma unroll
        for (int u = 0; u < NL; ++u) v[u] = ok[u] ? ld.cook(rw[u]) : vzero<T, N>();
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int s = threadIdx.x + u * TKT;
            if (s < W) {
#pragma unroll
                for (int q = 0; q < N; ++q) sm[(q * RKR + threadIdx.y) * W + s] = v[u].v[q];
            }
        }
    }
    T w[S + 1];
    load_taps<T, S>(taps, w);
    __syncthreads();
    const bool act = live && kk < d.nz;
    T res[N][R];
    if (act) {
#pragma unroll
        for (int q = 0; q < N; ++q) {
            const T* base = sm + (q * RKR + threadIdx.y) * W + threadIdx.x * R;
            T xa[XW];
            if (sizeof(T) == 4) {
#pragma unroll
                for (int t = 0; t < XW; t += 4) {
                    const float4 v4 = *reinterpret_cast<const float4*>(base + t);
                    xa[t] = v4.x; xa[t + 1] = v4.y; xa[t + 2] = v4.z; xa[t + 3] = v4.w;
                }
            } else {
#pragma unroll
                for (int t = 0; t < XW; t += 2) {
                    const double2 v2 = *reinterpret_cast<const double2*>(base + t);
                    xa[t] = v2.x; xa[t + 1] = v2.y;
                }
            }
            T x[R + 2 * S];
#pragma unroll
            for (int t = 0; t < R + 2 * S; ++t) x[t] = xa[t + SP - S];
            window_conv<T, S, R>(x, w, res[q]);
        }
    }
    if (!act) return;
#pragma unroll
    for (int g = 0; g < RG; ++g) {
        const int kg = kk + 4 * g;
        if (kg >= d.nz) break;
        Vec<T, N> vo[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#pragma unroll
            for (int q = 0; q < N; ++q) vo[r].v[q] = res[q][4 * g + r];
        }
        st.put4(pre[g], i, j, kg, vo, min(4, d.nz - kg));
    }
}

template <typename T, int N, int S, int TKT, int RKR, class Ld, class St, int RG = 1>
__global__ void __launch_bounds__(TKT* RKR) conv_k_win_kernel(Ld ld, St st, Dims d, const T* __restrict__ taps)
{
    conv_k_win_body<T, N, S, TKT, RKR, Ld, St, RG>(blockIdx, gridDim, ld, st, d, taps);
}

// FP32 passes of four fields convolve them in pairs (float2 in shared memory,
// __fadd2_rn / __ffma2_rn / __fmul2_rn): per component the operations of window_conv,
// so the sums are bit-identical. They run as conv_s_win_pair_kernel, held to 3 blocks
// per SM (80 registers, a few bytes spilled). Measured against the scalar form, same
// box: 4 fields 133 -> 117 us at 256^3 and 760 -> 602 us at 512x512x320; 2 fields
// 82 -> 74 and 442 -> 496 us, so the 2-field pass stays scalar.
template <typename T, int N>
constexpr bool kPairedS = sizeof(T) == 4 && N == 4;

// Along j (AXIS 1) or i (AXIS 0). Block TW x TY; each thread R consecutive outputs
// along the axis in one k column; tile TY*R along the axis x TW along k.
template <typename T, int N, int AXIS, int S, int TW, int TY, int R, class Ld, class St>
__device__ __forceinline__ void conv_s_win_body(const uint3 blockIdx, const dim3 gridDim, Ld ld, St st, Dims d, const T* __restrict__ taps)
{
    constexpr int TA = TY * R;
    constexpr int H = TA + 2 * S;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);  // [N][H][TW]
    const int k = blockIdx.x * TW + threadIdx.x;
    const int a0 = blockIdx.y * TA;
    const int other = blockIdx.z;
    const int len = AXIS == 0 ? d.nx : d.ny;
    const bool kin = k < d.nz;
    {
        constexpr int NL = (H + TY - 1) / TY;
        Vec<T, N> v[NL];
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int s = threadIdx.y + u * TY;
            int a = 0;
            v[u] = vzero<T, N>();
            if (s < H && kin && d.halo(a0 - S + s, len, a)) v[u] = AXIS == 0 ? ld(a, other, k) : ld(other, a, k);
        }
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int s = threadIdx.y + u * TY;
            if (s < H) {
                if constexpr (kPairedS<T, N>) {
                    // FP32 fields in pairs, [N/2][H][TW] of float2
#pragma unroll
                    for (int q = 0; q < N / 2; ++q)
                        reinterpret_cast<float2*>(sm)[(q * H + s) * TW + threadIdx.x] =
                            make_float2(v[u].v[2 * q], v[u].v[2 * q + 1]);
                } else {
#pragma unroll
                    for (int q = 0; q < N; ++q) sm[(q * H + s) * TW + threadIdx.x] = v[u].v[q];
                }
            }
        }
    }
    T w[S + 1];
    load_taps<T, S>(taps, w);
    __syncthreads();
    if (!kin) return;
    const int r0 = threadIdx.y * R;
    Vec<T, N> out[R];
    if constexpr (kPairedS<T, N>) {
        // window_conv of two fields at once with the paired FP32 instructions of sm_100:
        // per component the same operations, half the instructions and loads
        float2 w2[S + 1];
#pragma unroll
        for (int t = 0; t <= S; ++t) w2[t] = make_float2(w[t], w[t]);
#pragma unroll
        for (int q = 0; q < N / 2; ++q) {
            float2 x[R + 2 * S];
#pragma unroll
            for (int t = 0; t < R + 2 * S; ++t)
                x[t] = reinterpret_cast<const float2*>(sm)[(q * H + r0 + t) * TW + threadIdx.x];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                float2 acc = __fmul2_rn(w2[S], x[r + S]);
#pragma unroll
                for (int t = 0; t < S; ++t) acc = __ffma2_rn(w2[t], __fadd2_rn(x[r + t], x[r + 2 * S - t]), acc);
                out[r].v[2 * q] = acc.x;
                out[r].v[2 * q + 1] = acc.y;
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < N; ++q) {
            T x[R + 2 * S];
#pragma unroll
            for (int t = 0; t < R + 2 * S; ++t) x[t] = sm[(q * H + r0 + t) * TW + threadIdx.x];
            T o[R];
            window_conv<T, S, R>(x, w, o);
#pragma unroll
            for (int r = 0; r < R; ++r) out[r].v[q] = o[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int a = a0 + r0 + r;
        if (a < len) {
            if (AXIS == 0) st(a, other, k, out[r]);
            else st(other, a, k, out[r]);
        }
    }
}

template <typename T, int N, int AXIS, int S, int TW, int TY, int R, class Ld, class St>
__global__ void __launch_bounds__(TW* TY) conv_s_win_kernel(Ld ld, St st, Dims d, const T* __restrict__ taps)
{
    conv_s_win_body<T, N, AXIS, S, TW, TY, R, Ld, St>(blockIdx, gridDim, ld, st, d, taps);
}

// the paired form (kPairedS), held to 3 blocks per SM
template <typename T, int N, int AXIS, int S, int TW, int TY, int R, class Ld, class St>
__global__ void __launch_bounds__(TW* TY, 3) conv_s_win_pair_kernel(Ld ld, St st, Dims d, const T* __restrict__ taps)
{
    conv_s_win_body<T, N, AXIS, S, TW, TY, R, Ld, St>(blockIdx, gridDim, ld, st, d, taps);
}

// Fused i-axis stage with register windows (see conv_i_fit_kernel for the maths).
// First pass: RA = ceil((TA+2S)/TY) rows per thread over the four fields; second
// pass: RB = TA/TY rows per thread over the pair.
template <typename T, int S, int TW, int TY, int TA>
__device__ __forceinline__ void conv_i_fit_win_body(const uint3 blockIdx, const dim3 gridDim, const Vec<T, 4>* __restrict__ in, Vec<T, 2>* __restrict__ out, T* f1_out, T* f2_out, Dims d, const T* __restrict__ taps, T l1, T l2)
{
    constexpr int RA = (TA + 2 * S + TY - 1) / TY;
    constexpr int RB = TA / TY;
    constexpr int H2 = TY * RA;          // rows of the first pass's output (>= TA + 2S)
    constexpr int H1 = H2 + 2 * S;       // input rows
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sin = reinterpret_cast<T*>(smem_raw);   // [4][H1][TW]
    T* smid = sin + 4 * H1 * TW;               // [2][H2][TW]
    const int k = blockIdx.x * TW + threadIdx.x;
    const int i0 = blockIdx.y * TA;
    const int j = blockIdx.z;
    const bool kin = k < d.nz;
    {
        constexpr int NL = (H1 + TY - 1) / TY;
        Vec<T, 4> v[NL];
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int s = threadIdx.y + u * TY;
            int i = 0;
            v[u] = vzero<T, 4>();
            if (s < H1 && kin && d.halo(i0 - 2 * S + s, d.nx, i)) v[u] = in[d.idx(i, j, k)];
        }
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int s = threadIdx.y + u * TY;
            if (s < H1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) sin[(q * H1 + s) * TW + threadIdx.x] = v[u].v[q];
            }
        }
    }
    T w[S + 1];
    load_taps<T, S>(taps, w);
    __syncthreads();
    {
        const int r0 = threadIdx.y * RA;
        T c[4][RA];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            T x[RA + 2 * S];
#pragma unroll
            for (int t = 0; t < RA + 2 * S; ++t) x[t] = sin[(q * H1 + r0 + t) * TW + threadIdx.x];
            window_conv<T, S, RA>(x, w, c[q]);
        }
#pragma unroll
        for (int r = 0; r < RA; ++r) {
            const int s = r0 + r;           // first-pass row: i = i0 - S + s
            const int i = i0 - S + s;
            T pv = T(0), qv = T(0);
            // rows outside the volume are zero for the second convolution, or the
            // rows they wrap to for the periodic boundary
            const bool inside = i >= 0 && i < d.nx;
            if (kin && (inside || d.cyc)) {
                const T f1 = c[0][r] / c[1][r];
                const T f2 = c[2][r] / c[3][r];
                pv = f1 * l1 - f2 * l2;
                qv = (f1 * f1) * l1 - (f2 * f2) * l2;
                if (f1_out && inside && s >= S && s < S + TA) {
                    const long long qq = d.idx(i, j, k);
                    f1_out[qq] = f1;
                    f2_out[qq] = f2;
                }
            }
            smid[(0 * H2 + s) * TW + threadIdx.x] = pv;
            smid[(1 * H2 + s) * TW + threadIdx.x] = qv;
        }
    }
    __syncthreads();
    if (!kin) return;
    const int r0 = threadIdx.y * RB;
    T o[2][RB];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        T x[RB + 2 * S];
#pragma unroll
        for (int t = 0; t < RB + 2 * S; ++t) x[t] = smid[(q * H2 + r0 + t) * TW + threadIdx.x];
        window_conv<T, S, RB>(x, w, o[q]);
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        const int i = i0 + r0 + r;
        if (i < d.nx) {
            Vec<T, 2> v;
            v.v[0] = o[0][r];
            v.v[1] = o[1][r];
            out[d.idx(i, j, k)] = v;
        }
    }
}

template <typename T, int S, int TW, int TY, int TA>
__global__ void __launch_bounds__(TW* TY) conv_i_fit_win_kernel(const Vec<T, 4>* __restrict__ in, Vec<T, 2>* __restrict__ out, T* f1_out, T* f2_out, Dims d, const T* __restrict__ taps, T l1, T l2)
{
    conv_i_fit_win_body<T, S, TW, TY, TA>(blockIdx, gridDim, in, out, f1_out, f2_out, d, taps, l1, l2);
}

// One step of a running convolution along a march axis, on float pairs with the
// packed f32x2 pipes. acc[u] holds the partial sum of row p - S + u, where p is the
// plane being added: acc[u] <- acc[u+1] + w[u] x for u = 0 .. 2S-1 (w symmetric,
// w[u] = w[2S-u]) and acc[2S] <- w[0] x. After the step acc[0] is complete: its row
// has received w[t] x[row - S + t] for t = 0 .. 2S, in plane order. Every update
// reads a slot before the one it writes, so the window shifts with no moves and the
// 2S+1 updates of a step are independent.
template <int S>
__device__ __forceinline__ void shift_conv2(float2 (&acc)[2 * S + 1], const float2 (&w)[S + 1], float2 x)
{
#pragma unroll
    for (int u = 0; u < 2 * S; ++u) acc[u] = __ffma2_rn(w[u <= S ? u : 2 * S - u], x, acc[u + 1]);
    acc[2 * S] = __fmul2_rn(w[0], x);
}

// cp.async.wait_group with a count known only after unrolling (0 .. 15)
__device__ __forceinline__ void cp_async_wait_n(int n)
{
    switch (n) {
    case 0: cp_async_wait<0>(); break;
    case 1: cp_async_wait<1>(); break;
    case 2: cp_async_wait<2>(); break;
    case 3: cp_async_wait<3>(); break;
    case 4: cp_async_wait<4>(); break;
    case 5: cp_async_wait<5>(); break;
    case 6: cp_async_wait<6>(); break;
    case 7: cp_async_wait<7>(); break;
    case 8: cp_async_wait<8>(); break;
    case 9: cp_async_wait<9>(); break;
    case 10: cp_async_wait<10>(); break;
    case 11: cp_async_wait<11>(); break;
    case 12: cp_async_wait<12>(); break;
    case 13: cp_async_wait<13>(); break;
    case 14: cp_async_wait<14>(); break;
    default: cp_async_wait<15>(); break;
    }
}

// taps w[0] .. w[S] of a symmetric kernel, each as a float pair (w, w), passed by value
// so that the kernel reads them from the parameter bank
template <int S>
struct TapPairs {
    float2 w[S + 1];
};

// Fused i-axis stage, marching form (FP32): the maths of conv_i_fit_kernel with no
// recomputed rows. Block: 32 threads along k x JB along j, one (j, k) column per
// thread; blockIdx.z picks a chunk of `chunk` output rows along i. A thread streams
// the input planes p = i0-2S .. i1+2S-1 of its column: each 16-byte cell goes through
// a D-plane ring in shared memory by cp.async (zero filled outside the volume,
// wrapped for the periodic boundary) and is added into the accumulators of the first
// convolution (the four fields as two f32x2 pairs). Row m = p - S of that convolution
// is then complete: (num, den, numb, denb) give f1, f2 and the pair
// (l1 f1 - l2 f2, l1 f1^2 - l2 f2^2) (zero outside the volume unless periodic), which
// is added into the accumulators of the second convolution, completing its output
// row m - S. The march takes U planes per round: one barrier per round orders the
// reads of the previous round's ring slots before they are refilled, and the U steps
// between barriers overlap one plane's division and fit with the next plane's
// accumulation. Rounding differs from the tiled kernels by summation order only: each
// row adds its 2S+1 products in plane order, where the tiled kernels add symmetric
// pairs first; f1 and f2 use the fast division (within 2 ulp).
template <int S, int JB, int D, int U, int MINB>
__device__ __forceinline__ void conv_i_fit_march_body(const uint3 blockIdx, const dim3 gridDim, const float4* __restrict__ in, float2* __restrict__ out, float* f1_out, float* f2_out, Dims d, const TapPairs<S> tp, float l1, float l2, int chunk)
{
    constexpr int L = 2 * S + 1;
    static_assert((D & (D - 1)) == 0 && D >= 2 * U && D <= 16, "ring: a power of two, >= 2U");
    __shared__ __align__(16) float4 ring[D][JB][32];
    const int k = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * JB + threadIdx.y;
    const int i0 = blockIdx.z * chunk;
    const int i1 = min(i0 + chunk, d.nx);
    const bool col = k < d.nz && j < d.ny;
    const int pa = i0 - 2 * S;
    const int np = (i1 - i0) + 4 * S;
    const long long cq = (long long)j * d.nz + k;        // this column in plane 0
    const long long ps = (long long)d.ny * d.nz;         // plane stride
    float4* const mine = &ring[0][threadIdx.y][threadIdx.x];
    constexpr int SLOT = JB * 32;  // float4s between ring slots
    auto issue = [&](int n) {
        int i = 0;
        const bool ok = col && n < np && d.halo(pa + n, d.nx, i);
        const float4* src = ok ? in + (i * ps + cq) : in;
        cp_async16_zfill(mine + (n & (D - 1)) * SLOT, src, ok);
        cp_async_commit();
    };
    // planes 0 .. D-U-1 ahead of the first round
#pragma unroll
    for (int n = 0; n < D - U; ++n) issue(n);
    const float2 (&w2)[S + 1] = tp.w;
    // rows before the first one needed collect contributions and are never read
    float2 a0[L], a1[L], bq[L];
#pragma unroll
    for (int t = 0; t < L; ++t) a0[t] = a1[t] = bq[t] = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int n0 = 0; n0 < np; n0 += U) {
#pragma unroll
        for (int q = 0; q < U; ++q) {
            const int n = n0 + q;
            // groups issued: planes 0 .. n0+D-U-1; plane n is complete when at most
            // D-U-1-q of them are pending
            cp_async_wait_n(D - U - 1 - q);
            if (n < np) {
                const float4 x = mine[(n & (D - 1)) * SLOT];
                shift_conv2<S>(a0, w2, make_float2(x.x, x.y));
                shift_conv2<S>(a1, w2, make_float2(x.z, x.w));
                if (n >= 2 * S) {
                    // row m = p - S of the first convolution is complete
                    const int m = pa + n - S;
                    const bool inside = m >= 0 && m < d.nx;
                    float pv = 0.f, qv = 0.f;
                    if (col && (inside || d.cyc)) {
                        const float f1 = __fdividef(a0[0].x, a0[0].y);
                        const float f2 = __fdividef(a1[0].x, a1[0].y);
                        pv = f1 * l1 - f2 * l2;
                        qv = (f1 * f1) * l1 - (f2 * f2) * l2;
                        if (f1_out && inside && m >= i0 && m < i1) {
                            const long long qq = m * ps + cq;
                            f1_out[qq] = f1;
                            f2_out[qq] = f2;
                        }
                    }
                    // output row m - S is complete
                    shift_conv2<S>(bq, w2, make_float2(pv, qv));
                    if (n >= 4 * S && col) out[(m - S) * ps + cq] = bq[0];
                }
            }
        }
        // every thread has read this round's slots before the next rounds refill them
        __syncthreads();
#pragma unroll
        for (int q = 0; q < U; ++q) issue(n0 + D - U + q);
    }
    cp_async_wait<0>();
}

template <int S, int JB, int D, int U, int MINB>
__global__ void __launch_bounds__(32 * JB, MINB) conv_i_fit_march_kernel(const float4* __restrict__ in, float2* __restrict__ out, float* f1_out, float* f2_out, Dims d, const TapPairs<S> tp, float l1, float l2, int chunk)
{
    conv_i_fit_march_body<S, JB, D, U, MINB>(blockIdx, gridDim, in, out, f1_out, f2_out, d, tp, l1, l2, chunk);
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
        int i = 0;
        Vec<T, 4> v = vzero<T, 4>();
        if (kin && d.halo(i0 - 2 * S + s, d.nx, i)) v = in[d.idx(i, j, k)];
        sin[s * TW + threadIdx.x] = v;
    }
    __syncthreads();
    for (int s = threadIdx.y; s < H2; s += TY) {
        const int i = i0 - S + s;
        Vec<T, 2> m = vzero<T, 2>();
        const bool inside = i >= 0 && i < d.nx;
        if (kin && (inside || d.cyc)) {
            const Vec<T, 4> c = tap_sum<T, 4>(sin + s * TW + threadIdx.x, TW, wsm, nh);
            const T f1 = c.v[0] / c.v[1];
            const T f2 = c.v[2] / c.v[3];
            m.v[0] = f1 * l1 - f2 * l2;
            m.v[1] = (f1 * f1) * l1 - (f2 * f2) * l2;
            if (f1_out && inside && s >= S && s < S + TA) {
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
// x / (2h) of the difference stencils: FP64 divides, with the reference's operations;
// FP32 multiplies by the reciprocal, which gives the same value when 2h is a power of
// two (unit spacing) and is within 1 ulp of it otherwise, at a fraction of a
// division's instructions.
template <typename T>
__device__ __forceinline__ T over_two_h(T x, T two_h, T inv_two_h)
{
    if constexpr (sizeof(T) == 4) return x * inv_two_h;
    else return x / two_h;
}

// One component of image3d::grad at a point with position pos on an axis of length
// len (image3d_imp.hxx:762-838): central inside, one-sided second order on faces.
template <typename T>
__device__ __forceinline__ T grad_term(const T* f, long long p, long long stride, int pos,
                                       int len, double h)
{
    // FP32 multiplies by 1/(2h) as the vectorised kernels do (over_two_h); FP64 divides
    const T two_h = T(2. * h), inv_two_h = T(1. / (2. * h));
    if (pos == 0)
        return over_two_h(T(4) * f[p + stride] - T(3) * f[p] - f[p + 2 * stride], two_h, inv_two_h);
    if (pos == len - 1)
        return over_two_h(T(3) * f[p] - T(4) * f[p - stride] + f[p - 2 * stride], two_h, inv_two_h);
    return over_two_h(f[p + stride] - f[p - stride], two_h, inv_two_h);
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
__device__ __forceinline__ void div_body(const uint3 blockIdx, const dim3 gridDim, const T* __restrict__ v, T* __restrict__ out, Dims d, double hx, double hy, double hz)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long n = d.n();
    out[d.idx(i, j, k)] = div_point(v, v + n, v + 2 * n, d, i, j, k, hx, hy, hz);
}

template <typename T>
__global__ void div_kernel(const T* __restrict__ v, T* __restrict__ out, Dims d, double hx, double hy, double hz)
{
    div_body<T>(blockIdx, gridDim, v, out, d, hx, hy, hz);
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

// ------------------------------------------------------------- Gauss-Seidel
template <typename T>
struct GsCoef {
    // exact reference form (double): divisions by h*h and dt
    double hx, hy, hz, dt;
    // reciprocal form (float)
    T ihx2, ihy2, ihz2, idt;
    T htilde[8];   // indexed by (cx inside) | (cy inside) << 1 | (cz inside) << 2
    // FP32: the rounding of each reciprocal, htilde_lo = 1/ht - htilde. The update
    // fma(acc, htilde, acc * htilde_lo) multiplies by 1/ht to within the final
    // rounding; acc * htilde alone would scale every update by the same relative
    // error (-2.6e-8 for 1/7), a bias of the operator that the outer iterations
    // accumulate. Unused (zero) in FP64, which keeps the reference's form.
    T htilde_lo[8];
    T bcn[4];      // bc scaled by the oblique normal for 1, 2, 3 boundary axes
    double bcnd[4];
    T bc;
    int neu;
    // FP64 forms for the residual: 1/h^2 and the diagonal 1/dt + 2/hx^2 + 2/hy^2 + 2/hz^2
    double ihx2d, ihy2d, ihz2d, diagd;
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
            return fma(acc, c.htilde[7], acc * c.htilde_lo[7]);
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
        const int m = (cx == 1) | ((cy == 1) << 1) | ((cz == 1) << 2);
        return fma(acc, c.htilde[m], acc * c.htilde_lo[m]);
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

// FP64 residual of one unknown of (1/dt - Lap) u = b_eff:
//   r = sum of neighbour terms + b_eff - diag * u,  diag = 1/dt + sum_a c_a/h_a^2
// with c_a = 2 inside and 1 on a Neumann face (the same rows the sweep solves).
template <typename T, class R>
__device__ __forceinline__ double gs_residual_fp64(const GsCoef<T>& c, const Dims& d, int i,
                                                   int j, int k, double b, double u, R r)
{
    if (!c.neu) {
        const double sx = r(1, 0, 0) + r(-1, 0, 0);
        const double sy = r(0, 1, 0) + r(0, -1, 0);
        const double sz = r(0, 0, 1) + r(0, 0, -1);
        return sx * c.ihx2d + sy * c.ihy2d + sz * c.ihz2d + b - c.diagd * u;
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
    const double diag = 1.0 / c.dt + (cx == 1 ? 2.0 : 1.0) * c.ihx2d + (cy == 1 ? 2.0 : 1.0) * c.ihy2d +
                        (cz == 1 ? 2.0 : 1.0) * c.ihz2d;
    return tx * c.ihx2d + ty * c.ihy2d + tz * c.ihz2d + b - diag * u;
}


// The (vector group g, row j) pairs of a block of planes, flattened over the grid's x
// blocks, so that no lane idles when a row's `groups` are not a multiple of blockDim.x
// (40 groups at nz = 320 left 24 of every 64 lanes idle). A power-of-two number of
// groups (nz = 256) takes shifts instead of the division.
__device__ __forceinline__ void flat_pair(const uint3 blockIdx, unsigned groups, int& g, int& j)
{
    const unsigned lin = (blockIdx.x * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    if ((groups & (groups - 1)) == 0) {
        g = (int)(lin & (groups - 1));
        j = (int)(lin >> (__ffs((int)groups) - 1));
    } else {
        g = (int)(lin % groups);
        j = (int)(lin / groups);
    }
}

// Vectorised red-black half sweep: one thread per group of W = 16/sizeof(T)
// consecutive packed points (m0 .. m0+W-1) of row j, marching over NI planes of i.
// All points of a packed row share the parity of k, so their k neighbours are the
// other colour at (m-1, m) (k even) or (m, m+1) (k odd): one 16-byte vector plus one
// scalar. The i neighbours come from a register window of vectors along i.
// SELF: the point's own old value is read (use_self or omega != 1); the Poisson solve
// on b_eff needs neither. NEU: the Neumann boundary rule is compiled in (c.neu must
// match). Without both the kernel needs fewer registers and fits MINB blocks per SM.
// reverse: the blocks take the planes of i from the last to the first, so that a
// half-sweep following one in the other direction starts on the planes that are still
// in L2. IX: the type of the cell offsets, int where both colours' cells number less
// than 2^31 (fewer instructions per address), else long long.
template <typename T, int NI, bool SELF = true, bool NEU = true, int MINB = 1, typename IX = long long>
__device__ __forceinline__ void rb_half_vec_body(const uint3 blockIdx, const dim3 gridDim, T* __restrict__ U, const T* __restrict__ B, Dims d, GsCoef<T> c, int color, int use_self, T omega, int reverse)
{
    typedef V16<T> VT;
    typedef typename VT::type VV;
    constexpr int W = VT::W;
    // Launched as a programmatic dependent of the previous half-sweep: wait until its
    // writes are visible, then let the next half-sweep's blocks be scheduled while this
    // one drains (both are no-ops in an ordinary launch).
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    int g, j;
    flat_pair(blockIdx, (unsigned)(d.hz() / W), g, j);
    const int i0 = (reverse ? gridDim.z - 1 - blockIdx.z : blockIdx.z) * NI;
    const int hz = d.hz();
    const int m0 = g * W;
    if (m0 >= hz || j >= d.ny) return;
    const IX plane = (IX)d.ny * hz;
    const IX npk = plane * d.nx;
    T* own = U + (color ? npk : 0);
    const T* oth = U + (color ? 0 : npk);
    const T* bb = B + (color ? npk : 0);
    const bool jint = j >= 1 && j <= d.ny - 2;
    const IX q0 = ((IX)i0 * d.ny + j) * hz + m0;
    const bool relax = SELF && omega != T(1);
    if (!SELF) use_self = 0;
    // Every load of the NI planes is issued before the first store: the stores go to
    // the same array, so loads placed after one could not be moved ahead of it and each
    // thread would pay one memory round trip per plane.
    VV o[NI + 2], ymv[NI], ypv[NI], bvv[NI], sfv[NI];
    T exv[NI];
#pragma unroll
    for (int t = 0; t < NI + 2; ++t) {
        const int i = i0 - 1 + t;
        if (i >= 0 && i < d.nx) o[t] = *reinterpret_cast<const VV*>(oth + q0 + (IX)(t - 1) * plane);
        else o[t] = VV{};
    }
#pragma unroll
    for (int t = 0; t < NI; ++t) {
        const int i = i0 + t;
        const IX q = q0 + (IX)t * plane;
        const int par = (i + j + color) & 1;
        ymv[t] = ypv[t] = bvv[t] = sfv[t] = VV{};
        exv[t] = T(0);
        if (jint && i >= 1 && i <= d.nx - 2) {
            ymv[t] = *reinterpret_cast<const VV*>(oth + q - hz);
            ypv[t] = *reinterpret_cast<const VV*>(oth + q + hz);
            bvv[t] = *reinterpret_cast<const VV*>(bb + q);
            // the k neighbour not in the centre vector: m0-1 (k even) or m0+W (k odd)
            const bool e_ok = par ? (m0 + W < hz) : (m0 >= 1);
            if (e_ok) exv[t] = oth[par ? q + W : q - 1];
            if (SELF && (use_self || relax)) sfv[t] = *reinterpret_cast<const VV*>(own + q);
        }
    }
#pragma unroll
    for (int t = 0; t < NI; ++t) {
        const int i = i0 + t;
        if (i >= d.nx) break;
        const IX q = q0 + (IX)t * plane;
        const int par = (i + j + color) & 1;
        const bool rowint = jint && i >= 1 && i <= d.nx - 2;
        if (rowint) {
            const VV ym = ymv[t];
            const VV yp = ypv[t];
            const VV bv = bvv[t];
            const T extra = exv[t];
            const VV self = sfv[t];
            VV outv = self;
            bool all = true;
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
                const int k = 2 * (m0 + cc) + par;
                const bool in = k >= 1 && k <= d.nz - 2;
                if (!in) {
                    all = false;
                    continue;
                }
                const T ctr = VT::get(o[t + 1], cc);
                const T kn = par ? (cc + 1 < W ? VT::get(o[t + 1], cc + 1) : extra)
                                 : (cc >= 1 ? VT::get(o[t + 1], cc - 1) : extra);
                const T sz = ctr + kn;
                const T sy = VT::get(ym, cc) + VT::get(yp, cc);
                const T sx = VT::get(o[t], cc) + VT::get(o[t + 2], cc);
                const T b = VT::get(bv, cc);
                const T sf = VT::get(self, cc);
                T v;
                if (std::is_same<T, double>::value) {
                    double acc = sx / (c.hx * c.hx) + sy / (c.hy * c.hy) + sz / (c.hz * c.hz) + b;
                    if (use_self) acc = acc + sf / c.dt;
                    v = T(acc * (double)c.htilde[7]);
                } else {
                    T acc = fma(sx, c.ihx2, fma(sy, c.ihy2, fma(sz, c.ihz2, b)));
                    if (use_self) acc = fma(sf, c.idt, acc);
                    v = fma(acc, c.htilde[7], acc * c.htilde_lo[7]);
                }
                if (relax) v = sf + omega * (v - sf);
                VT::set(outv, cc, v);
            }
            if (all) {
                *reinterpret_cast<VV*>(own + q) = outv;
            } else {
#pragma unroll
                for (int cc = 0; cc < W; ++cc) {
                    const int k = 2 * (m0 + cc) + par;
                    if (k >= 1 && k <= d.nz - 2) own[q + cc] = VT::get(outv, cc);
                }
            }
        }
        if (NEU && c.neu) {
            // Neumann: boundary points (faces of i, j or k) through the generic rule
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
                const int k = 2 * (m0 + cc) + par;
                if (k >= d.nz) continue;
                if (rowint && k >= 1 && k <= d.nz - 2) continue;
                auto rd = [&](int oi, int oj, int ok) { return oth[d.pidx(i + oi, j + oj, k + ok)]; };
                const T sf = own[q + cc];
                T v = gs_value<T>(c, d, i, j, k, bb[q + cc], sf, use_self != 0, rd);
                if (relax) v = sf + omega * (v - sf);
                own[q + cc] = v;
            }
        }
    }
}

template <typename T, int NI, bool SELF = true, bool NEU = true, int MINB = 1, typename IX = long long>
__global__ void __launch_bounds__(128, MINB) rb_half_vec_kernel(T* __restrict__ U, const T* __restrict__ B, Dims d, GsCoef<T> c, int color, int use_self, T omega, int reverse = 0)
{
    rb_half_vec_body<T, NI, SELF, NEU, MINB, IX>(blockIdx, gridDim, U, B, d, c, color, use_self, omega, reverse);
}

// Vectorised FP64 residual, same walk as rb_half_vec_kernel; blockIdx.z covers
// (plane block, colour).
template <typename T, int NI, typename IX = long long>
__device__ __forceinline__ void rb_residual_vec_body(const uint3 blockIdx, const dim3 gridDim, const T* __restrict__ U, const T* __restrict__ B, Dims d, GsCoef<T> c, double* part, int want_beff)
{
    typedef V16<T> VT;
    typedef typename VT::type VV;
    constexpr int W = VT::W;
    int g, j;
    flat_pair(blockIdx, (unsigned)(d.hz() / W), g, j);
    const int color = blockIdx.z & 1;
    const int i0 = (blockIdx.z >> 1) * NI;
    const int hz = d.hz();
    const int m0 = g * W;
    double acc = 0, accb = 0;
    if (m0 < hz && j < d.ny) {
        const IX plane = (IX)d.ny * hz;
        const IX npk = plane * d.nx;
        const T* own = U + (color ? npk : 0);
        const T* oth = U + (color ? 0 : npk);
        const T* bb = B + (color ? npk : 0);
        const bool jint = j >= 1 && j <= d.ny - 2;
        const int lo = c.neu ? 0 : 1;
        const IX q0 = ((IX)i0 * d.ny + j) * hz + m0;
        VV o[NI + 2];
#pragma unroll
        for (int t = 0; t < NI + 2; ++t) {
            const int i = i0 - 1 + t;
            if (i >= 0 && i < d.nx) o[t] = *reinterpret_cast<const VV*>(oth + q0 + (IX)(t - 1) * plane);
            else o[t] = VV{};
        }
#pragma unroll
        for (int t = 0; t < NI; ++t) {
            const int i = i0 + t;
            if (i >= d.nx) break;
            const IX q = q0 + (IX)t * plane;
            const int par = (i + j + color) & 1;
            const bool rowint = jint && i >= 1 && i <= d.nx - 2;
            const VV bv = *reinterpret_cast<const VV*>(bb + q);
            const VV uv = *reinterpret_cast<const VV*>(own + q);
            if (rowint) {
                const VV ym = *reinterpret_cast<const VV*>(oth + q - hz);
                const VV yp = *reinterpret_cast<const VV*>(oth + q + hz);
                const IX qe = par ? q + W : q - 1;
                const bool e_ok = par ? (m0 + W < hz) : (m0 >= 1);
                const double extra = e_ok ? (double)oth[qe] : 0.0;
#pragma unroll
                for (int cc = 0; cc < W; ++cc) {
                    const int k = 2 * (m0 + cc) + par;
                    if (!(k >= 1 && k <= d.nz - 2)) continue;
                    const double ctr = (double)VT::get(o[t + 1], cc);
                    const double kn = par ? (cc + 1 < W ? (double)VT::get(o[t + 1], cc + 1) : extra)
                                          : (cc >= 1 ? (double)VT::get(o[t + 1], cc - 1) : extra);
                    const double b = (double)VT::get(bv, cc);
                    const double r = ((double)VT::get(o[t], cc) + (double)VT::get(o[t + 2], cc)) * c.ihx2d +
                                     ((double)VT::get(ym, cc) + (double)VT::get(yp, cc)) * c.ihy2d +
                                     (ctr + kn) * c.ihz2d + b - c.diagd * (double)VT::get(uv, cc);
                    acc += r * r;
                    accb += b * b;
                }
            }
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
                const int k = 2 * (m0 + cc) + par;
                if (k >= d.nz) continue;
                if (rowint && k >= 1 && k <= d.nz - 2) continue;
                if (!(i >= lo && j >= lo && k >= lo && i < d.nx - lo && j < d.ny - lo && k < d.nz - lo))
                    continue;
                auto rd = [&](int oi, int oj, int ok) {
                    return (double)oth[d.pidx(i + oi, j + oj, k + ok)];
                };
                const double b = (double)VT::get(bv, cc);
                const double r = gs_residual_fp64<T>(c, d, i, j, k, b, (double)VT::get(uv, cc), rd);
                acc += r * r;
                accb += b * b;
            }
        }
    }
    if (want_beff) block_sum2_store(acc, accb, part, block_linear_id(blockIdx, gridDim), grid_blocks(gridDim));
    else block_sum_store(acc, part, block_linear_id(blockIdx, gridDim));
}

template <typename T, int NI, typename IX = long long>
__global__ void __launch_bounds__(256, 4) rb_residual_vec_kernel(const T* __restrict__ U, const T* __restrict__ B, Dims d, GsCoef<T> c, double* part, int want_beff)
{
    rb_residual_vec_body<T, NI, IX>(blockIdx, gridDim, U, B, d, c, part, want_beff);
}


// cut_phi (rsfe_splitbregman_imp.hxx:320-339) and the tolerance sums of :1832:
// phi holds phiold on entry and the clamped solve result on exit (natural layout);
// u is the solve result (packed or natural); u_out, when given, receives it unclamped.
template <typename T, bool PACKED, int NI>
__device__ __forceinline__ void clamp_tol_body(const uint3 blockIdx, const dim3 gridDim, const T* __restrict__ u, T* phi, T* __restrict__ u_out, Dims d, T a0, T b0, double* part)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i0 = blockIdx.z * NI;
    double s_d = 0, s_o = 0;
    if (k < d.nz && j < d.ny) {
        const int cnt = min(NI, d.nx - i0);
        const long long plane = (long long)d.ny * d.nz;
        const long long pplane = (long long)d.ny * d.hz();
        const long long p0 = d.idx(i0, j, k);
        const long long pq0 = d.pidx(i0, j, k);
        const long long npk = pplane * d.nx;
        // every load of the NI planes before the first store: a store to phi would
        // otherwise hold the next plane's loads back (one memory round trip per plane)
        T uv[NI], ov[NI];
#pragma unroll
        for (int t = 0; t < NI; ++t) {
            if (t < cnt) {
                const long long p = p0 + t * plane;
                uv[t] = PACKED ? u[pq0 + t * pplane + (((i0 + t + j + k) & 1) ? npk : 0)] : u[p];
                ov[t] = phi[p];
            }
        }
#pragma unroll
        for (int t = 0; t < NI; ++t) {
            if (t < cnt) {
                const long long p = p0 + t * plane;
                if (u_out) u_out[p] = uv[t];
                T v = uv[t];
                if (v < a0) v = a0;
                else if (v > b0) v = b0;
                const T old = ov[t];
                phi[p] = v;
                const double df = (double)v - (double)old;
                s_d += df * df;
                s_o += (double)old * (double)old;
            }
        }
    }
    block_sum2_store(s_d, s_o, part, block_linear_id(blockIdx, gridDim), grid_blocks(gridDim));
}

template <typename T, bool PACKED, int NI>
__global__ void __launch_bounds__(256) clamp_tol_kernel(const T* __restrict__ u, T* phi, T* __restrict__ u_out, Dims d, T a0, T b0, double* part)
{
    clamp_tol_body<T, PACKED, NI>(blockIdx, gridDim, u, phi, u_out, d, a0, b0, part);
}

// The Split-Bregman update on the clamped phi (rsfe_splitbregman_imp.hxx:1868-1906),
// per component c: d = grad(phi)_c; b += d; d = shrink(b, g); b -= d; d -= b.
// Thread per (k, j) column marching over NI planes with phi(i-1), phi(i), phi(i+1)
// in registers; j and k neighbours come through L1.
template <typename T, int NI>
__device__ __forceinline__ void bregman_body(const uint3 blockIdx, const dim3 gridDim, const T* __restrict__ phi, T* __restrict__ b3, T* __restrict__ dmb, const T* __restrict__ g, Dims d, double hx, double hy, double hz)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i0 = blockIdx.z * NI;
    if (k >= d.nz || j >= d.ny) return;
    const int cnt = min(NI, d.nx - i0);
    const long long plane = (long long)d.ny * d.nz;
    const long long n = d.n();
    const long long sy = d.nz;
    const long long p0 = d.idx(i0, j, k);
    const T two_hx = T(2. * hx), two_hy = T(2. * hy), two_hz = T(2. * hz);
    const T ihx = T(1. / (2. * hx)), ihy = T(1. / (2. * hy)), ihz = T(1. / (2. * hz));
    // Every load of the NI planes is issued before the first store (the stores to b3
    // and dmb would otherwise hold the next plane's loads back): phi along i for planes
    // i0-1 .. i0+NI (and the second one-sided point on an i face), the j and k
    // neighbours of each plane, g and the three components of b.
    T fi[NI + 2], fi2[NI], fjm[NI], fjp[NI], fkm[NI], fkp[NI], gv[NI], bv0[NI][3];
#pragma unroll
    for (int t = 0; t < NI + 2; ++t) {
        const int i = i0 - 1 + t;
        fi[t] = (i >= 0 && i < d.nx && t <= cnt + 1) ? phi[p0 + (long long)(t - 1) * plane] : T(0);
    }
#pragma unroll
    for (int t = 0; t < NI; ++t) {
        if (t >= cnt) break;
        const int i = i0 + t;
        const long long p = p0 + (long long)t * plane;
        fi2[t] = i == 0 ? phi[p + 2 * plane] : (i == d.nx - 1 ? phi[p - 2 * plane] : T(0));
        if (j == 0) {
            fjp[t] = phi[p + sy];
            fjm[t] = phi[p + 2 * sy];
        } else if (j == d.ny - 1) {
            fjm[t] = phi[p - sy];
            fjp[t] = phi[p - 2 * sy];
        } else {
            fjp[t] = phi[p + sy];
            fjm[t] = phi[p - sy];
        }
        if (k == 0) {
            fkp[t] = phi[p + 1];
            fkm[t] = phi[p + 2];
        } else if (k == d.nz - 1) {
            fkm[t] = phi[p - 1];
            fkp[t] = phi[p - 2];
        } else {
            fkp[t] = phi[p + 1];
            fkm[t] = phi[p - 1];
        }
        gv[t] = g[p];
#pragma unroll
        for (int cmp = 0; cmp < 3; ++cmp) bv0[t][cmp] = b3[cmp * n + p];
    }
#pragma unroll
    for (int t = 0; t < NI; ++t) {
        if (t >= cnt) break;
        const int i = i0 + t;
        const long long p = p0 + (long long)t * plane;
        const T fm = fi[t], f0 = fi[t + 1], fp = fi[t + 2];
        T gr[3];
        if (i == 0) gr[0] = over_two_h(T(4) * fp - T(3) * f0 - fi2[t], two_hx, ihx);
        else if (i == d.nx - 1) gr[0] = over_two_h(T(3) * f0 - T(4) * fm + fi2[t], two_hx, ihx);
        else gr[0] = over_two_h(fp - fm, two_hx, ihx);
        // j == 0: fjp = phi(j+1), fjm = phi(j+2); j == ny-1: fjm = phi(j-1), fjp = phi(j-2)
        if (j == 0) gr[1] = over_two_h(T(4) * fjp[t] - T(3) * f0 - fjm[t], two_hy, ihy);
        else if (j == d.ny - 1) gr[1] = over_two_h(T(3) * f0 - T(4) * fjm[t] + fjp[t], two_hy, ihy);
        else gr[1] = over_two_h(fjp[t] - fjm[t], two_hy, ihy);
        if (k == 0) gr[2] = over_two_h(T(4) * fkp[t] - T(3) * f0 - fkm[t], two_hz, ihz);
        else if (k == d.nz - 1) gr[2] = over_two_h(T(3) * f0 - T(4) * fkm[t] + fkp[t], two_hz, ihz);
        else gr[2] = over_two_h(fkp[t] - fkm[t], two_hz, ihz);
        const T gg = gv[t];
#pragma unroll
        for (int cmp = 0; cmp < 3; ++cmp) {
            T bv = bv0[t][cmp];
            bv += gr[cmp];
            const T mag = fabs(bv) - gg;
            const T sgn = T((int)(bv > T(0)) - (int)(bv < T(0)));
            const T dn = sgn * ((mag < T(0)) ? T(0) : mag);
            bv -= dn;
            b3[cmp * n + p] = bv;
            dmb[cmp * n + p] = dn - bv;
        }
    }
}

template <typename T, int NI>
__global__ void __launch_bounds__(256) bregman_kernel(const T* __restrict__ phi, T* __restrict__ b3, T* __restrict__ dmb, const T* __restrict__ g, Dims d, double hx, double hy, double hz)
{
    bregman_body<T, NI>(blockIdx, gridDim, phi, b3, dmb, g, d, hx, hy, hz);
}

// ---- vectorised natural-layout kernels (nz a multiple of W = 16/sizeof(T)) ----
// Thread per group of W consecutive k of row j, marching over NI planes of i.

// cut_phi + tolerance sums, reading the solve result from the packed layout: for
// natural k = kb .. kb+W-1 (kb even) the even k sit in the colour array of (i+j)&1 and
// the odd k in the other, both at m = kb/2 .. kb/2 + W/2 - 1.
template <typename T, bool PACKED, int NI>
__device__ __forceinline__ void clamp_tol_vec_body(const uint3 blockIdx, const dim3 gridDim, const T* __restrict__ u, T* phi, T* __restrict__ u_out, Dims d, T a0, T b0, double* part)
{
    typedef V16<T> VT;
    typedef typename VT::type VV;
    constexpr int W = VT::W;
    int g, j;
    flat_pair(blockIdx, (unsigned)(d.nz / W), g, j);
    const int i0 = blockIdx.z * NI;
    const int kb = g * W;
    double s_d = 0, s_o = 0;
    if (kb < d.nz && j < d.ny) {
        const long long pplane = (long long)d.ny * d.hz();
        const long long npk = pplane * d.nx;
#pragma unroll
        for (int t = 0; t < NI; ++t) {
            const int i = i0 + t;
            if (i >= d.nx) break;
            const long long p = d.idx(i, j, kb);
            VV uv;
            if (PACKED) {
                const long long pq = ((long long)i * d.ny + j) * d.hz() + (kb >> 1);
                const int c0 = (i + j) & 1;  // colour of the even k
                const T* ev = u + (c0 ? npk : 0) + pq;
                const T* od = u + (c0 ? 0 : npk) + pq;
#pragma unroll
                for (int h = 0; h < W / 2; ++h) {
                    VT::set(uv, 2 * h, ev[h]);
                    VT::set(uv, 2 * h + 1, od[h]);
                }
            } else {
                uv = *reinterpret_cast<const VV*>(u + p);
            }
            if (u_out) *reinterpret_cast<VV*>(u_out + p) = uv;
            const VV old = *reinterpret_cast<const VV*>(phi + p);
            VV nv;
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
                T v = VT::get(uv, cc);
                if (v < a0) v = a0;
                else if (v > b0) v = b0;
                VT::set(nv, cc, v);
                const double o = (double)VT::get(old, cc);
                const double df = (double)v - o;
                s_d += df * df;
                s_o += o * o;
            }
            *reinterpret_cast<VV*>(phi + p) = nv;
        }
    }
    block_sum2_store(s_d, s_o, part, block_linear_id(blockIdx, gridDim), grid_blocks(gridDim));
}

template <typename T, bool PACKED, int NI>
__global__ void __launch_bounds__(256) clamp_tol_vec_kernel(const T* __restrict__ u, T* phi, T* __restrict__ u_out, Dims d, T a0, T b0, double* part)
{
    clamp_tol_vec_body<T, PACKED, NI>(blockIdx, gridDim, u, phi, u_out, d, a0, b0, part);
}

// Split-Bregman update (see bregman_kernel), vectorised along k; rows on an i or j face
// of the volume take the scalar one-sided stencils.
template <typename T, int NI>
__device__ __forceinline__ void bregman_vec_body(const uint3 blockIdx, const dim3 gridDim, const T* __restrict__ phi, T* __restrict__ b3, T* __restrict__ dmb, const T* __restrict__ g3, Dims d, double hx, double hy, double hz)
{
    typedef V16<T> VT;
    typedef typename VT::type VV;
    constexpr int W = VT::W;
    int g, j;
    flat_pair(blockIdx, (unsigned)(d.nz / W), g, j);
    const int i0 = blockIdx.z * NI;
    const int kb = g * W;
    if (kb >= d.nz || j >= d.ny) return;
    const long long plane = (long long)d.ny * d.nz;
    const long long sy = d.nz;
    const long long n = d.n();
    const T two_hx = T(2. * hx), two_hy = T(2. * hy), two_hz = T(2. * hz);
    const T ihx = T(1. / (2. * hx)), ihy = T(1. / (2. * hy)), ihz = T(1. / (2. * hz));
    const bool jint = j >= 1 && j <= d.ny - 2;
    const long long p0 = d.idx(i0, j, kb);
    VV f[NI + 2];
#pragma unroll
    for (int t = 0; t < NI + 2; ++t) {
        const int i = i0 - 1 + t;
        if (i >= 0 && i < d.nx) f[t] = *reinterpret_cast<const VV*>(phi + p0 + (long long)(t - 1) * plane);
        else f[t] = VV{};
    }
    // every read of the NI planes is issued before the first store: b3 is read and
    // written, so a read placed after a store could not be moved ahead of it
    VV yms[NI], yps[NI], ggs[NI], bos[NI][3];
    T zlo[NI], zhi[NI];
#pragma unroll
    for (int t = 0; t < NI; ++t) {
        const int i = i0 + t;
        const long long p = p0 + (long long)t * plane;
        yms[t] = yps[t] = ggs[t] = VV{};
        bos[t][0] = bos[t][1] = bos[t][2] = VV{};
        zlo[t] = zhi[t] = T(0);
        if (i < d.nx) {
            if (jint && i >= 1 && i <= d.nx - 2) {
                yms[t] = *reinterpret_cast<const VV*>(phi + p - sy);
                yps[t] = *reinterpret_cast<const VV*>(phi + p + sy);
            }
            if (kb >= 1) zlo[t] = phi[p - 1];
            if (kb + W < d.nz) zhi[t] = phi[p + W];
            ggs[t] = *reinterpret_cast<const VV*>(g3 + p);
#pragma unroll
            for (int cmp = 0; cmp < 3; ++cmp) bos[t][cmp] = *reinterpret_cast<const VV*>(b3 + cmp * n + p);
        }
    }
#pragma unroll
    for (int t = 0; t < NI; ++t) {
        const int i = i0 + t;
        if (i >= d.nx) break;
        const long long p = p0 + (long long)t * plane;
        const bool rowint = jint && i >= 1 && i <= d.nx - 2;
        const VV ym = yms[t], yp = yps[t];
        // phi at k = kb-1 .. kb+W of this row: zz[c + 1] = phi[kb + c]
        T zz[W + 2];
        zz[0] = zlo[t];
#pragma unroll
        for (int c = 0; c < W; ++c) zz[c + 1] = VT::get(f[t + 1], c);
        zz[W + 1] = zhi[t];
        const VV gg = ggs[t];
        VV bo[3], dn[3];
#pragma unroll
        for (int cmp = 0; cmp < 3; ++cmp) bo[cmp] = bos[t][cmp];
#pragma unroll
        for (int cc = 0; cc < W; ++cc) {
            const int k = kb + cc;
            T gr[3];
            if (rowint) {
                // i and j inside: central x and y terms; the z term is central or, on
                // the faces k = 0 and k = nz-1, grad_term's one-sided difference,
                // evaluated with the same operations without a branch
                gr[0] = over_two_h(VT::get(f[t + 2], cc) - VT::get(f[t], cc), two_hx, ihx);
                gr[1] = over_two_h(VT::get(yp, cc) - VT::get(ym, cc), two_hy, ihy);
                T tz = over_two_h(zz[cc + 2] - zz[cc], two_hz, ihz);
                if (cc == 0) {
                    const T lo = over_two_h(T(4) * zz[cc + 2] - T(3) * zz[cc + 1] - zz[cc + 3], two_hz, ihz);
                    tz = k == 0 ? lo : tz;
                }
                if (cc == W - 1) {
                    const T hi = over_two_h(T(3) * zz[cc + 1] - T(4) * zz[cc] + zz[cc - 1], two_hz, ihz);
                    tz = k == d.nz - 1 ? hi : tz;
                }
                gr[2] = tz;
            } else {
                const long long pc = p + cc;
                gr[0] = grad_term(phi, pc, plane, i, d.nx, hx);
                gr[1] = grad_term(phi, pc, sy, j, d.ny, hy);
                gr[2] = grad_term(phi, pc, 1, k, d.nz, hz);
            }
            const T gv = VT::get(gg, cc);
#pragma unroll
            for (int cmp = 0; cmp < 3; ++cmp) {
                T bv = VT::get(bo[cmp], cc);
                bv += gr[cmp];
                const T mag = fabs(bv) - gv;
                const T sgn = T((int)(bv > T(0)) - (int)(bv < T(0)));
                const T dd = sgn * ((mag < T(0)) ? T(0) : mag);
                bv -= dd;
                VT::set(bo[cmp], cc, bv);
                VT::set(dn[cmp], cc, dd - bv);
            }
        }
#pragma unroll
        for (int cmp = 0; cmp < 3; ++cmp) {
            *reinterpret_cast<VV*>(b3 + cmp * n + p) = bo[cmp];
            *reinterpret_cast<VV*>(dmb + cmp * n + p) = dn[cmp];
        }
    }
}

template <typename T, int NI>
__global__ void __launch_bounds__(256) bregman_vec_kernel(const T* __restrict__ phi, T* __restrict__ b3, T* __restrict__ dmb, const T* __restrict__ g3, Dims d, double hx, double hy, double hz)
{
    bregman_vec_body<T, NI>(blockIdx, gridDim, phi, b3, dmb, g3, d, hx, hy, hz);
}

// im3d::div vectorised along k (see div_point); rows on an i or j face of the volume
// take the scalar rule with the reference's quirks.
template <typename T, int NI>
__device__ __forceinline__ void div_vec_body(const uint3 blockIdx, const dim3 gridDim, const T* __restrict__ v, T* __restrict__ out, Dims d, double hx, double hy, double hz)
{
    typedef V16<T> VT;
    typedef typename VT::type VV;
    constexpr int W = VT::W;
    int g, j;
    flat_pair(blockIdx, (unsigned)(d.nz / W), g, j);
    const int i0 = blockIdx.z * NI;
    const int kb = g * W;
    if (kb >= d.nz || j >= d.ny) return;
    const long long plane = (long long)d.ny * d.nz;
    const long long sy = d.nz;
    const long long n = d.n();
    const T* f0 = v;
    const T* f1 = v + n;
    const T* f2 = v + 2 * n;
    const T two_hx = T(2. * hx), two_hy = T(2. * hy), two_hz = T(2. * hz);
    const T ihx = T(1. / (2. * hx)), ihy = T(1. / (2. * hy)), ihz = T(1. / (2. * hz));
    const bool jint = j >= 1 && j <= d.ny - 2;
    const long long p0 = d.idx(i0, j, kb);
    VV x[NI + 2];
#pragma unroll
    for (int t = 0; t < NI + 2; ++t) {
        const int i = i0 - 1 + t;
        if (i >= 0 && i < d.nx) x[t] = *reinterpret_cast<const VV*>(f0 + p0 + (long long)(t - 1) * plane);
        else x[t] = VV{};
    }
#pragma unroll
    for (int t = 0; t < NI; ++t) {
        const int i = i0 + t;
        if (i >= d.nx) break;
        const long long p = p0 + (long long)t * plane;
        const bool rowint = jint && i >= 1 && i <= d.nx - 2;
        VV o;
        if (rowint) {
            const VV ym = *reinterpret_cast<const VV*>(f1 + p - sy);
            const VV yp = *reinterpret_cast<const VV*>(f1 + p + sy);
            const VV zc = *reinterpret_cast<const VV*>(f2 + p);
            // f2 at k = kb-1 .. kb+W: zz[c + 1] = f2[kb + c]
            T zz[W + 2];
            zz[0] = kb >= 1 ? f2[p - 1] : T(0);
#pragma unroll
            for (int c = 0; c < W; ++c) zz[c + 1] = VT::get(zc, c);
            zz[W + 1] = kb + W < d.nz ? f2[p + W] : T(0);
            // i and j inside: div_point's x and y terms are central, and its z term is
            // central or, on the faces k = 0 and k = nz-1, grad_term's one-sided
            // difference; evaluated here with the same operations, without a branch
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
                const int k = kb + cc;
                const T tx = over_two_h(VT::get(x[t + 2], cc) - VT::get(x[t], cc), two_hx, ihx);
                const T ty = over_two_h(VT::get(yp, cc) - VT::get(ym, cc), two_hy, ihy);
                T tz = over_two_h(zz[cc + 2] - zz[cc], two_hz, ihz);
                if (cc == 0) {
                    const T lo = over_two_h(T(4) * zz[cc + 2] - T(3) * zz[cc + 1] - zz[cc + 3], two_hz, ihz);
                    tz = k == 0 ? lo : tz;
                }
                if (cc == W - 1) {
                    const T hi = over_two_h(T(3) * zz[cc + 1] - T(4) * zz[cc] + zz[cc - 1], two_hz, ihz);
                    tz = k == d.nz - 1 ? hi : tz;
                }
                VT::set(o, cc, tx + ty + tz);
            }
        } else {
#pragma unroll
            for (int cc = 0; cc < W; ++cc) VT::set(o, cc, div_point(f0, f1, f2, d, i, j, kb + cc, hx, hy, hz));
        }
        *reinterpret_cast<VV*>(out + p) = o;
    }
}

template <typename T, int NI>
__global__ void __launch_bounds__(256) div_vec_kernel(const T* __restrict__ v, T* __restrict__ out, Dims d, double hx, double hy, double hz)
{
    div_vec_body<T, NI>(blockIdx, gridDim, v, out, d, hx, hy, hz);
}

// sum (a - b)^2 and sum b^2 over n elements (relative change of a sweep)
template <typename T>
__global__ void diff_sums_kernel(const T* __restrict__ a, const T* __restrict__ b, long long n,
                                 double* part)
{
    double sd = 0, sb = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const double x = (double)a[q] - (double)b[q];
        sd += x * x;
        sb += (double)b[q] * (double)b[q];
    }
    block_sum2_store(sd, sb, part, block_linear_id(blockIdx, gridDim), grid_blocks(gridDim));
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
                                 Dims d, T inv_dt, T bc, int dirichlet, double* part)
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
    if (part) block_sum_store(acc, part, block_linear_id(blockIdx, gridDim));
}


// ------------------------------------------------------------------ utilities
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
    bool bad = false;  // a NaN or Inf seen: umax[3] is raised
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const double v = (double)p[q];
        bad |= !isfinite(v);
        const unsigned long long a = order_key(v), b = order_key(-v);
        mx = a > mx ? a : mx;
        mn = b > mn ? b : mn;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicMax(umax + 3, 1ull);
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

// ---- connected component (image3d<T>::connected_component, image3d_imp.hxx:1694-2120) ----
// One byte per cell: bit 1 = white in the black-and-white image (img >= pivot, or
// img < pivot in the negative image), bit 0 = in the component.

// im_to_black_and_white (image3d_imp.hxx:1592-1623) and the initial component: the
// cells where init != 0 and white (init != NULL), else only cell `seed` (>= 0).
template <typename T>
__global__ void cc_init_kernel(const T* __restrict__ img, const T* __restrict__ init,
                               unsigned char* __restrict__ m, long long n, T pivot, int negative,
                               long long seed)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const bool below = img[q] < pivot;
        const unsigned char white = (unsigned char)(negative ? below : !below);
        const unsigned char in = init ? (unsigned char)(init[q] != T(0) && white)
                                      : (unsigned char)(q == seed);
        m[q] = (unsigned char)((white << 1) | in);
    }
}

// One growth pass over tiles of 32 (k) x 8 (j) x 4 (i) cells. A tile and its one-cell
// halo are read from `in`; inside the tile the component grows to a local fixed point
// (a white cell joins when a neighbour in the component lies off the volume's faces:
// 1 <= i <= nx-2, 1 <= j <= ny-2 and, unless nz == 1, 1 <= k <= nz-2; 6 face
// neighbours, 26 with FULL), then the tile is written to `out` and *changed is raised
// if it grew. Growth only turns cells on, so passes repeated until nothing changes
// reach the reference's fixed point whatever the order.
constexpr int kCcK = 32, kCcJ = 8, kCcI = 4;
template <bool FULL>
__global__ void __launch_bounds__(256) cc_grow_kernel(const unsigned char* __restrict__ in,
                                                      unsigned char* __restrict__ out, Dims d,
                                                      unsigned long long* changed)
{
    constexpr int SK = kCcK + 2, SJ = kCcJ + 2, SI = kCcI + 2;
    __shared__ unsigned char tile[SI * SJ * SK];
    volatile unsigned char* t = tile;
    const int k0 = blockIdx.x * kCcK, j0 = blockIdx.y * kCcJ, i0 = blockIdx.z * kCcI;
    const int tid = threadIdx.y * kCcK + threadIdx.x;
    for (int e = tid; e < SI * SJ * SK; e += 256) {
        const int li = e / (SJ * SK), r = e - li * SJ * SK, lj = r / SK, lk = r - lj * SK;
        const int i = i0 - 1 + li, j = j0 - 1 + lj, k = k0 - 1 + lk;
        unsigned char v = 0;
        if (i >= 0 && i < d.nx && j >= 0 && j < d.ny && k >= 0 && k < d.nz) v = in[d.idx(i, j, k)];
        t[e] = v;
    }
    __syncthreads();
    const int lk = threadIdx.x + 1, lj = threadIdx.y + 1;
    const int k = k0 + threadIdx.x, j = j0 + threadIdx.y;
    auto spreads = [&](int i, int jj, int kk) {
        return i >= 1 && i <= d.nx - 2 && jj >= 1 && jj <= d.ny - 2 &&
               (d.nz == 1 || (kk >= 1 && kk <= d.nz - 2));
    };
    bool grew = false;
    bool step;
    do {
        step = false;
#pragma unroll
        for (int c = 0; c < kCcI; ++c) {
            const int li = c + 1;
            const int at = (li * SJ + lj) * SK + lk;
            if (t[at] != 2) continue;  // only white cells not yet in the component
            bool join = false;
#pragma unroll
            for (int di = -1; di <= 1; ++di)
#pragma unroll
                for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
                    for (int dk = -1; dk <= 1; ++dk) {
                        const int nnz = (di != 0) + (dj != 0) + (dk != 0);
                        if (nnz == 0 || (!FULL && nnz != 1)) continue;
                        const int nb = ((li + di) * SJ + lj + dj) * SK + lk + dk;
                        if ((t[nb] & 1) && spreads(i0 + c + di, j + dj, k + dk)) join = true;
                    }
            if (join) {
                t[at] = 3;
                step = true;
                grew = true;
            }
        }
    } while (__syncthreads_or(step));
    if (k < d.nz && j < d.ny) {
#pragma unroll
        for (int c = 0; c < kCcI; ++c) {
            const int i = i0 + c;
            if (i < d.nx) out[d.idx(i, j, k)] = t[((c + 1) * SJ + lj) * SK + lk];
        }
    }
    if (__syncthreads_or(grew) && tid == 0) atomicOr(changed, 1ull);
}

// The result: the component as 0 / 1, or with binary == 0 cc_not_binary_output
// (image3d_imp.hxx:1801-1817): (res + [img < pivot]) * (img - mn) + mn.
template <typename T>
__global__ void cc_output_kernel(const unsigned char* __restrict__ m, const T* __restrict__ img,
                                 T* __restrict__ res, long long n, int binary, T mn, T pivot)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        T v = (T)(m[q] & 1);
        if (!binary) {
            const T x = img[q];
            v += (T)(x < pivot ? 1 : 0);
            v *= x - mn;
            v += mn;
        }
        res[q] = v;
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

// ---- learned warm start: fields of one Poisson solve to and from the network ----
// Packed cell of natural (i, j, k): its colour's array at d.pidx(i, j, k).
__device__ __forceinline__ long long packed_at(const Dims& d, int i, int j, int k)
{
    return d.pidx(i, j, k) + (((i + j + k) & 1) ? d.npk() : 0);
}

// The network's inputs, four FP32 volumes x[f][n] (natural layout): the forcing term
// rhs = b_eff - u_in / dt, the previous solve's u, div(d - b) and phi.
static __global__ void ws_fields_kernel(const float* __restrict__ bpk, const float* __restrict__ upk,
                                 const float* __restrict__ prevu, const float* __restrict__ divdb,
                                 const float* __restrict__ phi, Dims d, float inv_dt, float* __restrict__ x)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long v = d.idx(i, j, k), pv = packed_at(d, i, j, k), n = d.n();
    x[v] = bpk[pv] - upk[pv] * inv_dt;
    x[n + v] = prevu[v];
    x[2 * n + v] = divdb[v];
    x[3 * n + v] = phi[v];
}

// u_in += the network's correction y on the cells the solve updates (all cells with
// Neumann conditions, the interior with Dirichlet ones, whose faces keep their value).
static __global__ void ws_apply_kernel(float* __restrict__ upk, const float* __restrict__ y, Dims d, int dirichlet)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    if (dirichlet && (i == 0 || j == 0 || k == 0 || i == d.nx - 1 || j == d.ny - 1 || k == d.nz - 1)) return;
    upk[packed_at(d, i, j, k)] += y[d.idx(i, j, k)];
}

// The correction the solve made, natural layout: t = u_solved - u_in.
static __global__ void ws_target_kernel(const float* __restrict__ upk, const float* __restrict__ upk0, Dims d,
                                 float* __restrict__ t)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return;
    const long long pv = packed_at(d, i, j, k);
    t[d.idx(i, j, k)] = upk[pv] - upk0[pv];
}

}  // namespace im3d

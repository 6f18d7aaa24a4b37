// codelets.cuh -- compile-time 1D DFT codelets on register arrays.
//
// Every codelet transforms N complex values held in a fully unrolled local array
// (the compiler keeps it in registers) with exponent sign S (-1 forward, +1
// backward, unnormalised), the convention of the reference contract
// (bench/geom/fft3d_api.h:5-9, python/fft3d.py:65-69).
//
// Routes, chosen at compile time from the factorisation of N:
//   N = 1, 2, 4               explicit butterflies (no multiplications)
//   N = 3                     Winograd 3-point
//   N odd prime (or odd with no better split)
//                             conjugate-pair folded direct sum: (N-1)^2 real FMA
//   N = 17, ALG_CRT           the folded sum with its cosine half as a length-8
//                             cyclic convolution through a CRT split (dft17_crt)
//   N = 17, ALG_RADER         Rader (python/fft3d.py:204-245): the 16 non-zero
//                             inputs permuted by the primitive root 3 and a
//                             length-16 cyclic convolution through a 16-point FFT,
//                             against a kernel spectrum precomputed at plan time
//   N = A*B, gcd(A,B) = 1     Good-Thomas prime-factor algorithm, no twiddles
//                             (6 = 2*3, 12 = 4*3, 24 = 8*3, 36 = 4*9, ...)
//   N = A*B otherwise         Cooley-Tukey (python/fft3d.py:166-188 is the radix-r
//                             DIT form of it): A-point DFTs, twiddles W_N^{n2*k1},
//                             B-point DFTs (8 = 2*4, 9 = 3*3, 16 = 4*4, 32 = 4*8)
//
// Twiddle factors come from a table cos/sin(2*pi*e/N), e in [0, N), that the plan
// computes in extended precision on the host and uploads to __constant__ memory;
// the index e is a compile-time constant, so each factor is a constant-bank
// operand of the FMA that uses it.  Host builds of this header (the CPU unit
// tests of the codelets) read a host copy of the same table.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#if defined(__CUDACC__)
#define FFT_HD __host__ __device__ __forceinline__
#else
#define FFT_HD inline
#endif

namespace fft3d {

template <typename T>
struct alignas(2 * sizeof(T)) cx {
    T re, im;
};

// ------------------------------------------------------------------ constexpr helpers

constexpr int ce_gcd(int a, int b) { return b == 0 ? a : ce_gcd(b, a % b); }

constexpr int ce_spf(int n)  // smallest prime factor
{
    if (n % 2 == 0) return 2;
    for (int d = 3; d * d <= n; d += 2)
        if (n % d == 0) return d;
    return n;
}

constexpr bool ce_is_prime(int n) { return n >= 2 && ce_spf(n) == n; }

constexpr int ce_modinv(int a, int m)  // a^-1 mod m, m > 1, gcd(a,m) = 1
{
    for (int x = 1; x < m; ++x)
        if ((a * x) % m == 1) return x;
    return 1;
}

constexpr int ce_pow2_part(int n)
{
    int p = 1;
    while (n % 2 == 0) { n /= 2; p *= 2; }
    return p;
}

// Split used for a composite N: returns A (the first-stage DFT size); B = N / A.
constexpr int ce_split(int n)
{
    const int p2 = ce_pow2_part(n);
    if (p2 > 1 && p2 < n) return p2;              // 2^a * odd, coprime: PFA
    if (p2 == n) {                                // power of two: CT
        if (n == 8) return 2;
        if (n == 16) return 4;
        if (n == 32) return 4;
        if (n == 64) return 8;
        return 2;
    }
    // odd composite: coprime split if one exists, else a prime-power CT split
    const int p = ce_spf(n);
    int q = 1, m = n;
    while (m % p == 0) { m /= p; q *= p; }
    if (m > 1) return q;                           // q and m coprime: PFA
    return p;                                      // p^k: CT(p, p^(k-1))
}

// ------------------------------------------------------------------ twiddle tables

// Extents with a table.  Offsets are in entries (one {cos, sin} pair per entry).
constexpr int TW_MAXN = 64;
constexpr int tw_off(int n) { return n * (n - 1) / 2; }   // N = 1..TW_MAXN, packed
constexpr int TW_ENTRIES = tw_off(TW_MAXN + 1);            // 2080
// Rader-17 kernel spectra: [sign index][16], sign index 0 = forward, 1 = backward.
constexpr int RADER17_ENTRIES = 32;
// CRT-17 kernel residues (dft17_crt): the cosine kernel c[m] = cos(2*pi*3^m/17),
// m = 0..7, reduced mod x-1, x+1 (scaled 1/8), x^2+1 (1/4) and x^4+1 (1/2).
constexpr int CRT17_ENTRIES = 8;
// Line lengths above TW_MAXN: one table per N in global memory, read through
// the read-only cache -- lines spread over several lanes (96..256; lane-dependent
// indices would serialise on the constant cache) and the primes 83 and 97 of the
// reference's test geometries (folded direct sums).
constexpr int twbig_off(int n)
{
    return n == 96 ? 0 : n == 128 ? 96 : n == 192 ? 224 : n == 256 ? 416 : n == 83 ? 672 : n == 97 ? 755 : -1;
}
constexpr int TWBIG_ENTRIES = 852;

}  // namespace fft3d

// Table storage.  The device copies are defined in exactly one translation unit
// (tables.cu) and declared here; host copies serve the host build of the codelets.
#if defined(__CUDACC__)
extern __constant__ double2 c_tw_d[fft3d::TW_ENTRIES];
extern __constant__ float2 c_tw_f[fft3d::TW_ENTRIES];
extern __constant__ double2 c_rader17_d[fft3d::RADER17_ENTRIES];
extern __constant__ float2 c_rader17_f[fft3d::RADER17_ENTRIES];
extern __constant__ double c_crt17_d[fft3d::CRT17_ENTRIES];
extern __constant__ float c_crt17_f[fft3d::CRT17_ENTRIES];
#endif
#if defined(__CUDACC__)
extern __device__ double2 g_twbig_d[fft3d::TWBIG_ENTRIES];
extern __device__ float2 g_twbig_f[fft3d::TWBIG_ENTRIES];
#endif
extern double2 h_tw_d[fft3d::TW_ENTRIES];
extern float2 h_tw_f[fft3d::TW_ENTRIES];
extern double2 h_twbig_d[fft3d::TWBIG_ENTRIES];
extern float2 h_twbig_f[fft3d::TWBIG_ENTRIES];
extern double2 h_rader17_d[fft3d::RADER17_ENTRIES];
extern float2 h_rader17_f[fft3d::RADER17_ENTRIES];
extern double h_crt17_d[fft3d::CRT17_ENTRIES];
extern float h_crt17_f[fft3d::CRT17_ENTRIES];

namespace fft3d {

template <typename T>
struct Tab;

template <>
struct Tab<double> {
    FFT_HD static double2 tw(int i)
    {
#if defined(__CUDA_ARCH__)
        return c_tw_d[i];
#else
        return h_tw_d[i];
#endif
    }
    FFT_HD static double2 rader17(int i)
    {
#if defined(__CUDA_ARCH__)
        return c_rader17_d[i];
#else
        return h_rader17_d[i];
#endif
    }
    FFT_HD static double crt17(int i)
    {
#if defined(__CUDA_ARCH__)
        return c_crt17_d[i];
#else
        return h_crt17_d[i];
#endif
    }
    FFT_HD static double2 twbig(int i)
    {
#if defined(__CUDA_ARCH__)
        return __ldg(&g_twbig_d[i]);
#else
        return h_twbig_d[i];
#endif
    }
};

template <>
struct Tab<float> {
    FFT_HD static float2 tw(int i)
    {
#if defined(__CUDA_ARCH__)
        return c_tw_f[i];
#else
        return h_tw_f[i];
#endif
    }
    FFT_HD static float2 rader17(int i)
    {
#if defined(__CUDA_ARCH__)
        return c_rader17_f[i];
#else
        return h_rader17_f[i];
#endif
    }
    FFT_HD static float crt17(int i)
    {
#if defined(__CUDA_ARCH__)
        return c_crt17_f[i];
#else
        return h_crt17_f[i];
#endif
    }
    FFT_HD static float2 twbig(int i)
    {
#if defined(__CUDA_ARCH__)
        return __ldg(&g_twbig_f[i]);
#else
        return h_twbig_f[i];
#endif
    }
};

// ------------------------------------------------------------------ complex arithmetic

template <typename T>
FFT_HD cx<T> cadd(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T>
FFT_HD cx<T> csub(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T>
FFT_HD cx<T> cscale(cx<T> a, T s) { return {a.re * s, a.im * s}; }

// a * (i*S), S = +-1
template <int S, typename T>
FFT_HD cx<T> cmul_iS(cx<T> a)
{
    if constexpr (S > 0) return {-a.im, a.re};
    else return {a.im, -a.re};
}

// {cos, sin}(2*pi*e/N), 0 <= e < N, from the table that holds N.
template <int N, typename T>
FFT_HD auto line_tw(int e)
{
    static_assert(N <= TW_MAXN || twbig_off(N) >= 0, "no twiddle table for this extent");
    if constexpr (N <= TW_MAXN) return Tab<T>::tw(tw_off(N) + e);
    else return Tab<T>::twbig(twbig_off(N) + e);
}

// a * W_N^e with W_N = exp(S*2*pi*i/N).  Callers pass an exponent that is a
// constant once their loops are unrolled, so the branches below fold away and
// the table read becomes a constant-bank operand.
template <int N, int S, typename T>
FFT_HD cx<T> ctwiddle(cx<T> a, int E)
{
    const int e = ((E % N) + N) % N;
    if (e == 0) return a;
    if (4 * e == N) return cmul_iS<S>(a);
    if (2 * e == N) return {-a.re, -a.im};
    if (4 * e == 3 * N) return cmul_iS<-S>(a);
    const auto w = line_tw<N, T>(e);  // {cos, sin}(2*pi*e/N)
    const T c = w.x;
    const T s = (S > 0) ? w.y : -w.y;
    return {a.re * c - a.im * s, a.re * s + a.im * c};
}

// ------------------------------------------------------------------ codelets

constexpr int ALG_DEFAULT = 0;
constexpr int ALG_RADER = 1;
constexpr int ALG_CRT = 2;

template <int N, int S, typename T, int ALG = ALG_DEFAULT>
FFT_HD void dft(cx<T> *v);

// Folded direct sum for odd N: with u_j = x_j + x_{N-j}, w_j = x_j - x_{N-j},
// X_k = x_0 + sum_j u_j cos(2*pi*jk/N) + i*S * sum_j w_j sin(2*pi*jk/N) and
// X_{N-k} the same with the sine term negated.
template <int N, int S, typename T>
FFT_HD void dft_odd_folded(cx<T> *v)
{
    constexpr int H = (N - 1) / 2;
    cx<T> u[H + 1], w[H + 1];
#pragma unroll
    for (int j = 1; j <= H; ++j) {
        u[j] = cadd(v[j], v[N - j]);
        w[j] = csub(v[j], v[N - j]);
    }
    cx<T> x0 = v[0];
    cx<T> sum = x0;
#pragma unroll
    for (int j = 1; j <= H; ++j) sum = cadd(sum, u[j]);
#pragma unroll
    for (int k = 1; k <= H; ++k) {
        cx<T> a = x0, b = {T(0), T(0)};
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            const int e = (j * k) % N;
            const auto t = line_tw<N, T>(e);
            a.re += u[j].re * t.x;
            a.im += u[j].im * t.x;
            b.re += w[j].re * t.y;
            b.im += w[j].im * t.y;
        }
        // i*S*b
        const cx<T> ib = cmul_iS<S>(b);
        v[k] = cadd(a, ib);
        v[N - k] = csub(a, ib);
    }
    v[0] = sum;
}

// Winograd 3-point.
template <int S, typename T>
FFT_HD void dft3(cx<T> *v)
{
    const cx<T> t = cadd(v[1], v[2]);
    const cx<T> d = csub(v[1], v[2]);
    const T h = T(0.5);
    const auto w = Tab<T>::tw(tw_off(3) + 1);  // sin(2*pi/3) = sqrt(3)/2
    const cx<T> m = {v[0].re - h * t.re, v[0].im - h * t.im};
    const cx<T> r = cscale(d, w.y);
    const cx<T> ir = cmul_iS<S>(r);
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, ir);
    v[2] = csub(m, ir);
}

// Cooley-Tukey, N = A*B: n = B*n1 + n2, k = k1 + A*k2,
// X[k1 + A*k2] = sum_n2 W_B^{n2 k2} W_N^{n2 k1} sum_n1 x[B n1 + n2] W_A^{n1 k1}.
template <int N, int A, int S, typename T>
FFT_HD void dft_ct(cx<T> *v)
{
    constexpr int B = N / A;
    cx<T> y[A][B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
        cx<T> t[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) t[n1] = v[B * n1 + n2];
        dft<A, S, T>(t);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) y[k1][n2] = t[k1];
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
        cx<T> t[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) t[n2] = ctwiddle<N, S>(y[k1][n2], n2 * k1);
        dft<B, S, T>(t);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
    }
}

// Good-Thomas, N = A*B with gcd(A,B) = 1: input n = (B*n1 + A*n2) mod N,
// output k = (B*(B^-1 mod A)*k1 + A*(A^-1 mod B)*k2) mod N; then
// W_N^{nk} = W_A^{n1 k1} W_B^{n2 k2} and no twiddles are needed.
template <int N, int A, int S, typename T>
FFT_HD void dft_pfa(cx<T> *v)
{
    constexpr int B = N / A;
    constexpr int CA = B * ce_modinv(B % A, A);  // k = k1 (mod A), 0 (mod B)
    constexpr int CB = A * ce_modinv(A % B, B);  // k = k2 (mod B), 0 (mod A)
    cx<T> y[A][B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
        cx<T> t[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) t[n1] = v[(B * n1 + A * n2) % N];
        dft<A, S, T>(t);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) y[k1][n2] = t[k1];
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
        cx<T> t[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) t[n2] = y[k1][n2];
        dft<B, S, T>(t);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) v[(CA * k1 + CB * k2) % N] = t[k2];
    }
}

// Rader for N = 17 with primitive root g = 3 (python/fft3d.py:204-245).
// a[q] = x[g^q], the outputs are X[g^-s] = x0 + (a (*) brev)[s] with brev[t] =
// W^{g^-t}; the length-16 cyclic convolution runs as 16-point FFT, pointwise
// product with the plan-time spectrum K = FFT16(brev)/16, inverse 16-point FFT.
// x0 is folded into the DC bin so the inverse FFT adds it to every output.
constexpr int rader17_pow(int q)  // 3^q mod 17
{
    int r = 1;
    for (int i = 0; i < q; ++i) r = (r * 3) % 17;
    return r;
}

template <int S, typename T>
FFT_HD void dft17_rader(cx<T> *v)
{
    cx<T> a[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) a[q] = v[rader17_pow(q)];
    const cx<T> x0 = v[0];
    dft<16, -1, T>(a);
    v[0] = cadd(x0, a[0]);
    constexpr int base = (S < 0) ? 0 : 16;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const auto kk = Tab<T>::rader17(base + k);
        const cx<T> p = {a[k].re * kk.x - a[k].im * kk.y, a[k].re * kk.y + a[k].im * kk.x};
        a[k] = p;
    }
    a[0] = cadd(a[0], x0);
    dft<16, +1, T>(a);
#pragma unroll
    for (int s = 0; s < 16; ++s) v[rader17_pow((16 - s) % 16)] = a[s];
}

// 17-point DFT, ALG_CRT: the conjugate-pair folded form of dft_odd_folded with
// its cosine half computed as a cyclic convolution.  The non-zero residues mod 17
// are +-3^a, a = 0..7 (3 is a primitive root, 3^8 = -1): with j_a = +-3^a in
// 1..8 (sign e_a), u_a = v[j_a] + v[17 - j_a] and w_a = e_a (v[j_a] - v[17 - j_a]),
//   cosine sums  A_b = x0 + sum_a u_a c[(a + b) mod 8],   c[m] = cos(2 pi 3^m / 17)
//   sine sums    B_b = e_b sum_a w_a s~[a + b],   s~[m] = s[m], s~[m + 8] = -s[m],
//                s[m] = sin(2 pi 3^m / 17)
// (Rader's re-indexing, folded to the 8 classes +-3^a).  The cosine correlation
// runs as the convolution of u reversed with c through the split
// x^8 - 1 = (x - 1)(x + 1)(x^2 + 1)(x^4 + 1): 14 additions reduce the input, 22
// products against the kernel's residues (a plan-time table with the
// reconstruction's halvings folded in; x0 rides on the x - 1 product) and 14
// additions rebuild the 8 sums -- 50 operations a real component instead of the
// 64 multiply-adds of the direct sum.  The sine half stays direct.
template <int S, typename T>
FFT_HD void dft17_crt(cx<T> *v)
{
    constexpr int J[8] = {1, 3, 8, 7, 4, 5, 2, 6};         // +-3^a mod 17 in 1..8
    constexpr int E[8] = {1, 1, -1, -1, -1, 1, -1, -1};    // its sign
    constexpr int P3[8] = {1, 3, 9, 10, 13, 5, 15, 11};    // 3^a mod 17
    cx<T> U[8], W[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        U[a] = cadd(v[J[a]], v[17 - J[a]]);
        W[a] = E[a] > 0 ? csub(v[J[a]], v[17 - J[a]]) : csub(v[17 - J[a]], v[J[a]]);
    }
    const cx<T> x0 = v[0];
    cx<T> sum = x0;
#pragma unroll
    for (int a = 0; a < 8; ++a) sum = cadd(sum, U[a]);
    // cosine half: y = V (*) c mod x^8 - 1 with V_i = U[(8 - i) mod 8]
    cx<T> P[4], Q[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const cx<T> lo = U[(8 - i) % 8], hi = U[(8 - i - 4) % 8];
        P[i] = cadd(lo, hi);
        Q[i] = csub(lo, hi);
    }
    const cx<T> P10 = cadd(P[0], P[2]), P11 = cadd(P[1], P[3]);
    const cx<T> P20 = csub(P[0], P[2]), P21 = csub(P[1], P[3]);
    const cx<T> e0 = cadd(P10, P11), e1 = csub(P10, P11);
    const T k0 = Tab<T>::crt17(0), k1 = Tab<T>::crt17(1), k20 = Tab<T>::crt17(2), k21 = Tab<T>::crt17(3);
    const cx<T> f0 = {x0.re + e0.re * k0, x0.im + e0.im * k0};
    const cx<T> f1 = cscale(e1, k1);
    const cx<T> F20 = {P20.re * k20 - P21.re * k21, P20.im * k20 - P21.im * k21};
    const cx<T> F21 = {P20.re * k21 + P21.re * k20, P20.im * k21 + P21.im * k20};
    cx<T> FQ[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        cx<T> acc = {T(0), T(0)};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const T kq = m - i >= 0 ? Tab<T>::crt17(4 + m - i) : -Tab<T>::crt17(8 + m - i);
            acc.re += Q[i].re * kq;
            acc.im += Q[i].im * kq;
        }
        FQ[m] = acc;
    }
    const cx<T> Y10 = cadd(f0, f1), Y11 = csub(f0, f1);
    const cx<T> YP[4] = {cadd(Y10, F20), cadd(Y11, F21), csub(Y10, F20), csub(Y11, F21)};
    cx<T> A[8];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        A[b] = cadd(YP[b], FQ[b]);
        A[b + 4] = csub(YP[b], FQ[b]);
    }
    // sine half, direct
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        cx<T> B = {T(0), T(0)};
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int m = a + b;
            const T sm = m < 8 ? line_tw<17, T>(P3[m]).y : -line_tw<17, T>(P3[m - 8]).y;
            B.re += W[a].re * sm;
            B.im += W[a].im * sm;
        }
        const cx<T> ib = cmul_iS<S>(B);
        if (E[b] > 0) {
            v[J[b]] = cadd(A[b], ib);
            v[17 - J[b]] = csub(A[b], ib);
        } else {
            v[J[b]] = csub(A[b], ib);
            v[17 - J[b]] = cadd(A[b], ib);
        }
    }
    v[0] = sum;
}

template <int N, int S, typename T, int ALG>
FFT_HD void dft(cx<T> *v)
{
    if constexpr (N == 1) {
    } else if constexpr (N == 2) {
        const cx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (N == 3) {
        dft3<S, T>(v);
    } else if constexpr (N == 4) {
        const cx<T> s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const cx<T> s13 = cadd(v[1], v[3]), d13 = cmul_iS<S>(csub(v[1], v[3]));
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    } else if constexpr (N == 17 && ALG == ALG_RADER) {
        dft17_rader<S, T>(v);
    } else if constexpr (N == 17 && ALG == ALG_CRT) {
        dft17_crt<S, T>(v);
    } else if constexpr (ce_is_prime(N)) {
        dft_odd_folded<N, S, T>(v);
    } else {
        constexpr int A = ce_split(N);
        if constexpr (ce_gcd(A, N / A) == 1) dft_pfa<N, A, S, T>(v);
        else dft_ct<N, A, S, T>(v);
    }
}

// Exponent sign of each direction.
constexpr int FWD = -1;
constexpr int INV = +1;

}  // namespace fft3d

// splitline.cuh -- a line of N = P*Q points transformed by P lanes of one warp.
//
// A line longer than one thread can hold in registers (the multi-GPU path's
// 96- to 256-point lines; 36-point complex-double lines, 170 registers in one
// thread, for the lane-split TWOPASS kernel) is spread over P lanes.  Lane t of
// the P lanes (P consecutive lanes of a warp for LineSplit, lanes LS apart for
// LaneSplit below) holds Q = N/P points:
//   1. it loads its points n = in(t, n2), n2 = 0..Q-1, and runs a Q-point DFT;
//   2. Cooley-Tukey splits (P, Q not coprime) multiply by W_N^(t*k2);
//   3. a P-point DFT across the P lanes, radix-2 decimation in frequency with
//      __shfl_xor_sync (lane distance P/2, ..., 1, times LS), leaves lane t with
//      frequency k1 = bitrev(t) of every k2;
//   4. it stores its Q results at k = out(k1, k2).
// Prime-factor splits (gcd(P, Q) = 1) use the Good-Thomas maps
//   in(t, n2) = (Q t + P n2) mod N,  out(k1, k2) = (Q (Q^-1 mod P) k1 + P (P^-1 mod Q) k2) mod N,
// under which W_N^(nk) = W_P^(n1 k1) W_Q^(n2 k2): no twiddles.  Cooley-Tukey
// splits use in(t, n2) = t + P n2 and out(k1, k2) = k2 + Q k1.
//
// The lane-exchange schedule exists twice: with shuffles on the device and on
// an array of P lanes on the host (hostcheck), from the same index maps.
#pragma once

#include "codelets.cuh"

namespace fft3d {

template <int N>
struct LineSplit {
    static constexpr int P = 1;
};
// Lines longer than one thread can hold (the multi-GPU large cubes).
template <>
struct LineSplit<96> {
    static constexpr int P = 8, Q = 12;
    static constexpr bool PFA = false;
};
template <>
struct LineSplit<128> {
    static constexpr int P = 8, Q = 16;
    static constexpr bool PFA = false;
};
template <>
struct LineSplit<192> {
    static constexpr int P = 16, Q = 12;
    static constexpr bool PFA = false;
};
template <>
struct LineSplit<256> {
    static constexpr int P = 16, Q = 16;
    static constexpr bool PFA = false;
};

template <int N>
struct SplitMap {
    using SP = LineSplit<N>;
    static constexpr int P = SP::P, Q = SP::Q;
    static constexpr int A = SP::PFA ? Q * ce_modinv(Q % P, P) : 0;  // output weight of k1
    static constexpr int B = SP::PFA ? P * ce_modinv(P % Q, Q) : 0;  // output weight of k2
    FFT_HD static int in(int t, int n2) { return SP::PFA ? (Q * t + P * n2) % N : t + P * n2; }
    FFT_HD static int out(int k1, int k2) { return SP::PFA ? (A * k1 + B * k2) % N : k2 + Q * k1; }
};

template <int P>
FFT_HD int lane_bitrev(int t)
{
    int r = 0;
    for (int b = 1; b < P; b <<= 1) r = (r << 1) | ((t & b) ? 1 : 0);
    return r;
}

#if defined(__CUDACC__)
// P-point DFT of the values a of P consecutive lanes (lane index t < P within
// the group); returns frequency bitrev(t).  Every lane of the warp must call it.
template <int H, int S, typename T>
__device__ __forceinline__ void xlane_stage(cx<T> &a, int t)
{
    if constexpr (H >= 1) {
        cx<T> b;
        b.re = __shfl_xor_sync(0xffffffffu, a.re, H);
        b.im = __shfl_xor_sync(0xffffffffu, a.im, H);
        const bool hi = (t & H) != 0;
        a = hi ? csub(b, a) : cadd(a, b);
        if constexpr (H > 1) {
            if (hi) a = ctwiddle<2 * H, S, T>(a, t & (H - 1));
        }
        xlane_stage<H / 2, S, T>(a, t);
    }
}

template <int P, int S, typename T>
__device__ __forceinline__ cx<T> xlane_dft(cx<T> a, int t)
{
    xlane_stage<P / 2, S, T>(a, t);
    return a;
}

// Lane t of a line: load Q points through ld(position), transform, store Q
// points through st(position, value).  Lanes with valid == false take part in
// the exchange with zeros and store nothing.
template <int N, int S, typename T, class Ld, class St>
__device__ __forceinline__ void split_line(int t, bool valid, Ld ld, St st)
{
    using SP = LineSplit<N>;
    using M = SplitMap<N>;
    cx<T> v[SP::Q];
#pragma unroll
    for (int n2 = 0; n2 < SP::Q; ++n2) v[n2] = valid ? ld(M::in(t, n2)) : cx<T>{T(0), T(0)};
    dft<SP::Q, S, T>(v);
    if constexpr (!SP::PFA) {
#pragma unroll
        for (int k2 = 1; k2 < SP::Q; ++k2) v[k2] = ctwiddle<N, S, T>(v[k2], t * k2);
    }
#pragma unroll
    for (int k2 = 0; k2 < SP::Q; ++k2) v[k2] = xlane_dft<SP::P, S, T>(v[k2], t);
    const int k1 = lane_bitrev<SP::P>(t);
    if (valid) {
#pragma unroll
        for (int k2 = 0; k2 < SP::Q; ++k2) st(M::out(k1, k2), v[k2]);
    }
}
#endif

// ---------------------------------------------------------------- explicit P, strided lanes
//
// The same split with P chosen by the kernel, and the P lanes of a line LS
// apart in the warp (lane t of a line is warp lane w + t*LS, w < LS): a warp
// holds LS lines side by side, so the 8 lanes of every shared-memory phase work
// on 8 different lines at the same position -- with an odd row pitch no bank
// conflicts on rows or columns -- and a global store of a warp covers LS
// consecutive points.  36 = 2 x 18 is a Cooley-Tukey split (the 18-point DFT
// of lane t's points x[t + 2 n2], then W_36^(t k2), then one exchange);
// 36 = 4 x 9 is the Good-Thomas split above.
template <int N, int P>
struct LaneSplit {
    static constexpr int Q = N / P;
    static_assert(P * Q == N && (P & (P - 1)) == 0, "P a power of two dividing N");
    static constexpr bool PFA = ce_gcd(P, Q) == 1;
    static constexpr int A = PFA ? Q * ce_modinv(Q % P, P) : 0;
    static constexpr int B = PFA ? P * ce_modinv(P % Q, Q) : 0;
    FFT_HD static constexpr int in(int t, int n2) { return PFA ? (Q * t + P * n2) % N : t + P * n2; }
    FFT_HD static constexpr int out(int k1, int k2) { return PFA ? (A * k1 + B * k2) % N : k2 + Q * k1; }
};

// W_N^(t k2) of a Cooley-Tukey split (k2 a constant after unrolling).  With
// P = 2 the twiddle of lane 1 is a constant-bank operand and lane 0 selects 1.
template <int N, int P, int S, typename T>
FFT_HD cx<T> lane_twiddle(cx<T> a, int t, int k2)
{
    if (k2 == 0) return a;
    if constexpr (P == 2) {
        const auto w = Tab<T>::tw(tw_off(N) + k2);
        const T c = t ? w.x : T(1);
        const T s = t ? ((S > 0) ? w.y : -w.y) : T(0);
        return {a.re * c - a.im * s, a.re * s + a.im * c};
    } else {
        return ctwiddle<N, S, T>(a, t * k2);
    }
}

#if defined(__CUDACC__)
// One radix-2 stage of the P-point DFT across the lanes (distance H*LS).
template <int H, int LS, int S, typename T>
__device__ __forceinline__ void xlane_stage_strided(cx<T> &a, int t)
{
    if constexpr (H >= 1) {
        cx<T> b;
        b.re = __shfl_xor_sync(0xffffffffu, a.re, H * LS);
        b.im = __shfl_xor_sync(0xffffffffu, a.im, H * LS);
        const bool hi = (t & H) != 0;
        const T sg = hi ? T(-1) : T(1);  // low lane a + b, high lane b - a
        a = {fma(sg, a.re, b.re), fma(sg, a.im, b.im)};
        if constexpr (H > 1) {
            if (hi) a = ctwiddle<2 * H, S, T>(a, t & (H - 1));
        }
        xlane_stage_strided<H / 2, LS, S, T>(a, t);
    }
}

// Lane t (0 <= t < P) of a line whose lanes are LS apart: load Q points, transform,
// store Q outputs.  Lanes with valid == false exchange zeros and store nothing;
// the P lanes of a line are valid together.
template <int N, int P, int LS, int S, typename T, class Ld, class St>
__device__ __forceinline__ void lane_split_line(int t, bool valid, Ld ld, St st)
{
    using M = LaneSplit<N, P>;
    cx<T> v[M::Q];
#pragma unroll
    for (int n2 = 0; n2 < M::Q; ++n2) v[n2] = valid ? ld(M::in(t, n2)) : cx<T>{T(0), T(0)};
    dft<M::Q, S, T>(v);
    if constexpr (!M::PFA) {
#pragma unroll
        for (int k2 = 1; k2 < M::Q; ++k2) v[k2] = lane_twiddle<N, P, S, T>(v[k2], t, k2);
    }
#pragma unroll
    for (int k2 = 0; k2 < M::Q; ++k2) xlane_stage_strided<P / 2, LS, S, T>(v[k2], t);
    const int k1 = lane_bitrev<P>(t);
    if (valid) {
#pragma unroll
        for (int k2 = 0; k2 < M::Q; ++k2) st(M::out(k1, k2), v[k2]);
    }
}
#endif

// The lane network of xlane_stage on an array a[t] of the P lanes.
template <int H, int P, int S, typename T>
void xlane_stage_host(cx<T> *a)
{
    if constexpr (H >= 1) {
        cx<T> nv[P];
        for (int t = 0; t < P; ++t) {
            const cx<T> b = a[t ^ H];
            const bool hi = (t & H) != 0;
            nv[t] = hi ? csub(b, a[t]) : cadd(a[t], b);
            if constexpr (H > 1) {
                if (hi) nv[t] = ctwiddle<2 * H, S, T>(nv[t], t & (H - 1));
            }
        }
        for (int t = 0; t < P; ++t) a[t] = nv[t];
        xlane_stage_host<H / 2, P, S, T>(a);
    }
}

// The same computation for all P lanes of one line on the host (hostcheck).
template <int N, int S, typename T, class Ld, class St>
void split_line_host(Ld ld, St st)
{
    using SP = LineSplit<N>;
    using M = SplitMap<N>;
    cx<T> v[SP::P][SP::Q];
    for (int t = 0; t < SP::P; ++t) {
        for (int n2 = 0; n2 < SP::Q; ++n2) v[t][n2] = ld(M::in(t, n2));
        dft<SP::Q, S, T>(v[t]);
        if (!SP::PFA)
            for (int k2 = 1; k2 < SP::Q; ++k2) v[t][k2] = ctwiddle<N, S, T>(v[t][k2], t * k2);
    }
    for (int k2 = 0; k2 < SP::Q; ++k2) {
        cx<T> a[SP::P];
        for (int t = 0; t < SP::P; ++t) a[t] = v[t][k2];
        xlane_stage_host<SP::P / 2, SP::P, S, T>(a);
        for (int t = 0; t < SP::P; ++t) v[t][k2] = a[t];
    }
    for (int t = 0; t < SP::P; ++t)
        for (int k2 = 0; k2 < SP::Q; ++k2) st(M::out(lane_bitrev<SP::P>(t), k2), v[t][k2]);
}

// lane_split_line for all P lanes of one line on the host (hostcheck).
template <int N, int P, int S, typename T, class Ld, class St>
void lane_split_line_host(Ld ld, St st)
{
    using M = LaneSplit<N, P>;
    cx<T> v[P][M::Q];
    for (int t = 0; t < P; ++t) {
        for (int n2 = 0; n2 < M::Q; ++n2) v[t][n2] = ld(M::in(t, n2));
        dft<M::Q, S, T>(v[t]);
        if (!M::PFA)
            for (int k2 = 1; k2 < M::Q; ++k2) v[t][k2] = lane_twiddle<N, P, S, T>(v[t][k2], t, k2);
    }
    for (int k2 = 0; k2 < M::Q; ++k2) {
        cx<T> a[P];
        for (int t = 0; t < P; ++t) a[t] = v[t][k2];
        xlane_stage_host<P / 2, P, S, T>(a);
        for (int t = 0; t < P; ++t) v[t][k2] = a[t];
    }
    for (int t = 0; t < P; ++t)
        for (int k2 = 0; k2 < M::Q; ++k2) st(M::out(lane_bitrev<P>(t), k2), v[t][k2]);
}

}  // namespace fft3d

// volume.cuh -- shared-memory layout and the three axis passes of one volume.
//
// The row-column structure of the reference (python/fft3d.py:349-399: a 1D
// transform along every line of each axis in turn) applied to volumes resident
// in one CTA's shared memory.  The functions here are __host__ __device__ so the
// CPU unit tests exercise exactly the index arithmetic the kernels run.
//
// Shared-memory layout of VPC volumes, row r = (vol*N0 + x)*N1 + y holding the
// N2 points of one z-line.  One pass reads each line with one thread, so the
// layout must keep the threads of one access phase on distinct bank groups
// (8 lanes x 16 B for complex double, 16 lanes x 8 B for complex float):
//   POL 0  N2 odd:                     natural, row pitch N2 (odd strides never collide)
//   POL 1  N2 even, not a multiple of the phase width: row pitch N2 + 1
//   POL 2  N2 a multiple of the phase width: pitch N2, point z stored at
//          z ^ (r mod width) -- an XOR swizzle, no padding
#pragma once

#include "codelets.cuh"

namespace fft3d {

//   PITCH > 0 overrides the policy with a plain row pitch (for rows that bulk
//   copies move: their shared-memory start must be 16-byte aligned).
template <int N0_, int N1_, int N2_, typename T_, int PITCH = 0>
struct Geom {
    using T = T_;
    static constexpr int N0 = N0_, N1 = N1_, N2 = N2_;
    static constexpr int V = N0 * N1 * N2;
    static constexpr int ROWS = N0 * N1;
    static constexpr int EB = 2 * (int)sizeof(T);
    static constexpr int GROUP = (EB == 16) ? 8 : 16;
    static_assert(PITCH == 0 || PITCH >= N2, "row pitch below the row length");
    static constexpr int POL = PITCH > 0 ? 1 : (N2 % 2 == 1) ? 0 : ((N2 % GROUP == 0) ? 2 : 1);
    static constexpr int P2 = PITCH > 0 ? PITCH : (POL == 1) ? N2 + 1 : N2;
    static constexpr int PV = ROWS * P2;  // shared-memory elements per volume

    FFT_HD static int off(int r, int z)
    {
        if constexpr (POL == 2) return r * N2 + (z ^ (r & (GROUP - 1)));
        else return r * P2 + z;
    }
};

// Pass along z for row r (lines are rows).
template <class G, int S, int ALG>
FFT_HD void pass_z(cx<typename G::T> *sm, int r)
{
    using T = typename G::T;
    cx<T> v[G::N2];
#pragma unroll
    for (int j = 0; j < G::N2; ++j) v[j] = sm[G::off(r, j)];
    dft<G::N2, S, T, ALG>(v);
#pragma unroll
    for (int j = 0; j < G::N2; ++j) sm[G::off(r, j)] = v[j];
}

// Pass along z for row r read straight from HBM: rows are contiguous in the
// input (row r of the CTA's slice starts at element r*N2), so a thread streams
// its N2 points with back-to-back vector loads and the transform needs no
// staging copy; the result goes to the shared-memory layout.
template <class G, int S, int ALG>
FFT_HD void pass_z_from_global(cx<typename G::T> *sm, const cx<typename G::T> *gin, int r)
{
    using T = typename G::T;
    cx<T> v[G::N2];
    const cx<T> *p = gin + (long long)r * G::N2;
#pragma unroll
    for (int j = 0; j < G::N2; ++j) v[j] = load_in(p + j);
    dft<G::N2, S, T, ALG>(v);
#pragma unroll
    for (int j = 0; j < G::N2; ++j) sm[G::off(r, j)] = v[j];
}

// Pass along y for line l = (vol*N0 + x)*N2 + z.
template <class G, int S, int ALG>
FFT_HD void pass_y(cx<typename G::T> *sm, int l)
{
    using T = typename G::T;
    const int z = l % G::N2;
    const int rb = (l / G::N2) * G::N1;
    cx<T> v[G::N1];
#pragma unroll
    for (int j = 0; j < G::N1; ++j) v[j] = sm[G::off(rb + j, z)];
    dft<G::N1, S, T, ALG>(v);
#pragma unroll
    for (int j = 0; j < G::N1; ++j) sm[G::off(rb + j, z)] = v[j];
}

// Pass along x for line l = (vol*N1 + y)*N2 + z, read from shared memory and
// written straight to the output volume: consecutive l are consecutive (y, z),
// so each store instruction of a warp covers a contiguous range.
template <typename T>
FFT_HD void store_out(cx<T> *p, cx<T> v)
{
#if defined(__CUDA_ARCH__)
    if constexpr (sizeof(T) == 8) {
        __stcs(reinterpret_cast<double2 *>(p), make_double2(v.re, v.im));
    } else {
        __stcs(reinterpret_cast<float2 *>(p), make_float2(v.re, v.im));
    }
#else
    *p = v;
#endif
}

template <typename T>
FFT_HD cx<T> load_in(const cx<T> *p)
{
#if defined(__CUDA_ARCH__)
    if constexpr (sizeof(T) == 8) {
        const double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
        return {t.x, t.y};
    } else {
        const float2 t = __ldcs(reinterpret_cast<const float2 *>(p));
        return {t.x, t.y};
    }
#else
    return *p;
#endif
}

// x lines of a prime length above 31 (47, 83 and 97 among the reference's test
// extents): a folded sum held in registers would spill kilobytes a thread, so
// the line is summed straight out of shared memory, one output at a time, with
// double twiddles and accumulators; only x-pass lines are that long.
constexpr bool x_direct_sum(int n) { return ce_is_prime(n) && n > 31; }

template <class G, int S, bool KEEP>
FFT_HD void pass_x_out_direct(const cx<typename G::T> *sm, int l, cx<typename G::T> *gout,
                              typename G::T scale)
{
    using T = typename G::T;
    constexpr int N = G::N0;
    const int z = l % G::N2;
    const int t = l / G::N2;
    const int y = t % G::N1;
    const int vol = t / G::N1;
    cx<T> *o = gout + (long long)vol * G::V + y * G::N2 + z;
    for (int k = 0; k < N; ++k) {
        double ar = 0.0, ai = 0.0;
        int e = 0;  // j * k mod N
        for (int j = 0; j < N; ++j) {
            const cx<T> x = sm[G::off((vol * N + j) * G::N1 + y, z)];
            const auto w = line_tw<N, double>(e);  // {cos, sin}(2*pi*e/N)
            const double sn = S > 0 ? w.y : -w.y;
            ar += (double)x.re * w.x - (double)x.im * sn;
            ai += (double)x.re * sn + (double)x.im * w.x;
            e += k;
            if (e >= N) e -= N;
        }
        cx<T> r = {(T)ar, (T)ai};
        if constexpr (S > 0) r = cscale(r, scale);
        if constexpr (KEEP) o[k * (G::N1 * G::N2)] = r;
        else store_out(o + k * (G::N1 * G::N2), r);
    }
}

// KEEP: plain stores instead of streaming (evict-first) ones, for outputs that
// a following transform may still find in L2.
template <class G, int S, int ALG, bool KEEP = false>
FFT_HD void pass_x_out(const cx<typename G::T> *sm, int l, cx<typename G::T> *gout,
                       typename G::T scale)
{
    using T = typename G::T;
    if constexpr (x_direct_sum(G::N0)) {
        pass_x_out_direct<G, S, KEEP>(sm, l, gout, scale);
    } else {
        const int z = l % G::N2;
        const int t = l / G::N2;
        const int y = t % G::N1;
        const int vol = t / G::N1;
        cx<T> v[G::N0];
#pragma unroll
        for (int j = 0; j < G::N0; ++j) v[j] = sm[G::off((vol * G::N0 + j) * G::N1 + y, z)];
        dft<G::N0, S, T, ALG>(v);
        cx<T> *o = gout + (long long)vol * G::V + y * G::N2 + z;
#pragma unroll
        for (int j = 0; j < G::N0; ++j) {
            cx<T> r = v[j];
            if constexpr (S > 0) r = cscale(r, scale);
            if constexpr (KEEP) o[j * (G::N1 * G::N2)] = r;
            else store_out(o + j * (G::N1 * G::N2), r);
        }
    }
}

// Pass along x for line l = (vol*N1 + y)*N2 + z in place in shared memory,
// scaled for the inverse: for kernels that move the finished stage to HBM with
// one bulk copy instead of storing from registers.
template <class G, int S, int ALG>
FFT_HD void pass_x(cx<typename G::T> *sm, int l, typename G::T scale)
{
    static_assert(!x_direct_sum(G::N0), "long prime x lines are summed out of shared memory");
    using T = typename G::T;
    const int z = l % G::N2;
    const int t = l / G::N2;
    const int y = t % G::N1;
    const int vol = t / G::N1;
    cx<T> v[G::N0];
#pragma unroll
    for (int j = 0; j < G::N0; ++j) v[j] = sm[G::off((vol * G::N0 + j) * G::N1 + y, z)];
    dft<G::N0, S, T, ALG>(v);
#pragma unroll
    for (int j = 0; j < G::N0; ++j) {
        cx<T> r = v[j];
        if constexpr (S > 0) r = cscale(r, scale);
        sm[G::off((vol * G::N0 + j) * G::N1 + y, z)] = r;
    }
}

// Pass along x for line l into registers (scaled for the inverse), and the
// matching store of the line at its natural (unpadded, unswizzled) place in the
// same buffer.  Kernels with padded or swizzled layouts and one x line per
// thread run the first for every line, wait at a barrier (a natural slot may
// hold a point another thread has not read yet), then the second, and move the
// natural-layout stage to HBM with one bulk copy.
template <class G, int S, int ALG>
FFT_HD void pass_x_regs(const cx<typename G::T> *sm, int l, typename G::T scale,
                        cx<typename G::T> (&v)[G::N0])
{
    static_assert(!x_direct_sum(G::N0), "long prime x lines are summed out of shared memory");
    const int z = l % G::N2;
    const int t = l / G::N2;
    const int y = t % G::N1;
    const int vol = t / G::N1;
#pragma unroll
    for (int j = 0; j < G::N0; ++j) v[j] = sm[G::off((vol * G::N0 + j) * G::N1 + y, z)];
    dft<G::N0, S, typename G::T, ALG>(v);
    if constexpr (S > 0) {
#pragma unroll
        for (int j = 0; j < G::N0; ++j) v[j] = cscale(v[j], scale);
    }
}

template <class G>
FFT_HD void store_x_natural(cx<typename G::T> *sm, int l, const cx<typename G::T> (&v)[G::N0])
{
    const int zy = l % (G::N1 * G::N2);  // y*N2 + z
    const int vol = l / (G::N1 * G::N2);
#pragma unroll
    for (int j = 0; j < G::N0; ++j) sm[vol * G::V + j * (G::N1 * G::N2) + zy] = v[j];
}

// Chain-step epilogues applied to each output point of the last pass.
constexpr int EPI_UNITARY = 1;  // state <- FFT(state) * V^(-1/2)
constexpr int EPI_MAP = 2;      // z = FFT(state) + c;  state <- z / (1 + |z|)

template <int EPI, typename T>
FFT_HD cx<T> chain_epilogue(cx<T> r, const cx<T> *cmap, long long e, T uscale)
{
    if constexpr (EPI == EPI_UNITARY) {
        return cscale(r, uscale);
    } else {
        const cx<T> c = cmap[e];
        const T re = r.re + c.re, im = r.im + c.im;
        const T s = T(1) / (T(1) + std::sqrt(re * re + im * im));
        return {re * s, im * s};
    }
}

// Pass along x for line l = (vol*N1 + y)*N2 + z with the chain epilogue, result
// written back into the shared-memory layout (the state stays on chip between
// chain steps).  `e0` is the global element index of the CTA's first volume.
template <class G, int ALG, int EPI>
FFT_HD void pass_x_chain(cx<typename G::T> *sm, int l, const cx<typename G::T> *cmap, long long e0,
                         typename G::T uscale)
{
    using T = typename G::T;
    const int z = l % G::N2;
    const int t = l / G::N2;
    const int y = t % G::N1;
    const int vol = t / G::N1;
    cx<T> v[G::N0];
#pragma unroll
    for (int j = 0; j < G::N0; ++j) v[j] = sm[G::off((vol * G::N0 + j) * G::N1 + y, z)];
    dft<G::N0, -1, T, ALG>(v);
    const long long eb = e0 + (long long)vol * G::V + y * G::N2 + z;
#pragma unroll
    for (int j = 0; j < G::N0; ++j)
        sm[G::off((vol * G::N0 + j) * G::N1 + y, z)] =
            chain_epilogue<EPI>(v[j], cmap, eb + (long long)j * (G::N1 * G::N2), uscale);
}

// Pass along x over a y-slab held as an (N0, YS, N2) block G, written into a
// volume whose y extent is GN1, at y offset y0 (two-phase large cubes).
template <class G, int S, int GN1>
FFT_HD void pass_x_slab(const cx<typename G::T> *sm, int l, cx<typename G::T> *gvol, int y0,
                        typename G::T scale)
{
    using T = typename G::T;
    const int z = l % G::N2;
    const int y = l / G::N2;  // 0 .. YS-1
    cx<T> v[G::N0];
#pragma unroll
    for (int j = 0; j < G::N0; ++j) v[j] = sm[G::off(j * G::N1 + y, z)];
    dft<G::N0, S, T>(v);
#pragma unroll
    for (int j = 0; j < G::N0; ++j) {
        cx<T> r = v[j];
        if constexpr (S > 0) r = cscale(r, scale);
        store_out(gvol + ((long long)j * GN1 + y0 + y) * G::N2 + z, r);
    }
}

// L2-only accesses, for buffers that other SMs write during the launch (the
// per-SM L1 is not coherent with them).  Plain accesses on the host.
template <typename T>
FFT_HD void store_l2(cx<T> *p, cx<T> v)
{
#if defined(__CUDA_ARCH__)
    if constexpr (sizeof(T) == 8) __stcg(reinterpret_cast<double2 *>(p), make_double2(v.re, v.im));
    else __stcg(reinterpret_cast<float2 *>(p), make_float2(v.re, v.im));
#else
    *p = v;
#endif
}

template <typename T>
FFT_HD cx<T> load_l2(const cx<T> *p)
{
#if defined(__CUDA_ARCH__)
    if constexpr (sizeof(T) == 8) {
        const double2 t = __ldcg(reinterpret_cast<const double2 *>(p));
        return {t.x, t.y};
    } else {
        const float2 t = __ldcg(reinterpret_cast<const float2 *>(p));
        return {t.x, t.y};
    }
#else
    return *p;
#endif
}

// Pass along y for line l = g*N2 + z of a block of planes G = (planes, N1, N2)
// in shared memory, written straight to a volume-shaped buffer whose plane g
// is plane x0 + g, with L2-only stores.  Consecutive l are consecutive z, so
// each store instruction of a warp covers contiguous ranges.
template <class G, int S>
FFT_HD void pass_y_store_l2(const cx<typename G::T> *sm, int l, cx<typename G::T> *gvol, int x0)
{
    using T = typename G::T;
    const int z = l % G::N2;
    const int g = l / G::N2;
    cx<T> v[G::N1];
#pragma unroll
    for (int j = 0; j < G::N1; ++j) v[j] = sm[G::off(g * G::N1 + j, z)];
    dft<G::N1, S, T>(v);
    cx<T> *o = gvol + (long long)(x0 + g) * G::N1 * G::N2 + z;
#pragma unroll
    for (int j = 0; j < G::N1; ++j) store_l2(o + j * G::N2, v[j]);
}

// Pass along x for line l of y-rows [y0, ...) of an N0 x N1 x N2 volume-shaped
// buffer, read straight from it with L2-only loads (line l is the point
// (y0*N2 + l) of every plane: consecutive l are consecutive addresses) and
// streamed to gvol at the same offsets.
template <int N0, int N1, int N2, int S, typename T>
FFT_HD void pass_x_load_l2(const cx<T> *src, int l, cx<T> *gvol, int y0, T scale)
{
    constexpr long long PLANE = (long long)N1 * N2;
    const long long e = (long long)y0 * N2 + l;
    cx<T> v[N0];
#pragma unroll
    for (int j = 0; j < N0; ++j) v[j] = load_l2(src + j * PLANE + e);
    dft<N0, S, T>(v);
#pragma unroll
    for (int j = 0; j < N0; ++j) {
        cx<T> r = v[j];
        if constexpr (S > 0) r = cscale(r, scale);
        store_out(gvol + j * PLANE + e, r);
    }
}

// Copy element g (in [0, nv*V)) of the CTA's input slice into its layout slot.
template <class G>
FFT_HD void stage_in(cx<typename G::T> *sm, const cx<typename G::T> *gin, int g)
{
    const int vol = g / G::V;
    const int rem = g - vol * G::V;
    const int r = vol * G::ROWS + rem / G::N2;
    const int z = rem % G::N2;
    sm[G::off(r, z)] = load_in(gin + g);
}

}  // namespace fft3d

// staged.cuh -- long lines as two thread-level stages through shared memory
// (host and device): the line policies of the staged TWOPASS kernel.
//
// A 64-point complex-double line held by one thread needs 256 registers for its
// data alone, a 45-point one 180: one-thread-per-line kernels spill or run a
// handful of warps per SM.  Splitting N = A x B gives independent tasks:
//   stage 1, task (line, b): the A-point DFT over the A points of residue
//            class b, stored back into the same slots;
//   stage 2, task (line, a): the B-point DFT over the B points of class a,
//            producing B outputs of the line.
// A task holds A or B points, and each stage reads and writes only its own
// slots of the line, so both stages work in place with a CTA barrier between
// them.  Stored in place, stage 2 leaves output k in slot slot(k); at(p) is
// the output index held in slot p.  Callers that store elsewhere get the
// natural index k.  Tasks are numbered line-fastest: the lanes of a warp share
// the residue class, so twiddle indices are warp-uniform and consecutive lanes
// touch consecutive lines.
#pragma once

#include "codelets.cuh"

namespace fft3d {

// 64 = 8 x 8 Cooley-Tukey, decimation in time (the mixed-radix route of the
// reference's python/fft3d.py:166-188): x[8 n1 + n2]; stage 1 multiplies by
// W64^(n2 k1); X[k1 + 8 k2] lands in slot 8 k1 + k2 (digit-reversed, an
// involution).
struct LineCT64 {
    static constexpr int N = 64, T1 = 8, T2 = 8;
    FFT_HD static constexpr int slot(int k) { return 8 * (k % 8) + k / 8; }
    FFT_HD static constexpr int at(int p) { return 8 * (p % 8) + p / 8; }

    template <int S, typename T, class Addr>
    FFT_HD static void stage1(cx<T> *sm, int lines, int t, Addr addr)
    {
        const int line = t % lines, n2 = t / lines;
        cx<T> v[8];
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) v[n1] = sm[addr(line, 8 * n1 + n2)];
        dft<8, S, T>(v);
#pragma unroll
        for (int k1 = 1; k1 < 8; ++k1) {
            const auto w = Tab<T>::tw(tw_off(64) + n2 * k1);  // {cos, sin}(2 pi n2 k1 / 64), n2 k1 < 64
            const T c = w.x, s = (S > 0) ? w.y : -w.y;
            v[k1] = {v[k1].re * c - v[k1].im * s, v[k1].re * s + v[k1].im * c};
        }
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) sm[addr(line, 8 * k1 + n2)] = v[k1];
    }

    template <int S, typename T, class Addr, class Store>
    FFT_HD static void stage2(const cx<T> *sm, int lines, int t, Addr addr, Store store)
    {
        const int line = t % lines, k1 = t / lines;
        cx<T> v[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) v[n2] = sm[addr(line, 8 * k1 + n2)];
        dft<8, S, T>(v);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) store(line, k1 + 8 * k2, v[k2]);
    }
};

// 45 = 5 x 9 Good-Thomas (no twiddles; the prime-factor route of
// python/fft3d.py:166-188 with coprime factors): x at slot (9 n1 + 5 n2) mod 45,
// X[(36 k1 + 10 k2) mod 45] (36 = 9 * (9^-1 mod 5), 10 = 5 * (5^-1 mod 9)), so
// that n k = 9 n1 k1 + 5 n2 k2 (mod 45).  Stage 1 (5-point DFTs, class n2)
// stores a[k1][n2] at slot (9 k1 + 5 n2) mod 45; stage 2 (9-point DFTs, class
// k1) puts X[(36 k1 + 10 k2) mod 45] in place at slot (9 k1 + 5 k2) mod 45.
struct LinePFA45 {
    static constexpr int N = 45, T1 = 9, T2 = 5;
    // output k: k1 = k mod 5, k2 = k mod 9
    FFT_HD static constexpr int slot(int k) { return (9 * (k % 5) + 5 * (k % 9)) % 45; }
    // slot p: k1 = 4 (p mod 5) mod 5, k2 = 2 (p mod 9) mod 9 (4 = 9^-1 mod 5, 2 = 5^-1 mod 9)
    FFT_HD static constexpr int at(int p) { return (36 * ((4 * (p % 5)) % 5) + 10 * ((2 * (p % 9)) % 9)) % 45; }

    template <int S, typename T, class Addr>
    FFT_HD static void stage1(cx<T> *sm, int lines, int t, Addr addr)
    {
        const int line = t % lines, n2 = t / lines;
        const int b = 5 * n2;  // < 45
        cx<T> v[5];
#pragma unroll
        for (int n1 = 0; n1 < 5; ++n1) {
            int e = 9 * n1 + b;
            e = e >= 45 ? e - 45 : e;
            v[n1] = sm[addr(line, e)];
        }
        dft<5, S, T>(v);
#pragma unroll
        for (int k1 = 0; k1 < 5; ++k1) {
            int e = 9 * k1 + b;
            e = e >= 45 ? e - 45 : e;
            sm[addr(line, e)] = v[k1];
        }
    }

    template <int S, typename T, class Addr, class Store>
    FFT_HD static void stage2(const cx<T> *sm, int lines, int t, Addr addr, Store store)
    {
        const int line = t % lines, k1 = t / lines;
        const int a = 9 * k1;  // < 45
        cx<T> v[9];
#pragma unroll
        for (int n2 = 0; n2 < 9; ++n2) {
            int e = a + 5 * n2;
            e = e >= 45 ? e - 45 : e;
            v[n2] = sm[addr(line, e)];
        }
        dft<9, S, T>(v);
#pragma unroll
        for (int k2 = 0; k2 < 9; ++k2) store(line, (36 * k1 + 10 * k2) % 45, v[k2]);
    }
};

}  // namespace fft3d

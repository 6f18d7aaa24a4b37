// pfa36.cuh -- 36-point lines as two thread-level stages through shared memory
// (host and device).
//
// A 36-point complex-double line held by one thread needs about 170 registers,
// which caps a kernel at 12 warps per SM.  Good-Thomas (36 = 4 x 9, no
// twiddles between the factors; the prime-factor route of the reference's
// bench/geom/best/kernels/L36_mixedradix.c:9-18) splits it into independent
// tasks: stage 1 runs the 4-point DFTs (one task per line and n2), stage 2 the
// 9-point DFTs (one task per line and k1), each task loading its points from
// shared memory and storing them back, with a CTA barrier between the stages.
// A task holds 4 or 9 points, so the kernel fits in ~85 registers per thread.
//
// Index maps (n = input index, k = output index of the line):
//   n = (9 n1 + 4 n2) mod 36,   k = (9 k1 + 28 k2) mod 36,
// so that n k = 9 n1 k1 + 4 n2 k2 (mod 36): w36^(nk) = w4^(n1 k1) w9^(n2 k2).
// Stage 1 writes a[k1][n2] back into the slot of x[n1 = k1][n2]; stage 2 reads
// the 9 slots {(9 k1 + 4 n2) mod 36} and writes X[(9 k1 + 28 k2) mod 36] -- the
// same 9 slots, since 28 = 4 * 7 and 7 is invertible mod 9 -- so both stages
// work in place and tasks of one stage never touch one another's slots.
//
// Tasks are numbered line-fastest, so the lanes of a warp work on consecutive
// lines with the same (n2 or k1): with line addresses at an odd stride or at
// consecutive elements, every access phase is free of bank conflicts.
#pragma once

#include "codelets.cuh"

namespace fft3d {

FFT_HD constexpr int pfa36_slot(int a, int b) { return (9 * a + 4 * b) % 36; }  // x[a][b], a[k1=a][b]
FFT_HD constexpr int pfa36_out(int k1, int k2) { return (9 * k1 + 28 * k2) % 36; }

// Stage 1 over `lines` lines: task t = n2 * lines + line.  addr(line, e) is
// the shared-memory index of element e of the line.
template <int S, typename T, class Addr>
FFT_HD void pfa36_stage1(cx<T> *sm, int lines, int t, Addr addr)
{
    const int line = t % lines, n2 = t / lines;
    const int b = 4 * n2;  // < 36
    cx<T> v[4];
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) {
        int e = 9 * n1 + b;
        e = e >= 36 ? e - 36 : e;
        v[n1] = sm[addr(line, e)];
    }
    dft<4, S, T>(v);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        int e = 9 * k1 + b;
        e = e >= 36 ? e - 36 : e;
        sm[addr(line, e)] = v[k1];
    }
}

// Stage 2: task t = k1 * lines + line; store(line, k, value) receives output k.
template <int S, typename T, class Addr, class Store>
FFT_HD void pfa36_stage2(const cx<T> *sm, int lines, int t, Addr addr, Store store)
{
    const int line = t % lines, k1 = t / lines;
    const int a = 9 * k1;  // < 36
    cx<T> v[9];
#pragma unroll
    for (int n2 = 0; n2 < 9; ++n2) {
        int e = a + (4 * n2) % 36;
        e = e >= 36 ? e - 36 : e;
        v[n2] = sm[addr(line, e)];
    }
    dft<9, S, T>(v);
#pragma unroll
    for (int k2 = 0; k2 < 9; ++k2) {
        int k = a + (28 * k2) % 36;
        k = k >= 36 ? k - 36 : k;
        store(line, k, v[k2]);
    }
}

}  // namespace fft3d

// ct64.cuh -- 64-point lines as two thread-level stages through shared memory
// (host and device).
//
// A 64-point complex-double line held by one thread needs 256 registers for
// its data alone, so a one-thread-per-line kernel spills heavily.  Cooley-Tukey
// with 64 = 8 x 8 (decimation in time, the mixed-radix route of the
// reference's python/fft3d.py:166-188) splits it into independent tasks:
//   stage 1, task (line, n2): the 8-point DFT over n1 of x[8 n1 + n2], times
//            the twiddle W64^(n2 k1), stored back into the slots 8 k1 + n2;
//   stage 2, task (line, k1): the 8-point DFT over n2 of those slots, giving
//            X[k1 + 8 k2] for k2 = 0..7.
// A task holds 8 points (about 40 registers), and each stage reads and writes
// only its own 8 slots of the line, so both stages work in place with a CTA
// barrier between them.  Stored in place, stage 2 leaves X[k] in slot
// ct64_slot(k) = 8 (k mod 8) + k / 8 (digit-reversed; the map is its own
// inverse); callers that store elsewhere get the natural index k.
//
// Tasks are numbered line-fastest: the lanes of a warp share n2 (or k1), so the
// twiddle index is warp-uniform (a constant-cache broadcast) and consecutive
// lanes touch consecutive lines.
#pragma once

#include "codelets.cuh"

namespace fft3d {

FFT_HD constexpr int ct64_slot(int k) { return 8 * (k % 8) + k / 8; }

// Stage 1 over `lines` lines: task t = n2 * lines + line; addr(line, e) is the
// shared-memory index of element e of the line.
template <int S, typename T, class Addr>
FFT_HD void ct64_stage1(cx<T> *sm, int lines, int t, Addr addr)
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

// Stage 2: task t = k1 * lines + line; store(line, k, value) receives output k.
template <int S, typename T, class Addr, class Store>
FFT_HD void ct64_stage2(const cx<T> *sm, int lines, int t, Addr addr, Store store)
{
    const int line = t % lines, k1 = t / lines;
    cx<T> v[8];
#pragma unroll
    for (int n2 = 0; n2 < 8; ++n2) v[n2] = sm[addr(line, 8 * k1 + n2)];
    dft<8, S, T>(v);
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) store(line, k1 + 8 * k2, v[k2]);
}

}  // namespace fft3d

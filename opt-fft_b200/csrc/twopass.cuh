// twopass.cuh -- work decomposition of the TWOPASS family (host and device).
//
// A volume too large for one SM's shared memory is transformed in two kinds of
// work item of the same size:
//   plane item (v, j): x-planes [j*G, (j+1)*G) of volume v -- contiguous in the
//       input -- through the z and y passes, written to scratch slot v % R;
//   row item (v, j):   y-rows [j*G, (j+1)*G) of every x-plane of scratch slot
//       v % R through the x pass, written to the output.
// Items are handed out by one atomic ticket in steps: step s holds the NA plane
// items of volume s, then the NB row items of volume s - D.  A row item waits
// for the plane items of its volume (D steps earlier); a plane item that reuses
// a slot waits for the row items of the slot's previous volume (step v - R + D,
// earlier because D < R).  Every wait is on a smaller ticket, which a running
// CTA holds, so the order cannot deadlock.  With D about two grids' worth of
// tickets (twopass_ring), the waits are normally satisfied on arrival, and the ring of R
// volumes is small enough to stay in L2, so the intermediate costs no HBM
// traffic: each volume is read from HBM once and written once.
#pragma once

#include "internal.h"
#include "volume.cuh"

namespace fft3d {

template <int N0, int N1, int N2, typename T, int G, int PITCH = 0>
struct TwoPassGeom {
    static_assert(N0 % G == 0 && N1 % G == 0, "planes and rows per item must divide n0, n1");
    using XG = Geom<G, N1, N2, T, PITCH>;   // plane item: G planes of N1 x N2
    using YG = Geom<N0, G, N2, T, PITCH>;   // row item: G rows (y) of all N0 planes
    static constexpr int N1F = N1;  // full y extent
    static constexpr int NA = N0 / G;
    static constexpr int NB = N1 / G;
    static constexpr long long V = (long long)N0 * N1 * N2;
    static constexpr int PV = XG::PV > YG::PV ? XG::PV : YG::PV;
    static constexpr int SMEM = ((PV * XG::EB) + 127) / 128 * 128;
    static constexpr int PLANE_ELEMS = G * N1 * N2;  // elements of a plane item
    static constexpr int ROW_ELEMS = N0 * G * N2;    // elements of a row item
};

// The 128-byte lines of scratch that a row item (v, j) may drop from L2 once
// it has read its rows for the last time: in each x-plane x, the whole lines
// inside its G consecutive y-rows [j*G, (j+1)*G) (a line shared with a
// neighbouring item's rows is kept -- that item may not have read it yet).
// Line index q runs over [0, N0 * twopass_row_lines_per_plane<TG>()); false
// when q names no whole line.
template <class TG>
FFT_HD constexpr int twopass_row_lines_per_plane()
{
    return TG::YG::N1 * TG::YG::N2 * TG::XG::EB / 128 + 1;
}

template <class TG>
FFT_HD bool twopass_row_line(const void *slot, int j, int q, uintptr_t *line)
{
    constexpr int G = TG::YG::N1, N2 = TG::YG::N2, PER = twopass_row_lines_per_plane<TG>();
    constexpr long long EB = TG::XG::EB;
    const int x = q / PER, k = q % PER;
    const uintptr_t a = (uintptr_t)slot + (uintptr_t)(((long long)x * TG::N1F + (long long)j * G) * N2 * EB);
    const uintptr_t first = (a + 127) & ~(uintptr_t)127;
    *line = first + (uintptr_t)k * 128;
    return *line + 128 <= a + (uintptr_t)(G * N2 * EB);
}

struct TwoPassItem {
    bool plane;
    long long vol;
    int j;
};

// Ticket t -> item, for nvol volumes, NA plane and NB row items per volume, lag D.
FFT_HD TwoPassItem twopass_decode(long long t, long long nvol, int na, int nb, int lag)
{
    TwoPassItem it;
    const long long A = na, B = nb, AB = A + B, D = lag;
    if (nvol <= D) {
        if (t < A * nvol) {
            it.plane = true, it.vol = t / A, it.j = (int)(t % A);
        } else {
            t -= A * nvol;
            it.plane = false, it.vol = t / B, it.j = (int)(t % B);
        }
        return it;
    }
    if (t < A * D) {  // steps 0 .. D-1: plane items only
        it.plane = true, it.vol = t / A, it.j = (int)(t % A);
        return it;
    }
    t -= A * D;
    const long long mid = AB * (nvol - D);
    if (t < mid) {  // steps D .. nvol-1
        const long long s = D + t / AB;
        const int r = (int)(t % AB);
        if (r < na) it.plane = true, it.vol = s, it.j = r;
        else it.plane = false, it.vol = s - D, it.j = r - na;
        return it;
    }
    t -= mid;  // steps nvol .. nvol+D-1: row items only
    it.plane = false, it.vol = nvol - D + t / B, it.j = (int)(t % B);
    return it;
}

// Ring geometry for `held` tickets in flight: D = their worth of steps + 2, R = 2D + 2.
FFT_HD int twopass_ring_size(int na, int nb, long long held, int *lag)
{
    const long long ab = na + nb;
    long long d = (held + ab - 1) / ab + 2;
    const long long dmax = (TWOPASS_RMAX - 2) / 2;
    if (d > dmax) d = dmax;
    *lag = (int)d;
    return (int)(2 * d + 2);
}

// Element g of a plane item: source/destination offset within the volume and
// slot in the XG layout.
template <class TG>
FFT_HD void twopass_plane_elem(int j, int g, long long *vo, int *so)
{
    constexpr int N1 = TG::XG::N1, N2 = TG::XG::N2, G = TG::XG::N0;
    *vo = (long long)j * G * N1 * N2 + g;
    *so = TG::XG::off(g / N2, g % N2);
}

// Element g of a row item (g = (x*G + yl)*N2 + z): scratch offset and YG slot.
template <class TG>
FFT_HD void twopass_row_elem(int j, int g, long long *vo, int *so)
{
    constexpr int G = TG::YG::N1, N2 = TG::YG::N2;
    const int z = g % N2, row = g / N2;  // row = x*G + yl
    const int x = row / G, yl = row % G;
    *vo = ((long long)x * TG::N1F + (long long)j * G + yl) * N2 + z;
    *so = TG::YG::off(row, z);
}

}  // namespace fft3d

// hostcheck.cpp -- CPU execution of the kernels' pass code, for unit tests only.
//
// Test infrastructure: built into build/libfft3d_hostcheck.so, loaded only by
// tests/, never linked into libfft3d_b200.so.  It runs the very functions the
// VOLUME kernels run (stage_in, pass_z, pass_y, pass_x_out of volume.cuh, the
// codelets of codelets.cuh, the layouts of Geom), one "thread" after another and
// one CTA after another, so the index arithmetic, the shared-memory layouts and
// every codelet are checked against the oracle without a GPU.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "staged.cuh"
#include "mgpu.cuh"
#include "splitline.cuh"
#include "twopass.cuh"
#include "volume.cuh"

namespace fft3d {
void ensure_host_tables();
}

using namespace fft3d;

template <int N0, int N1, int N2, typename T, int S, int ALG, int VPC>
static void emulate(const void *vin, void *vout, long long nvol)
{
    using G = Geom<N0, N1, N2, T>;
    const cx<T> *in = (const cx<T> *)vin;
    cx<T> *out = (cx<T> *)vout;
    std::vector<cx<T>> sm((size_t)VPC * G::PV);
    const T scale = S > 0 ? T(1) / T(G::V) : T(1);
    for (long long v0 = 0; v0 < nvol; v0 += VPC) {
        const int nv = (int)((nvol - v0) < VPC ? (nvol - v0) : VPC);
        // poison the layout so a slot the kernels never write would show up
        for (auto &e : sm) e = {T(12345.0), T(-6789.0)};
        for (int g = 0; g < nv * G::V; ++g) stage_in<G>(sm.data(), in + v0 * G::V, g);
        for (int r = 0; r < nv * G::ROWS; ++r) pass_z<G, S, ALG>(sm.data(), r);
        for (int l = 0; l < nv * G::N0 * G::N2; ++l) pass_y<G, S, ALG>(sm.data(), l);
        for (int l = 0; l < nv * G::N1 * G::N2; ++l)
            pass_x_out<G, S, ALG>(sm.data(), l, out + v0 * G::V, scale);
    }
}

// The STREAM kernel's bulk-store item (BST): the x pass leaves the stage in
// natural layout (in place for natural layouts; padded and swizzled ones read
// every line into registers before any line is stored at its natural place),
// then the stage is copied to the output as one block.
template <int N0, int N1, int N2, typename T, int S, int ALG, int VPC>
static void emulate_bst(const void *vin, void *vout, long long nvol)
{
    using G = Geom<N0, N1, N2, T>;
    struct Line {
        cx<T> v[N0];
    };
    const cx<T> *in = (const cx<T> *)vin;
    cx<T> *out = (cx<T> *)vout;
    std::vector<cx<T>> sm((size_t)VPC * G::PV);
    const T scale = S > 0 ? T(1) / T(G::V) : T(1);
    for (long long v0 = 0; v0 < nvol; v0 += VPC) {
        const int nv = (int)((nvol - v0) < VPC ? (nvol - v0) : VPC);
        for (auto &e : sm) e = {T(12345.0), T(-6789.0)};
        for (int g = 0; g < nv * G::V; ++g) stage_in<G>(sm.data(), in + v0 * G::V, g);
        for (int r = 0; r < nv * G::ROWS; ++r) pass_z<G, S, ALG>(sm.data(), r);
        for (int l = 0; l < nv * G::N0 * G::N2; ++l) pass_y<G, S, ALG>(sm.data(), l);
        if constexpr (G::POL == 0) {
            for (int l = 0; l < nv * G::N1 * G::N2; ++l) pass_x<G, S, ALG>(sm.data(), l, scale);
        } else {
            std::vector<Line> regs((size_t)nv * G::N1 * G::N2);
            for (int l = 0; l < nv * G::N1 * G::N2; ++l)
                pass_x_regs<G, S, ALG>(sm.data(), l, scale, regs[l].v);
            for (int l = 0; l < nv * G::N1 * G::N2; ++l) store_x_natural<G>(sm.data(), l, regs[l].v);
        }
        std::copy(sm.begin(), sm.begin() + (size_t)nv * G::V, out + v0 * G::V);
    }
}

// The CLUSTER kernel's data movement: C slabs of PL = N0/C planes, local z and y
// passes, x lines split n1*n2/C per rank and gathered from the owning slabs.
template <int N0, int N1, int N2, typename T, int S, int C>
static void emulate_cluster(const void *vin, void *vout, long long nvol)
{
    constexpr int PL = N0 / C;
    using SG = Geom<PL, N1, N2, T>;
    constexpr int V = N0 * N1 * N2;
    constexpr int LPC = N1 * N2 / C;
    const cx<T> *in = (const cx<T> *)vin;
    cx<T> *out = (cx<T> *)vout;
    const T scale = S > 0 ? T(1) / T(V) : T(1);
    std::vector<std::vector<cx<T>>> slab(C, std::vector<cx<T>>(SG::PV));
    for (long long vol = 0; vol < nvol; ++vol) {
        for (int rank = 0; rank < C; ++rank) {
            cx<T> *sm = slab[rank].data();
            for (auto &e : slab[rank]) e = {T(12345.0), T(-6789.0)};
            const cx<T> *gin = in + vol * V + (long long)rank * PL * N1 * N2;
            for (int g = 0; g < PL * N1 * N2; ++g) sm[SG::off(g / N2, g % N2)] = gin[g];
            for (int r = 0; r < PL * N1; ++r) pass_z<SG, S, ALG_DEFAULT>(sm, r);
            for (int l = 0; l < PL * N2; ++l) pass_y<SG, S, ALG_DEFAULT>(sm, l);
        }
        cx<T> *gout = out + vol * V;
        for (int rank = 0; rank < C; ++rank) {
            for (int l = rank * LPC; l < (rank + 1) * LPC; ++l) {
                const int y = l / N2, z = l % N2;
                cx<T> v[N0];
                for (int j = 0; j < N0; ++j) v[j] = slab[j / PL][SG::off((j % PL) * N1 + y, z)];
                dft<N0, S, T>(v);
                for (int j = 0; j < N0; ++j) {
                    cx<T> r = v[j];
                    if (S > 0) r = cscale(r, scale);
                    gout[(long long)(j * N1 + y) * N2 + z] = r;
                }
            }
        }
    }
}

// The batch kernel's two-phase cube: x-slabs (z pass, y pass stored to scratch), then
// the x pass of every line straight out of scratch (batch_kernel.cu big_cube).
template <int L, typename T, int S, int PL>
static void emulate_big_cube(const void *vin, void *vout, long long nvol)
{
    constexpr int NS = L / PL;
    using XG = Geom<PL, L, L, T>;
    constexpr long long V = (long long)L * L * L;
    const T scale = S > 0 ? T(1) / T(V) : T(1);
    std::vector<cx<T>> sm((size_t)XG::PV);
    std::vector<cx<T>> scratch((size_t)V, cx<T>{T(-777.0), T(555.0)});
    for (long long vol = 0; vol < nvol; ++vol) {
        const cx<T> *gin = (const cx<T> *)vin + vol * V;
        cx<T> *gout = (cx<T> *)vout + vol * V;
        for (int s = 0; s < NS; ++s) {
            for (auto &e : sm) e = {T(12345.0), T(-6789.0)};
            for (int g = 0; g < PL * L * L; ++g)
                sm[XG::off(g / L, g % L)] = gin[(long long)s * PL * L * L + g];
            for (int r = 0; r < PL * L; ++r) pass_z<XG, S, ALG_DEFAULT>(sm.data(), r);
            for (int l = 0; l < PL * L; ++l) pass_y_store_l2<XG, S>(sm.data(), l, scratch.data(), s * PL);
        }
        for (int l = 0; l < L * L; ++l) pass_x_load_l2<L, L, L, S, T>(scratch.data(), l, gout, 0, scale);
    }
}

static long long g_twopass_violations = 0;

// The ring as the kernels see it: 128-byte aligned, filled with a marker.
template <typename T>
static cx<T> *aligned_ring(std::vector<cx<T>> &buf, long long elems)
{
    buf.assign((size_t)elems + 128 / sizeof(cx<T>), cx<T>{T(-777.0), T(555.0)});
    return reinterpret_cast<cx<T> *>(((uintptr_t)buf.data() + 127) & ~(uintptr_t)127);
}

// A row item's discards (twopass_kernels.cu twopass_discard_rows): the lines
// it drops hold garbage afterwards, so a later read of one shows up as NaN.
template <class TG>
static void poison_discarded_rows(void *slot, int j)
{
    constexpr int NQ = TG::YG::N0 * twopass_row_lines_per_plane<TG>();
    for (int q = 0; q < NQ; ++q) {
        uintptr_t line;
        if (twopass_row_line<TG>(slot, j, q, &line)) memset((void *)line, 0xff, 128);
    }
}

// The TWOPASS kernel's work items (twopass_kernels.cu k_twopass), taken in
// ticket order with the kernel's decode, element maps and ring of R slots.
// Ticket order satisfies every dependency, so one "CTA" can run them in turn;
// the small grid of 7 CTAs keeps R small, so the ring wraps many times.
template <int N0, int N1, int N2, typename T, int S, int G>
static void emulate_twopass(const void *vin, void *vout, long long nvol)
{
    using TG = TwoPassGeom<N0, N1, N2, T, G>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    const T scale = S > 0 ? T(1) / T(TG::V) : T(1);
    int lag = 0;
    const int R = twopass_ring_size(TG::NA, TG::NB, 7, &lag);
    std::vector<cx<T>> sm((size_t)TG::PV), ringbuf;
    cx<T> *ring = aligned_ring(ringbuf, (long long)R * TG::V);
    const cx<T> *in = (const cx<T> *)vin;
    cx<T> *out = (cx<T> *)vout;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    std::vector<long long> cnt_plane(R, 0), cnt_row(R, 0);
    for (long long t = 0; t < total; ++t) {
        const TwoPassItem it = twopass_decode(t, nvol, TG::NA, TG::NB, lag);
        const int slot = (int)(it.vol % R);
        const long long round = it.vol / R;
        cx<T> *sv = ring + slot * TG::V;
        for (auto &e : sm) e = {T(12345.0), T(-6789.0)};
        // the kernel's waits must already hold in ticket order
        if (it.plane ? cnt_row[slot] < TG::NB * round : cnt_plane[slot] < TG::NA * (round + 1))
            g_twopass_violations++;
        (it.plane ? cnt_plane : cnt_row)[slot]++;
        if (it.plane) {
            for (int g = 0; g < TG::PLANE_ELEMS; ++g) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                sm[so] = in[it.vol * TG::V + vo];
            }
            for (int r = 0; r < G * N1; ++r) pass_z<XG, S, ALG_DEFAULT>(sm.data(), r);
            for (int l = 0; l < G * N2; ++l) pass_y<XG, S, ALG_DEFAULT>(sm.data(), l);
            for (int g = 0; g < TG::PLANE_ELEMS; ++g) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                sv[vo] = sm[so];
            }
        } else {
            for (int g = 0; g < TG::ROW_ELEMS; ++g) {
                long long vo;
                int so;
                twopass_row_elem<TG>(it.j, g, &vo, &so);
                sm[so] = sv[vo];
            }
            poison_discarded_rows<TG>(sv, it.j);
            for (int l = 0; l < G * N2; ++l)
                pass_x_slab<YG, S, N1>(sm.data(), l, out + it.vol * TG::V, it.j * G, scale);
        }
    }
}

// The lean-control TWOPASS variants (k_twopass_regs): z pass in the plane
// layout; y pass stored straight into the slot; x pass loaded straight from
// the slot or from rows gathered into the row layout (XBULK).  Same tickets,
// ring and dependency checks as emulate_twopass.
template <int N0, int N1, int N2, typename T, int S, int G, bool XBULK, int PITCH = 0>
static void emulate_twopass_regs(const void *vin, void *vout, long long nvol)
{
    using TG = TwoPassGeom<N0, N1, N2, T, G, PITCH>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    const T scale = S > 0 ? T(1) / T(TG::V) : T(1);
    int lag = 0;
    const int R = twopass_ring_size(TG::NA, TG::NB, 7, &lag);
    std::vector<cx<T>> sm((size_t)TG::PV), ringbuf;
    cx<T> *ring = aligned_ring(ringbuf, (long long)R * TG::V);
    const cx<T> *in = (const cx<T> *)vin;
    cx<T> *out = (cx<T> *)vout;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    std::vector<long long> cnt_plane(R, 0), cnt_row(R, 0);
    for (long long t = 0; t < total; ++t) {
        const TwoPassItem it = twopass_decode(t, nvol, TG::NA, TG::NB, lag);
        const int slot = (int)(it.vol % R);
        const long long round = it.vol / R;
        cx<T> *sv = ring + slot * TG::V;
        if (it.plane ? cnt_row[slot] < TG::NB * round : cnt_plane[slot] < TG::NA * (round + 1))
            g_twopass_violations++;
        (it.plane ? cnt_plane : cnt_row)[slot]++;
        for (auto &e : sm) e = {T(12345.0), T(-6789.0)};
        if (it.plane) {
            const cx<T> *rows = in + it.vol * TG::V + (long long)it.j * G * N1 * N2;
            for (int r = 0; r < XG::ROWS; ++r)  // the bulk copy of row r
                for (int z = 0; z < N2; ++z) sm[XG::off(r, z)] = rows[(long long)r * N2 + z];
            for (int r = 0; r < XG::ROWS; ++r) pass_z<XG, S, ALG_DEFAULT>(sm.data(), r);
            for (int l = 0; l < G * N2; ++l) pass_y_store_l2<XG, S>(sm.data(), l, sv, it.j * G);
        } else if (XBULK) {
            for (int q = 0; q < N0 * G; ++q) {
                const int x = q / G, yl = q % G;
                for (int z = 0; z < N2; ++z)
                    sm[YG::off(q, z)] = sv[((long long)x * N1 + it.j * G + yl) * N2 + z];
            }
            poison_discarded_rows<TG>(sv, it.j);
            for (int l = 0; l < G * N2; ++l)
                pass_x_slab<YG, S, N1>(sm.data(), l, out + it.vol * TG::V, it.j * G, scale);
        } else {
            for (int l = 0; l < G * N2; ++l)
                pass_x_load_l2<N0, N1, N2, S, T>(sv, l, out + it.vol * TG::V, it.j * G, scale);
            poison_discarded_rows<TG>(sv, it.j);
        }
    }
}

// The lane-split TWOPASS kernel (k_twopass_lanes): rows at the odd pitch N|1,
// every line's P lanes run by lane_split_line_host with the kernel's own index
// maps -- z pass in place, y pass into the slot, x pass to the output.
// Tickets, ring and dependency checks as emulate_twopass.
template <int N, int S, int G, int P>
static void emulate_twopass_lanes(const void *vin, void *vout, long long nvol)
{
    using T = double;
    constexpr int PITCH = N | 1;
    using TG = TwoPassGeom<N, N, N, T, G, PITCH>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    constexpr int LINES = G * N;
    const T scale = S > 0 ? T(1) / T(TG::V) : T(1);
    int lag = 0;
    const int R = twopass_ring_size(TG::NA, TG::NB, 7, &lag);
    std::vector<cx<T>> sm((size_t)TG::PV), ringbuf;
    cx<T> *ring = aligned_ring(ringbuf, (long long)R * TG::V);
    const cx<T> *in = (const cx<T> *)vin;
    cx<T> *out = (cx<T> *)vout;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    std::vector<long long> cnt_plane(R, 0), cnt_row(R, 0);
    for (long long tk = 0; tk < total; ++tk) {
        const TwoPassItem it = twopass_decode(tk, nvol, TG::NA, TG::NB, lag);
        const int slot = (int)(it.vol % R);
        const long long round = it.vol / R;
        cx<T> *sv = ring + slot * TG::V;
        if (it.plane ? cnt_row[slot] < TG::NB * round : cnt_plane[slot] < TG::NA * (round + 1))
            g_twopass_violations++;
        (it.plane ? cnt_plane : cnt_row)[slot]++;
        for (auto &e : sm) e = {T(12345.0), T(-6789.0)};
        if (it.plane) {
            const cx<T> *rows = in + it.vol * TG::V + (long long)it.j * G * N * N;
            for (int r = 0; r < XG::ROWS; ++r)
                for (int z = 0; z < N; ++z) sm[XG::off(r, z)] = rows[(long long)r * N + z];
            for (int r = 0; r < LINES; ++r) {
                cx<T> *row = sm.data() + XG::off(r, 0);
                lane_split_line_host<N, P, S, T>([&](int z) { return row[z]; },
                                                 [&](int z, cx<T> v) { row[z] = v; });
            }
            for (int l = 0; l < LINES; ++l) {
                const int g = l / N, z = l % N;
                const cx<T> *col = sm.data() + XG::off(g * N, z);
                cx<T> *o = sv + (long long)(it.j * G + g) * N * N + z;
                lane_split_line_host<N, P, S, T>([&](int y) { return col[y * PITCH]; },
                                                 [&](int y, cx<T> v) { o[y * N] = v; });
            }
        } else {
            for (int q = 0; q < N * G; ++q) {
                const int x = q / G, yl = q % G;
                for (int z = 0; z < N; ++z) sm[YG::off(q, z)] = sv[((long long)x * N + it.j * G + yl) * N + z];
            }
            poison_discarded_rows<TG>(sv, it.j);
            cx<T> *gvol = out + it.vol * TG::V;
            for (int l = 0; l < LINES; ++l) {
                const int yl = l / N, z = l % N;
                const cx<T> *col = sm.data() + YG::off(yl, z);
                cx<T> *o = gvol + (long long)(it.j * G + yl) * N + z;
                lane_split_line_host<N, P, S, T>([&](int x) { return col[x * G * PITCH]; },
                                                 [&](int x, cx<T> v) {
                                                     if (S > 0) v = cscale(v, scale);
                                                     o[(long long)x * N * N] = v;
                                                 });
            }
        }
    }
}

// The staged TWOPASS kernel (k_twopass_staged; staged.cuh line policies):
// rows at the kernel's pitch, z pass in place (rows end in Line::slot order),
// y pass stored into the slot at the natural z, x pass streamed out; every
// stage-1 task of a pass before any stage-2 task, as the kernel's barrier
// orders them.  Tickets, ring and dependency checks as emulate_twopass.
template <class Line, int S, typename T = double>
static void emulate_twopass_staged(const void *vin, void *vout, long long nvol)
{
    constexpr int N = Line::N, P = sizeof(T) == 8 ? (N | 1) : ((N + 2) & ~1);
    constexpr long long PLANE = (long long)N * N;
    using TG = TwoPassGeom<N, N, N, T, 1>;
    const T scale = S > 0 ? T(1) / T(TG::V) : T(1);
    int lag = 0;
    const int R = twopass_ring_size(TG::NA, TG::NB, 7, &lag);
    std::vector<cx<T>> smv((size_t)N * P), ringbuf;
    cx<T> *ring = aligned_ring(ringbuf, (long long)R * TG::V);
    cx<T> *sm = smv.data();
    const cx<T> *in = (const cx<T> *)vin;
    cx<T> *out = (cx<T> *)vout;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    std::vector<long long> cnt_plane(R, 0), cnt_row(R, 0);
    auto rowaddr = [](int l, int e) { return l * P + e; };
    auto coladdr = [](int l, int e) { return e * P + l; };
    for (long long t = 0; t < total; ++t) {
        const TwoPassItem it = twopass_decode(t, nvol, TG::NA, TG::NB, lag);
        const int slot = (int)(it.vol % R);
        const long long round = it.vol / R;
        cx<T> *sv = ring + slot * TG::V;
        if (it.plane ? cnt_row[slot] < TG::NB * round : cnt_plane[slot] < TG::NA * (round + 1))
            g_twopass_violations++;
        (it.plane ? cnt_plane : cnt_row)[slot]++;
        for (auto &e : smv) e = {T(12345.0), T(-6789.0)};
        if (it.plane) {
            const cx<T> *rows = in + it.vol * TG::V + (long long)it.j * PLANE;
            for (int r = 0; r < N; ++r)
                for (int z = 0; z < N; ++z) sm[r * P + z] = rows[(long long)r * N + z];
            for (int q = 0; q < N * Line::T1; ++q) Line::template stage1<S, T>(sm, N, q, rowaddr);
            for (int q = 0; q < N * Line::T2; ++q)
                Line::template stage2<S, T>(sm, N, q, rowaddr, [&](int l, int k, cx<T> v) { sm[rowaddr(l, Line::slot(k))] = v; });
            for (int q = 0; q < N * Line::T1; ++q) Line::template stage1<S, T>(sm, N, q, coladdr);
            cx<T> *dst = sv + (long long)it.j * PLANE;
            for (int q = 0; q < N * Line::T2; ++q)
                Line::template stage2<S, T>(sm, N, q, coladdr, [&](int p, int k, cx<T> v) { dst[k * N + Line::at(p)] = v; });
        } else {
            for (int x = 0; x < N; ++x)
                for (int z = 0; z < N; ++z) sm[x * P + z] = sv[((long long)x * N + it.j) * N + z];
            poison_discarded_rows<TG>(sv, it.j);
            for (int q = 0; q < N * Line::T1; ++q) Line::template stage1<S, T>(sm, N, q, coladdr);
            cx<T> *gvol = out + it.vol * TG::V + (long long)it.j * N;
            for (int q = 0; q < N * Line::T2; ++q)
                Line::template stage2<S, T>(sm, N, q, coladdr, [&](int z, int k, cx<T> v) {
                    if (S > 0) v = cscale(v, scale);
                    gvol[k * PLANE + z] = v;
                });
        }
    }
}


typedef void (*emu_fn)(const void *, void *, long long);

#define EMU_TPR_(N0, N1, N2, G, A, XB)                                                       \
    {N0, N1, N2, 0, -1, A + G, 1, &emulate_twopass_regs<N0, N1, N2, double, -1, G, XB>},       \
    {N0, N1, N2, 0, +1, A + G, 1, &emulate_twopass_regs<N0, N1, N2, double, +1, G, XB>}
#define EMU_TPR(N0, N1, N2, G) EMU_TPR_(N0, N1, N2, G, 500, false)
#define EMU_TPRQ(N0, N1, N2, G) EMU_TPR_(N0, N1, N2, G, 540, true)
#define EMU_TPRQF(G)                                                                          \
    {36, 36, 36, 1, -1, 540 + G, 1, &emulate_twopass_regs<36, 36, 36, float, -1, G, true, 38>},  \
    {36, 36, 36, 1, +1, 540 + G, 1, &emulate_twopass_regs<36, 36, 36, float, +1, G, true, 38>}
#define EMU_TPL(N, G, P)                                                                      \
    {N, N, N, 0, -1, 1024 + P, G, &emulate_twopass_lanes<N, -1, G, P>},                        \
    {N, N, N, 0, +1, 1024 + P, G, &emulate_twopass_lanes<N, +1, G, P>}
#define EMU_TPST(LINE, N, T)                                                                  \
    {N, N, N, sizeof(T) == 8 ? 0 : 1, -1, 701, 1, &emulate_twopass_staged<LINE, -1, T>},         \
    {N, N, N, sizeof(T) == 8 ? 0 : 1, +1, 701, 1, &emulate_twopass_staged<LINE, +1, T>}
#define EMU_TP(N0, N1, N2, T, G)                                                              \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, -1, 300 + G, 1,                                    \
     &emulate_twopass<N0, N1, N2, T, -1, G>},                                                \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, +1, 300 + G, 1, &emulate_twopass<N0, N1, N2, T, +1, G>}

#define EMU_BIG(L, T, PL)                                                               \
    {L, L, L, sizeof(T) == 8 ? 0 : 1, -1, 200 + PL, 1, &emulate_big_cube<L, T, -1, PL>}, \
    {L, L, L, sizeof(T) == 8 ? 0 : 1, +1, 200 + PL, 1, &emulate_big_cube<L, T, +1, PL>}

#define EMU_BST(N0, N1, N2, T, ALG, VPC)                                                      \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, -1, 400 + ALG, VPC,                                 \
     &emulate_bst<N0, N1, N2, T, -1, ALG, VPC>},                                             \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, +1, 400 + ALG, VPC, &emulate_bst<N0, N1, N2, T, +1, ALG, VPC>}

#define EMU_CL(N0, N1, N2, T, C)                                                             \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, -1, 100 + C, 1,                                   \
     &emulate_cluster<N0, N1, N2, T, -1, C>},                                               \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, +1, 100 + C, 1, &emulate_cluster<N0, N1, N2, T, +1, C>}

struct EmuEntry {
    int n0, n1, n2, prec, sign, alg, vpc;
    emu_fn fn;
};

#define EMU(N0, N1, N2, T, ALG, VPC)                                                           \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, -1, ALG, VPC, &emulate<N0, N1, N2, T, -1, ALG, VPC>}, \
    {N0, N1, N2, sizeof(T) == 8 ? 0 : 1, +1, ALG, VPC, &emulate<N0, N1, N2, T, +1, ALG, VPC>}

static const EmuEntry kEmu[] = {
    EMU(6, 6, 6, double, 0, 16),   EMU(8, 8, 8, double, 0, 8),     EMU(12, 12, 12, double, 0, 2),
    EMU(16, 16, 16, double, 0, 1), EMU(17, 17, 17, double, 0, 1),  EMU(17, 17, 17, double, 1, 1),
    EMU(24, 24, 24, double, 0, 1), EMU(8, 8, 16, double, 0, 8),    EMU(16, 16, 32, double, 0, 1),
    EMU(36, 36, 36, double, 0, 1), EMU(6, 6, 6, float, 0, 32),     EMU(8, 8, 8, float, 0, 16),
    EMU(12, 12, 12, float, 0, 4),  EMU(16, 16, 16, float, 0, 2),   EMU(17, 17, 17, float, 0, 2),
    EMU(17, 17, 17, float, 1, 2),  EMU(24, 24, 24, float, 0, 1),   EMU(8, 8, 16, float, 0, 16),
    EMU(16, 16, 32, float, 0, 1),  EMU(36, 36, 36, float, 0, 1),   EMU(2, 3, 5, double, 0, 3),
    EMU(7, 11, 13, double, 0, 2),  EMU(9, 9, 9, double, 0, 2),     EMU(5, 8, 12, double, 0, 1),
    EMU(32, 8, 4, double, 0, 1),   EMU(13, 5, 8, double, 0, 1),    EMU(4, 4, 4, double, 0, 2),
    EMU(1, 8, 8, double, 0, 1),    EMU(8, 1, 8, double, 0, 1),     EMU(8, 8, 1, double, 0, 1),
    EMU(1, 1, 1, double, 0, 1),    EMU(3, 3, 3, double, 0, 1),     EMU(17, 2, 2, double, 0, 1),
    EMU_CL(36, 36, 36, double, 4), EMU_CL(36, 36, 36, double, 6),  EMU_CL(36, 36, 36, double, 9),
    EMU_CL(36, 36, 36, float, 2),  EMU_CL(36, 36, 36, float, 4),   EMU_CL(36, 36, 36, float, 6),
    EMU_BIG(36, double, 4),        EMU_BIG(36, float, 6),   EMU_BIG(36, float, 4),
    EMU_TP(36, 36, 36, double, 4), EMU_TP(36, 36, 36, double, 2),  EMU_TP(36, 36, 36, double, 6),
    EMU_TP(36, 36, 36, float, 4),  EMU_TP(36, 36, 36, float, 6),   EMU_TP(16, 16, 32, double, 4),
    EMU_TP(16, 16, 32, double, 8), EMU_TP(6, 9, 5, double, 3),     EMU_TP(36, 36, 36, double, 3),
    EMU(13, 13, 13, double, 0, 2), EMU(23, 23, 23, double, 0, 1),  EMU(13, 13, 13, float, 0, 4),
    EMU(23, 23, 23, float, 0, 1),  EMU_TP(45, 45, 45, double, 3), EMU_TP(45, 45, 45, float, 5),
    EMU_TP(64, 64, 64, double, 1), EMU_TP(64, 64, 64, float, 2),
    EMU_TPR(36, 36, 36, 3), EMU_TPR(36, 36, 36, 2), EMU_TPR(36, 36, 36, 4), EMU_TPRQ(36, 36, 36, 3),
    EMU_TPRQ(36, 36, 36, 2), EMU_TPRQ(6, 9, 5, 3), EMU_TPRQF(3), EMU_TPRQF(2), EMU_TPRQF(4), EMU_TPST(LineCT64, 64, double), EMU_TPST(LineCT64, 64, float), EMU_TPST(LinePFA45, 45, double),
    EMU_TPR(6, 9, 5, 3),
    EMU_TPL(36, 2, 2), EMU_TPL(36, 2, 4), EMU_TPL(36, 1, 4), EMU_TPL(36, 3, 4),
    // the group sizes the VOLUME kernels of these extents use
    EMU(1, 1, 1, double, 0, 64),  EMU(3, 3, 3, double, 0, 32),   EMU(4, 4, 4, double, 0, 16),
    EMU(9, 9, 9, double, 0, 4),   EMU(10, 10, 10, double, 0, 2), EMU(15, 15, 15, double, 0, 1),
    EMU(2, 3, 5, double, 0, 32),  EMU(5, 8, 12, double, 0, 4),   EMU(13, 5, 8, double, 0, 4),
    EMU(17, 2, 2, double, 0, 16), EMU(32, 8, 4, double, 0, 2),   EMU(1, 8, 8, double, 0, 32),
    EMU(8, 1, 8, double, 0, 32),  EMU(8, 8, 1, double, 0, 32),
    EMU(1, 1, 1, float, 0, 128),  EMU(3, 3, 3, float, 0, 64),    EMU(4, 4, 4, float, 0, 32),
    EMU(9, 9, 9, float, 0, 8),    EMU(10, 10, 10, float, 0, 4),  EMU(15, 15, 15, float, 0, 2),
    EMU(2, 3, 5, float, 0, 64),   EMU(7, 11, 13, float, 0, 4),   EMU(5, 8, 12, float, 0, 8),
    EMU(13, 5, 8, float, 0, 8),   EMU(17, 2, 2, float, 0, 32),   EMU(32, 8, 4, float, 0, 4),
    EMU(1, 8, 8, float, 0, 64),   EMU(8, 1, 8, float, 0, 64),    EMU(8, 8, 1, float, 0, 64),
    // the rest of the reference's test geometries, at their VOLUME group sizes
    EMU(2, 2, 2, double, 0, 64),   EMU(5, 5, 5, double, 0, 24),  EMU(7, 7, 7, double, 0, 8),
    EMU(11, 11, 11, double, 0, 2), EMU(49, 2, 2, double, 0, 10), EMU(25, 4, 3, double, 0, 10),
    EMU(27, 2, 2, double, 0, 18),  EMU(19, 3, 2, double, 0, 17), EMU(23, 2, 2, double, 0, 22),
    EMU(47, 3, 2, double, 0, 7),   EMU(83, 2, 1, double, 0, 18), EMU(97, 2, 1, double, 0, 15),
    EMU(1, 1, 16, double, 0, 64),  EMU(1, 7, 1, double, 0, 64),  EMU(3, 5, 7, double, 0, 29),
    EMU(4, 6, 10, double, 0, 11),  EMU(16, 3, 5, double, 0, 12), EMU(24, 18, 12, double, 0, 1),
    EMU(2, 2, 64, double, 0, 12),  EMU(64, 2, 2, double, 0, 8),  EMU(9, 25, 7, double, 0, 1),
    EMU(20, 12, 6, double, 0, 1),  EMU(11, 4, 9, double, 0, 7),
    EMU(2, 2, 2, float, 0, 64),    EMU(5, 5, 5, float, 0, 49),   EMU(7, 7, 7, float, 0, 17),
    EMU(11, 11, 11, float, 0, 4),  EMU(49, 2, 2, float, 0, 20),  EMU(25, 4, 3, float, 0, 20),
    EMU(27, 2, 2, float, 0, 37),   EMU(19, 3, 2, float, 0, 35),  EMU(23, 2, 2, float, 0, 44),
    EMU(47, 3, 2, float, 0, 14),   EMU(83, 2, 1, float, 0, 37),  EMU(97, 2, 1, float, 0, 31),
    EMU(1, 1, 16, float, 0, 64),   EMU(1, 7, 1, float, 0, 64),   EMU(3, 5, 7, float, 0, 58),
    EMU(4, 6, 10, float, 0, 23),   EMU(16, 3, 5, float, 0, 25),  EMU(24, 18, 12, float, 0, 1),
    EMU(30, 30, 30, float, 0, 1),  EMU(2, 2, 64, float, 0, 24),  EMU(64, 2, 2, float, 0, 16),
    EMU(9, 25, 7, float, 0, 3),    EMU(20, 12, 6, float, 0, 3),  EMU(11, 4, 9, float, 0, 15),
    EMU_TP(30, 30, 30, double, 3), EMU_TP(30, 30, 30, double, 5),
    EMU_BST(17, 17, 17, double, 0, 1), EMU_BST(17, 17, 17, float, 0, 2),
    EMU(17, 17, 17, double, 2, 1),     EMU(17, 17, 17, float, 2, 2),
    EMU_BST(17, 17, 17, double, 2, 1), EMU_BST(17, 17, 17, float, 2, 2),
    EMU_BST(13, 13, 13, double, 0, 1), EMU_BST(13, 13, 13, double, 0, 2),
    EMU_BST(13, 13, 13, float, 0, 2),  EMU_BST(8, 8, 8, double, 0, 1),
    EMU_BST(16, 16, 16, double, 0, 1), EMU_BST(16, 16, 16, float, 0, 1),
};

// The chain kernel's per-CTA loop (chain_kernels.cu k_chain) for one volume per CTA.
template <int N0, int N1, int N2, typename T, int EPI>
static void emulate_chain(const void *vin, void *vout, const void *vc, long long nvol, long long steps)
{
    using G = Geom<N0, N1, N2, T>;
    const cx<T> *in = (const cx<T> *)vin;
    const cx<T> *cmap = (const cx<T> *)vc;
    cx<T> *out = (cx<T> *)vout;
    const T us = T(1) / std::sqrt(T(G::V));
    std::vector<cx<T>> sm((size_t)G::PV);
    for (long long v = 0; v < nvol; ++v) {
        const long long e0 = v * G::V;
        for (int g = 0; g < G::V; ++g) stage_in<G>(sm.data(), in + e0, g);
        for (long long s = 0; s < steps; ++s) {
            for (int r = 0; r < G::ROWS; ++r) pass_z<G, -1, ALG_DEFAULT>(sm.data(), r);
            for (int l = 0; l < G::N0 * G::N2; ++l) pass_y<G, -1, ALG_DEFAULT>(sm.data(), l);
            for (int l = 0; l < G::N1 * G::N2; ++l)
                pass_x_chain<G, ALG_DEFAULT, EPI>(sm.data(), l, cmap, e0, us);
        }
        for (int g = 0; g < G::V; ++g) out[e0 + g] = sm[G::off(g / G::N2, g % G::N2)];
    }
}

extern "C" int hostcheck_chain(int n, int prec, int epi, const void *in, void *out, const void *c,
                               long long nvol, long long steps)
{
    ensure_host_tables();
#define HC_CHAIN(L, T)                                                                          \
    if (n == L && prec == (sizeof(T) == 8 ? 0 : 1)) {                                          \
        if (epi == EPI_UNITARY) emulate_chain<L, L, L, T, EPI_UNITARY>(in, out, c, nvol, steps); \
        else emulate_chain<L, L, L, T, EPI_MAP>(in, out, c, nvol, steps);                       \
        return 0;                                                                               \
    }
    HC_CHAIN(6, double) HC_CHAIN(8, double) HC_CHAIN(17, double) HC_CHAIN(8, float)
#undef HC_CHAIN
    return -2;
}

// The multi-GPU slab path (mgpu.cu): n "GPUs" as separate buffers, the same layout
// functions, the z and y passes of each x-plane with each point stored into the
// middle buffer of its y owner, then the x lines of each y-slab, then the
// gather of download().  Poisoned middle buffers show any point not delivered.
template <int L, int SGN>
static void emulate_mgpu(int n, const cx<double> *in, cx<double> *out, long long B)
{
    using PG = Geom<1, L, L, double>;
    using RG = Geom<L, 1, L, double>;
    const MgpuShape m{L, n, L / n};
    const size_t slab = (size_t)B * m.S * L * L;
    std::vector<std::vector<cx<double>>> mid(n, std::vector<cx<double>>(slab, cx<double>{-1e300, 1e300}));
    std::vector<std::vector<cx<double>>> res(n, std::vector<cx<double>>(slab));
    std::vector<cx<double>> sm((size_t)PG::PV);
    const double scale = SGN > 0 ? 1.0 / ((double)L * L * L) : 1.0;
    for (int g = 0; g < n; ++g) {
        for (long long p = 0; p < B * m.S; ++p) {
            const long long b = p / m.S, x = g * m.S + p % m.S;
            const cx<double> *src = in + (b * L + x) * (long long)L * L;  // upload(): x-slab g
            for (int e = 0; e < L * L; ++e) sm[PG::off(e / L, e % L)] = src[e];
            for (int r = 0; r < L; ++r) pass_z<PG, SGN, ALG_DEFAULT>(sm.data(), r);
            for (int l = 0; l < L; ++l) pass_y<PG, SGN, ALG_DEFAULT>(sm.data(), l);
            for (int e = 0; e < L * L; ++e) {
                int h;
                const long long off = mgpu_mid_offset(m, g, p, e / L, e % L, &h);
                mid[h][off] = sm[PG::off(e / L, e % L)];
            }
        }
    }
    std::vector<cx<double>> row((size_t)RG::PV);
    for (int h = 0; h < n; ++h) {
        for (long long r = 0; r < B * m.S; ++r) {
            const long long b = r / m.S;
            const int yl = (int)(r % m.S);
            for (int e = 0; e < L * L; ++e)
                row[RG::off(e / L, e % L)] = mid[h][mgpu_yslab_offset(m, b, e / L, yl, e % L)];
            for (int z = 0; z < L; ++z) {
                cx<double> v[L];
                for (int j = 0; j < L; ++j) v[j] = row[RG::off(j, z)];
                dft<L, SGN, double>(v);
                for (int j = 0; j < L; ++j) {
                    cx<double> o = v[j];
                    if (SGN > 0) o = cscale(o, scale);
                    res[h][mgpu_yslab_offset(m, b, j, yl, z)] = o;
                }
            }
        }
    }
    for (long long b = 0; b < B; ++b)  // download(): ky = h*S + yl
        for (int kx = 0; kx < L; ++kx)
            for (int ky = 0; ky < L; ++ky)
                for (int kz = 0; kz < L; ++kz)
                    out[((b * L + kx) * L + ky) * (long long)L + kz] =
                        res[ky / m.S][mgpu_yslab_offset(m, b, kx, ky % m.S, kz)];
}

// Large L (mgpu.cu k_mgl_*): z lines of the x-slab into tmp, y lines of tmp to
// the middle buffer of each point's y owner, x lines of each y-slab; every line
// through split_line_host, the host form of the kernels' lane exchange.
template <int L, int SGN>
static void emulate_mgpu_large(int n, const cx<double> *in, cx<double> *out, long long B)
{
    const MgpuShape m{L, n, L / n};
    const size_t slab = (size_t)B * m.S * L * L;
    std::vector<cx<double>> tmp(slab);
    std::vector<std::vector<cx<double>>> mid(n, std::vector<cx<double>>(slab, cx<double>{-1e300, 1e300}));
    std::vector<std::vector<cx<double>>> res(n, std::vector<cx<double>>(slab));
    const double scale = SGN > 0 ? 1.0 / ((double)L * L * L) : 1.0;
    for (int g = 0; g < n; ++g) {
        for (long long p = 0; p < B * m.S; ++p) {
            const long long b = p / m.S, x = g * m.S + p % m.S;
            const cx<double> *src = in + (b * L + x) * (long long)L * L;
            cx<double> *t = tmp.data() + p * L * L;
            for (int e = 0; e < L * L; ++e) t[e] = src[e];
            for (int r = 0; r < L; ++r)
                split_line_host<L, SGN, double>([&](int k) { return t[r * L + k]; },
                                                [&](int k, cx<double> v) { t[r * L + k] = v; });
            for (int z = 0; z < L; ++z)
                split_line_host<L, SGN, double>([&](int y) { return t[y * L + z]; },
                                                [&](int y, cx<double> v) { t[y * L + z] = v; });
            for (int e = 0; e < L * L; ++e) {
                int h;
                const long long off = mgpu_mid_offset(m, g, p, e / L, e % L, &h);
                mid[h][off] = t[e];
            }
        }
    }
    for (int h = 0; h < n; ++h)
        for (long long r = 0; r < B * m.S; ++r) {
            const long long b = r / m.S;
            const int yl = (int)(r % m.S);
            for (int z = 0; z < L; ++z)
                split_line_host<L, SGN, double>(
                    [&](int x) { return mid[h][mgpu_yslab_offset(m, b, x, yl, z)]; },
                    [&](int x, cx<double> v) {
                        res[h][mgpu_yslab_offset(m, b, x, yl, z)] = SGN > 0 ? cscale(v, scale) : v;
                    });
        }
    for (long long b = 0; b < B; ++b)
        for (int kx = 0; kx < L; ++kx)
            for (int ky = 0; ky < L; ++ky)
                for (int kz = 0; kz < L; ++kz)
                    out[((b * L + kx) * L + ky) * (long long)L + kz] =
                        res[ky / m.S][mgpu_yslab_offset(m, b, kx, ky % m.S, kz)];
}

extern "C" int hostcheck_mgpu(int L, int n, int sign, const void *in, void *out, long long B)
{
    ensure_host_tables();
    if (n < 1 || L % n) return -1;
    const cx<double> *x = (const cx<double> *)in;
    cx<double> *y = (cx<double> *)out;
#define HC_MG(LL)                                                          \
    if (L == LL) {                                                         \
        if (sign < 0) emulate_mgpu<LL, -1>(n, x, y, B);                    \
        else emulate_mgpu<LL, +1>(n, x, y, B);                             \
        return 0;                                                          \
    }
    HC_MG(36) HC_MG(45) HC_MG(64)
#undef HC_MG
#define HC_MGL(LL)                                                         \
    if (L == LL) {                                                         \
        if (sign < 0) emulate_mgpu_large<LL, -1>(n, x, y, B);              \
        else emulate_mgpu_large<LL, +1>(n, x, y, B);                       \
        return 0;                                                          \
    }
    HC_MGL(96) HC_MGL(128) HC_MGL(192) HC_MGL(256)
#undef HC_MGL
    return -2;
}

// The t pass of a 4D plan (plan4d.cu k_tpass) on the host: each spatial point
// of each lattice, its nt points strided by V, in place.
template <int TL, int SGN>
static void emulate_tpass(cx<double> *data, long long vol_elems, long long batch)
{
    const double scale = SGN > 0 ? 1.0 / TL : 1.0;
    for (long long b = 0; b < batch; ++b)
        for (long long p = 0; p < vol_elems; ++p) {
            cx<double> *col = data + b * TL * vol_elems + p;
            cx<double> v[TL];
            for (int t = 0; t < TL; ++t) v[t] = col[t * vol_elems];
            dft<TL, SGN, double>(v);
            for (int t = 0; t < TL; ++t) col[t * vol_elems] = SGN > 0 ? cscale(v[t], scale) : v[t];
        }
}

extern "C" int hostcheck_tpass(int tl, int sign, void *data, long long vol_elems, long long batch)
{
    ensure_host_tables();
    cx<double> *d = (cx<double> *)data;
#define HC_TP(TL)                                                                   \
    if (tl == TL) {                                                                 \
        if (sign < 0) emulate_tpass<TL, -1>(d, vol_elems, batch);                   \
        else emulate_tpass<TL, +1>(d, vol_elems, batch);                            \
        return 0;                                                                   \
    }
    HC_TP(2) HC_TP(4) HC_TP(6) HC_TP(8) HC_TP(12) HC_TP(16) HC_TP(17) HC_TP(24) HC_TP(32)
    HC_TP(36) HC_TP(48) HC_TP(64)
#undef HC_TP
    return -2;
}

// Items whose dependency wait would not hold when taken in ticket order (the
// TWOPASS deadlock-freedom argument); reset by reading.
extern "C" long long hostcheck_twopass_violations()
{
    const long long v = g_twopass_violations;
    g_twopass_violations = 0;
    return v;
}

extern "C" int hostcheck_fft3d(int n0, int n1, int n2, int prec, int sign, int alg, int vpc,
                               const void *in, void *out, long long nvol)
{
    ensure_host_tables();
    for (const auto &e : kEmu) {
        if (e.n0 == n0 && e.n1 == n1 && e.n2 == n2 && e.prec == prec && e.sign == sign &&
            e.alg == alg && (vpc <= 0 || e.vpc == vpc)) {
            e.fn(in, out, nvol);
            return 0;
        }
    }
    return -2;
}

// twopass_kernels.cu -- kernel family TWOPASS: volumes larger than one SM's
// shared memory (36^3 complex double is 746 KB, 64^3 is 4 MB), in plane and
// row items through an L2-resident scratch ring (twopass.cuh).
//
// Persistent CTAs take tickets.  A plane item copies its G contiguous x-planes
// into shared memory (cp.async, or one bulk copy per row), runs the z and y
// passes, and writes the planes to the volume's scratch slot with L2-only
// stores; a row item reads its G y-rows of all planes back with L2-only loads
// (never through L1, which is not coherent with other SMs' stores), runs the
// x pass and streams the result to the output.  Completion is published per
// slot by one thread's gpu-scope release add after a CTA-wide barrier -- the
// release is cumulative (PTX memory model: causality order runs through the
// barrier), so it publishes every thread's stores and no thread needs a fence
// of its own -- and observed with an acquire load, by one thread, before a
// barrier.  Several CTAs per SM (small items) overlap one another's loads,
// arithmetic and stores, so unlike a thread-block cluster that moves one
// volume in lock-step, HBM stays busy.
//
// Every wait is bounded in time (ptx.cuh wait_counter_geq); a timeout records
// DEV_ERR_DEP_TIMEOUT, raises the workspace abort flag so that the other CTAs
// stop too, and the last CTA to leave clears the control block for the next
// launch, on the error path as well.
#include <algorithm>

#include "internal.h"
#include "ptx.cuh"
#include "splitline.cuh"
#include "staged.cuh"
#include "twopass.cuh"

namespace fft3d {

// Every thread: drop from L2, without a write-back, the scratch lines whose
// rows row item j has read for the last time (twopass_row_line).  A barrier
// must follow before the slot is released to the next volume's plane items.
template <class TG>
__device__ __forceinline__ void twopass_discard_rows(const void *slot, int j, int tid, int nt)
{
    constexpr int NQ = TG::YG::N0 * twopass_row_lines_per_plane<TG>();
    for (int q = tid; q < NQ; q += nt) {
        uintptr_t line;
        if (twopass_row_line<TG>(slot, j, q, &line)) discard_l2_line(line);
    }
}

template <typename T>
__device__ __forceinline__ cx<T> ld_l2(const cx<T> *p)
{
    if constexpr (sizeof(T) == 8) {
        const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
        return {v.x, v.y};
    } else {
        const float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
        return {v.x, v.y};
    }
}

template <typename T>
__device__ __forceinline__ void st_l2(cx<T> *p, cx<T> v)
{
    if constexpr (sizeof(T) == 8) __stcg(reinterpret_cast<double2 *>(p), make_double2(v.re, v.im));
    else __stcg(reinterpret_cast<float2 *>(p), make_float2(v.re, v.im));
}

template <int N0, int N1, int N2, typename T, int S, int G, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_twopass(const cx<T> *__restrict__ in, cx<T> *__restrict__ out, long long nvol, T scale,
              int *err, unsigned char *work, int R, int D)
{
    pdl_begin();
    using TG = TwoPassGeom<N0, N1, N2, T, G>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    constexpr int U = 8;  // L2 loads in flight per thread in the row gather
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    __shared__ long long s_t;
    __shared__ int s_stop;
    TwoPassCtl *ctl = reinterpret_cast<TwoPassCtl *>(work);
    cx<T> *ring = reinterpret_cast<cx<T> *>(work + TWOPASS_CTL_BYTES);
    const int tid = threadIdx.x;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;

    for (;;) {
        if (tid == 0) {
            const long long t = (long long)atomicAdd(&ctl->ticket, 1ull);
            s_t = t;
            s_stop = (t >= total || ld_acquire_gpu(&ctl->abort) != 0) ? 1 : 0;
        }
        __syncthreads();
        if (s_stop) break;
        const TwoPassItem it = twopass_decode(s_t, nvol, TG::NA, TG::NB, D);
        const int slot = (int)(it.vol % R);
        const unsigned round = (unsigned)(it.vol / R);
        cx<T> *sv = ring + (long long)slot * TG::V;

        if (it.plane) {
            // 1. G contiguous planes of the input
            const cx<T> *src = in + it.vol * TG::V;
            for (int g = tid; g < TG::PLANE_ELEMS; g += NT) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                if constexpr (sizeof(T) == 8) cp_async_16(sm + so, src + vo);
                else cp_async_8(sm + so, src + vo);
            }
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
            // 2. z and y passes
            for (int r = tid; r < G * N1; r += NT) pass_z<XG, S, ALG_DEFAULT>(sm, r);
            __syncthreads();
            for (int l = tid; l < G * N2; l += NT) pass_y<XG, S, ALG_DEFAULT>(sm, l);
            // 3. the slot's previous volume must have been read out
            if (tid == 0)
                s_stop = wait_counter_geq(&ctl->cnt[TWOPASS_RMAX + slot], (unsigned)TG::NB * round,
                                          &ctl->abort)
                             ? 0
                             : 1;
            __syncthreads();
            if (s_stop) break;
            // 4. to scratch, same offsets as in the volume, L2 only
            for (int g = tid; g < TG::PLANE_ELEMS; g += NT) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                st_l2(sv + vo, sm[so]);
            }
            __syncthreads();  // then one cumulative release publishes every thread's stores
            if (tid == 0) red_release_gpu_add(&ctl->cnt[slot], 1u);
        } else {
            // 1. all plane items of this volume must be in scratch
            if (tid == 0)
                s_stop = wait_counter_geq(&ctl->cnt[slot], (unsigned)TG::NA * (round + 1u), &ctl->abort)
                             ? 0
                             : 1;
            __syncthreads();
            if (s_stop) break;
            // 2. gather the G rows of every plane
            for (int base = 0; base < TG::ROW_ELEMS; base += NT * U) {
                cx<T> v[U];
                int so[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int g = base + u * NT + tid;
                    so[u] = -1;
                    if (g < TG::ROW_ELEMS) {
                        long long vo;
                        twopass_row_elem<TG>(it.j, g, &vo, &so[u]);
                        v[u] = ld_l2(sv + vo);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (so[u] >= 0) sm[so[u]] = v[u];
            }
            __syncthreads();
            // read for the last time: drop the rows from L2 unwritten; then the
            // slot may be overwritten once every row item has read it
            twopass_discard_rows<TG>(sv, it.j, tid, NT);
            __syncthreads();
            if (tid == 0) red_release_gpu_add(&ctl->cnt[TWOPASS_RMAX + slot], 1u);
            // 3. x pass, straight to the output
            cx<T> *gvol = out + it.vol * TG::V;
            for (int l = tid; l < G * N2; l += NT) pass_x_slab<YG, S, N1>(sm, l, gvol, it.j * G, scale);
        }
        __syncthreads();  // the next item reuses shared memory
    }

    // A wait that timed out: record it and stop the other CTAs.
    if (tid == 0 && s_stop && s_t < total) {
        report_error(err, DEV_ERR_DEP_TIMEOUT);
        atomicExch(&ctl->abort, 1u);
    }
    // The last CTA to leave clears the control block for the next launch.
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();  // every other CTA's updates of the block precede the reset
            ctl->ticket = 0ull;
            for (int i = 0; i < 2 * TWOPASS_RMAX; ++i) ctl->cnt[i] = 0u;
            ctl->abort = 0u;
            __threadfence();
            ctl->done = 0u;
        }
    }
}

// Pipelined TWOPASS (complex double): two shared-memory stages per CTA; while
// one item is transformed, the next item's copies are in flight.  The next
// ticket is taken at the top of each iteration; its load is issued at once when
// it can start -- a plane item always (its input is read-only), a row item only
// when a non-blocking check finds its volume's plane items done -- and
// otherwise after the current item, with a blocking wait.  A CTA therefore
// blocks only on the dependencies of its single unfinished item, as in
// k_twopass, and the ticket-order argument against deadlock still holds.
// Row items read scratch with cp.async.cg (L2 only, never a stale L1 line).
template <int N0, int N1, int N2, int S, int G, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_twopass_pipe(const cx<double> *__restrict__ in, cx<double> *__restrict__ out, long long nvol,
                   double scale, int *err, unsigned char *work, int R, int D)
{
    pdl_begin();
    using T = double;
    using TG = TwoPassGeom<N0, N1, N2, T, G>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    constexpr int STAGE = TG::SMEM;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ long long s_tk[2];
    __shared__ int s_next;  // 1: next item's load issued, 0: deferred, -1: no next item
    __shared__ int s_stop;
    TwoPassCtl *ctl = reinterpret_cast<TwoPassCtl *>(work);
    cx<T> *ring = reinterpret_cast<cx<T> *>(work + TWOPASS_CTL_BYTES);
    const int tid = threadIdx.x;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    auto stage = [&](int s) { return reinterpret_cast<cx<T> *>(smraw + s * STAGE); };
    auto issue = [&](const TwoPassItem &it, int s) {
        cx<T> *sm = stage(s);
        if (it.plane) {
            const cx<T> *src = in + it.vol * TG::V;
            for (int g = tid; g < TG::PLANE_ELEMS; g += NT) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                cp_async_16(sm + so, src + vo);
            }
        } else {
            const cx<T> *sv = ring + (it.vol % R) * TG::V;
            for (int g = tid; g < TG::ROW_ELEMS; g += NT) {
                long long vo;
                int so;
                twopass_row_elem<TG>(it.j, g, &vo, &so);
                cp_async_16(sm + so, sv + vo);
            }
        }
        cp_async_commit();
    };
    auto plane_target = [&](const TwoPassItem &it) { return (unsigned)TG::NA * (unsigned)(it.vol / R + 1); };

    int cur = 0;
    if (tid == 0) {
        const long long t = (long long)atomicAdd(&ctl->ticket, 1ull);
        s_tk[0] = t;
        s_stop = (t >= total || ld_acquire_gpu(&ctl->abort) != 0) ? 1 : 0;
        if (!s_stop) {
            const TwoPassItem it = twopass_decode(t, nvol, TG::NA, TG::NB, D);
            if (!it.plane && !wait_counter_geq(&ctl->cnt[it.vol % R], plane_target(it), &ctl->abort))
                s_stop = 2;
        }
    }
    __syncthreads();
    if (s_stop == 0) issue(twopass_decode(s_tk[0], nvol, TG::NA, TG::NB, D), 0);

    while (s_stop == 0) {
        const TwoPassItem it = twopass_decode(s_tk[cur], nvol, TG::NA, TG::NB, D);
        const int slot = (int)(it.vol % R);
        if (tid == 0) {
            const long long t = (long long)atomicAdd(&ctl->ticket, 1ull);
            s_tk[cur ^ 1] = t;
            int st = -1;
            if (t < total && ld_acquire_gpu(&ctl->abort) == 0) {
                const TwoPassItem nx = twopass_decode(t, nvol, TG::NA, TG::NB, D);
                st = (nx.plane || ld_acquire_gpu(&ctl->cnt[nx.vol % R]) >= plane_target(nx)) ? 1 : 0;
            }
            s_next = st;
        }
        __syncthreads();
        const int nstate = s_next;
        if (nstate == 1) issue(twopass_decode(s_tk[cur ^ 1], nvol, TG::NA, TG::NB, D), cur ^ 1);
        if (nstate == 1) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();
        cx<T> *sm = stage(cur);
        cx<T> *sv = ring + (long long)slot * TG::V;
        if (it.plane) {
            for (int r = tid; r < G * N1; r += NT) pass_z<XG, S, ALG_DEFAULT>(sm, r);
            __syncthreads();
            for (int l = tid; l < G * N2; l += NT) pass_y<XG, S, ALG_DEFAULT>(sm, l);
            if (tid == 0 && !wait_counter_geq(&ctl->cnt[TWOPASS_RMAX + slot],
                                              (unsigned)TG::NB * (unsigned)(it.vol / R), &ctl->abort))
                s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            for (int g = tid; g < TG::PLANE_ELEMS; g += NT) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                st_l2(sv + vo, sm[so]);
            }
            __syncthreads();  // then one cumulative release publishes every thread's stores
            if (tid == 0) red_release_gpu_add(&ctl->cnt[slot], 1u);
        } else {
            // the copies of this row item are complete: drop its rows from L2
            // unwritten, then the slot may be reused
            twopass_discard_rows<TG>(sv, it.j, tid, NT);
            __syncthreads();
            if (tid == 0) red_release_gpu_add(&ctl->cnt[TWOPASS_RMAX + slot], 1u);
            cx<T> *gvol = out + it.vol * TG::V;
            for (int l = tid; l < G * N2; l += NT) pass_x_slab<YG, S, N1>(sm, l, gvol, it.j * G, scale);
        }
        __syncthreads();  // stage `cur` is free again
        if (nstate == -1) break;
        if (nstate == 0) {
            const TwoPassItem nx = twopass_decode(s_tk[cur ^ 1], nvol, TG::NA, TG::NB, D);
            if (tid == 0 && !wait_counter_geq(&ctl->cnt[nx.vol % R], plane_target(nx), &ctl->abort))
                s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            issue(nx, cur ^ 1);
        }
        cur ^= 1;
    }
    cp_async_wait<0>();  // no copy in flight when the CTA leaves

    if (tid == 0 && s_stop == 2) {
        report_error(err, DEV_ERR_DEP_TIMEOUT);
        atomicExch(&ctl->abort, 1u);
    }
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            ctl->ticket = 0ull;
            for (int i = 0; i < 2 * TWOPASS_RMAX; ++i) ctl->cnt[i] = 0u;
            ctl->abort = 0u;
            __threadfence();
            ctl->done = 0u;
        }
    }
}

// TWOPASS with lean item control (complex double, row-major layouts).  Thread
// 0 takes the next ticket while the current item runs.  A row item's
// dependency (the plane items of its volume) is waited for before the barrier
// that starts it; a plane item's (the slot's previous reader) while its input
// rows are in flight, before the y pass stores into the slot.  The abort flag
// is read only inside waits that do not return at once.  A CTA
// holds at most two tickets and works them in increasing order, so the
// smallest unfinished ticket always belongs to a CTA that can run it: the
// ticket-order argument against deadlock still holds.
//
// Plane items move their G planes into shared memory by bulk copies and run
// the z pass there; the y pass stores straight into the scratch slot from
// registers (L2-only stores).  Row items either load their x-lines straight
// from the slot into registers (L2-only loads, a warp reading contiguous
// ranges; no shared memory at all, "regs" in the name) or gather their rows by
// bulk copies first (XBULK, "bulkqh").  HINT adds the L2 policies: input rows
// evict_first, ring stores evict_last.
template <int N0, int N1, int N2, int S, int G, int NT, int MINB, bool XBULK = false,
          bool HINT = false, typename T = double, int PITCH = 0>
__global__ void __launch_bounds__(NT, MINB)
    k_twopass_regs(const cx<T> *__restrict__ in, cx<T> *__restrict__ out, long long nvol, T scale,
                   int *err, unsigned char *work, int R, int D)
{
    pdl_begin();
    using TG = TwoPassGeom<N0, N1, N2, T, G, PITCH>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    static_assert(XG::POL != 2 && YG::POL != 2 && NT % 32 == 0, "row-major layouts, whole warps");
    constexpr uint32_t ROW_BYTES = (uint32_t)(N2 * sizeof(cx<T>));
    static_assert(ROW_BYTES % 16 == 0 && (XG::P2 * XG::EB) % 16 == 0,
                  "bulk row copies: 16-byte rows at 16-byte aligned shared-memory starts");
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    __shared__ long long s_t;
    __shared__ int s_stop;
    __shared__ __align__(8) uint64_t s_bar;
    TwoPassCtl *ctl = reinterpret_cast<TwoPassCtl *>(work);
    cx<T> *ring = reinterpret_cast<cx<T> *>(work + TWOPASS_CTL_BYTES);
    const int tid = threadIdx.x;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    uint32_t phase = 0;
    bool copies_pending = false;
    long long next = 0;  // thread 0: the ticket taken ahead
    uint64_t pol_first = 0, pol_last = 0;
    if constexpr (HINT) {
        pol_first = l2_policy_evict_first();
        pol_last = l2_policy_evict_last();
    }
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        fence_mbar_init();
        next = (long long)atomicAdd(&ctl->ticket, 1ull);
    }
    // bounded wait for all bulk copies of the current phase; false on timeout
    auto wait_copies = [&]() {
        copies_pending = true;
        const bool ok = mbar_wait_bounded(&s_bar, phase);
        phase ^= 1u;
        if (ok) copies_pending = false;
        return ok;
    };

    for (;;) {
        if (tid == 0) {
            const long long t = next;
            int stop = t >= total ? 1 : 0;
            if (!stop) {
                next = (long long)atomicAdd(&ctl->ticket, 1ull);
                const TwoPassItem it = twopass_decode(t, nvol, TG::NA, TG::NB, D);
                // a row item reads its slot: its plane items must be done first
                const unsigned target = (unsigned)TG::NA * (unsigned)(it.vol / R + 1);
                if (!it.plane && !wait_counter_geq(&ctl->cnt[it.vol % R], target, &ctl->abort)) stop = 2;
            }
            s_t = t;
            s_stop = stop;
        }
        __syncthreads();
        if (s_stop) break;
        const TwoPassItem it = twopass_decode(s_t, nvol, TG::NA, TG::NB, D);
        const int slot = (int)(it.vol % R);
        cx<T> *sv = ring + (long long)slot * TG::V;

        if (it.plane) {
            // 1. G contiguous planes of the input, one bulk copy per row
            if (tid == 0) mbar_arrive_expect_tx(&s_bar, (uint32_t)XG::ROWS * ROW_BYTES);
            const cx<T> *rows = in + it.vol * TG::V + (long long)it.j * G * N1 * N2;
            for (int r = tid; r < XG::ROWS; r += NT) {
                if constexpr (HINT)  // read once: do not displace the ring
                    bulk_g2s_hint(sm + XG::off(r, 0), rows + (long long)r * N2, ROW_BYTES, &s_bar, pol_first);
                else
                    bulk_g2s(sm + XG::off(r, 0), rows + (long long)r * N2, ROW_BYTES, &s_bar);
            }
            // while the rows are in flight: the slot's previous volume must have
            // been read out before this item's y pass stores into it
            if (tid == 0) {
                const unsigned target = (unsigned)TG::NB * (unsigned)(it.vol / R);
                if (target > 0 && !wait_counter_geq(&ctl->cnt[TWOPASS_RMAX + slot], target, &ctl->abort))
                    s_stop = 2;
            }
            if (!wait_copies()) s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            // 2. z pass in shared memory
            for (int r = tid; r < XG::ROWS; r += NT) pass_z<XG, S, ALG_DEFAULT>(sm, r);
            __syncthreads();
            // 3. y pass into the scratch slot (its previous reader is done: checked in step 1)
            if constexpr (HINT) {
                // ring lines stay in L2 (evict_last): a slot is rewritten in L2, not written back
                for (int l = tid; l < G * N2; l += NT) {
                    const int z = l % N2, g = l / N2;
                    cx<T> v[N1];
#pragma unroll
                    for (int j = 0; j < N1; ++j) v[j] = sm[XG::off(g * N1 + j, z)];
                    dft<N1, S, T>(v);
                    cx<T> *o = sv + (long long)(it.j * G + g) * N1 * N2 + z;
#pragma unroll
                    for (int j = 0; j < N1; ++j) {
                        if constexpr (sizeof(T) == 8)
                            st_cg_hint(reinterpret_cast<double2 *>(o + j * N2), make_double2(v[j].re, v[j].im), pol_last);
                        else
                            st_cg_hint(reinterpret_cast<float2 *>(o + j * N2), make_float2(v[j].re, v[j].im), pol_last);
                    }
                }
            } else {
                for (int l = tid; l < G * N2; l += NT) pass_y_store_l2<XG, S>(sm, l, sv, it.j * G);
            }
            fence_proxy_async_smem();  // these reads before the next item's bulk copies
            __syncthreads();  // then one cumulative release publishes every thread's stores
            if (tid == 0) red_release_gpu_add(&ctl->cnt[slot], 1u);
        } else if constexpr (XBULK) {
            // 1. the G y-rows of every plane of the slot (its plane items are done)
            if (tid == 0) mbar_arrive_expect_tx(&s_bar, (uint32_t)(N0 * G) * ROW_BYTES);
            for (int q = tid; q < N0 * G; q += NT) {
                const int x = q / G, yl = q % G;
                fence_proxy_async_global();  // the acquire above precedes these reads
                bulk_g2s(sm + YG::off(q, 0), sv + ((long long)x * N1 + it.j * G + yl) * N2, ROW_BYTES,
                         &s_bar);
            }
            if (!wait_copies()) s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            // its rows are in shared memory: drop them from L2 unwritten, then
            // the slot may be overwritten
            twopass_discard_rows<TG>(sv, it.j, tid, NT);
            __syncthreads();
            if (tid == 0) red_release_gpu_add(&ctl->cnt[TWOPASS_RMAX + slot], 1u);
            // 2. x pass, straight to the output
            for (int l = tid; l < G * N2; l += NT)
                pass_x_slab<YG, S, N1>(sm, l, out + it.vol * TG::V, it.j * G, scale);
            fence_proxy_async_smem();
            __syncthreads();
        } else {
            // x pass from the scratch slot (its plane items are done: checked above)
            for (int l = tid; l < G * N2; l += NT)
                pass_x_load_l2<N0, N1, N2, S, T>(sv, l, out + it.vol * TG::V, it.j * G, scale);
            __syncthreads();  // every load of the slot has returned
            twopass_discard_rows<TG>(sv, it.j, tid, NT);
            __syncthreads();
            if (tid == 0) red_release_gpu_add(&ctl->cnt[TWOPASS_RMAX + slot], 1u);
        }
    }
    // a bulk copy that timed out may still land: wait once more (bounded)
    if (copies_pending) mbar_wait_bounded(&s_bar, phase ^ 1u);

    if (tid == 0 && s_stop == 2) {
        report_error(err, DEV_ERR_DEP_TIMEOUT);
        atomicExch(&ctl->abort, 1u);
    }
    // The last CTA to leave clears the control block for the next launch.
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            ctl->ticket = 0ull;
            for (int i = 0; i < 2 * TWOPASS_RMAX; ++i) ctl->cnt[i] = 0u;
            ctl->abort = 0u;
            __threadfence();
            ctl->done = 0u;
        }
    }
}

// TWOPASS for N^3 complex double with every line split over P lanes of a warp
// (splitline.cuh lane_split_line: 36 = 2 x 18 Cooley-Tukey or 4 x 9 Good-Thomas),
// under the lean item control, bulk row copies and L2 policies of
// k_twopass_regs ("bulkqh").  A warp holds 32/P lines side by side (lane t of a
// line is LS = 32/P lanes from lane t-1), so a lane keeps N/P points -- 18 or 9
// complex doubles instead of 36 -- and many more warps fit an SM; the price is
// the cross-lane exchange (P = 2: one shuffle stage, P = 4: two).  Rows sit at
// the odd pitch N|1: every 8-lane shared-memory phase touches 8 lines at one
// position, conflict-free along rows and columns.  The z pass works in place
// in shared memory, the y pass stores into the scratch slot from registers,
// the x pass streams the output.  "lanesP" in the name.
template <int N, int S, int G, int NT, int MINB, int P>
__global__ void __launch_bounds__(NT, MINB)
    k_twopass_lanes(const cx<double> *__restrict__ in, cx<double> *__restrict__ out, long long nvol,
                    double scale, int *err, unsigned char *work, int R, int D)
{
    pdl_begin();
    using T = double;
    constexpr int PITCH = N | 1;
    using TG = TwoPassGeom<N, N, N, T, G, PITCH>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    constexpr int LS = 32 / P;                  // lines per warp, lane distance within a line
    constexpr int WARPS = NT / 32;
    constexpr int LINES = G * N;                // lines of one pass of an item
    static_assert(NT % 32 == 0 && 32 % P == 0, "whole warps, P | 32");
    constexpr uint32_t ROW_BYTES = (uint32_t)(N * sizeof(cx<T>));
    static_assert(ROW_BYTES % 16 == 0, "bulk row copies: 16-byte rows");
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    __shared__ long long s_t;
    __shared__ int s_stop;
    __shared__ __align__(8) uint64_t s_bar;
    TwoPassCtl *ctl = reinterpret_cast<TwoPassCtl *>(work);
    cx<T> *ring = reinterpret_cast<cx<T> *>(work + TWOPASS_CTL_BYTES);
    const int tid = threadIdx.x;
    const int warp = tid / 32, lane = tid % 32;
    const int t = lane / LS, lw = lane % LS;   // lane of its line, line slot in the warp
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    uint32_t phase = 0;
    bool copies_pending = false;
    long long next = 0;
    const uint64_t pol_first = l2_policy_evict_first();
    const uint64_t pol_last = l2_policy_evict_last();
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        fence_mbar_init();
        next = (long long)atomicAdd(&ctl->ticket, 1ull);
    }
    auto wait_copies = [&]() {
        copies_pending = true;
        const bool ok = mbar_wait_bounded(&s_bar, phase);
        phase ^= 1u;
        if (ok) copies_pending = false;
        return ok;
    };

    for (;;) {
        if (tid == 0) {
            const long long tk = next;
            int stop = tk >= total ? 1 : 0;
            if (!stop) {
                next = (long long)atomicAdd(&ctl->ticket, 1ull);
                const TwoPassItem it = twopass_decode(tk, nvol, TG::NA, TG::NB, D);
                const unsigned target = (unsigned)TG::NA * (unsigned)(it.vol / R + 1);
                if (!it.plane && !wait_counter_geq(&ctl->cnt[it.vol % R], target, &ctl->abort)) stop = 2;
            }
            s_t = tk;
            s_stop = stop;
        }
        __syncthreads();
        if (s_stop) break;
        const TwoPassItem it = twopass_decode(s_t, nvol, TG::NA, TG::NB, D);
        const int slot = (int)(it.vol % R);
        cx<T> *sv = ring + (long long)slot * TG::V;

        if (it.plane) {
            // 1. G contiguous planes of the input, one bulk copy per row
            if (tid == 0) mbar_arrive_expect_tx(&s_bar, (uint32_t)XG::ROWS * ROW_BYTES);
            const cx<T> *rows = in + it.vol * TG::V + (long long)it.j * G * N * N;
            for (int r = tid; r < XG::ROWS; r += NT)
                bulk_g2s_hint(sm + XG::off(r, 0), rows + (long long)r * N, ROW_BYTES, &s_bar, pol_first);
            if (tid == 0) {
                const unsigned target = (unsigned)TG::NB * (unsigned)(it.vol / R);
                if (target > 0 && !wait_counter_geq(&ctl->cnt[TWOPASS_RMAX + slot], target, &ctl->abort))
                    s_stop = 2;
            }
            if (!wait_copies()) s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            // 2. z pass in place: line = row r
            for (int base = 0; base < LINES; base += WARPS * LS) {
                const int r = base + warp * LS + lw;
                const bool valid = r < LINES;
                cx<T> *row = sm + XG::off(valid ? r : 0, 0);
                lane_split_line<N, P, LS, S, T>(t, valid, [&](int z) { return row[z]; },
                                                 [&](int z, cx<T> v) { row[z] = v; });
            }
            __syncthreads();
            // 3. y pass into the scratch slot: line = (g, z)
            for (int base = 0; base < LINES; base += WARPS * LS) {
                const int l = base + warp * LS + lw;
                const bool valid = l < LINES;
                const int g = valid ? l / N : 0, z = l % N;
                const cx<T> *col = sm + XG::off(g * N, z);
                cx<T> *o = sv + (long long)(it.j * G + g) * N * N + z;
                lane_split_line<N, P, LS, S, T>(
                    t, valid, [&](int y) { return col[y * PITCH]; },
                    [&](int y, cx<T> v) {
                        st_cg_hint(reinterpret_cast<double2 *>(o + y * N), make_double2(v.re, v.im), pol_last);
                    });
            }
            fence_proxy_async_smem();  // these reads before the next item's bulk copies
            __syncthreads();           // then one cumulative release publishes every thread's stores
            if (tid == 0) red_release_gpu_add(&ctl->cnt[slot], 1u);
        } else {
            // 1. the G y-rows of every plane of the slot (its plane items are done)
            if (tid == 0) mbar_arrive_expect_tx(&s_bar, (uint32_t)(N * G) * ROW_BYTES);
            for (int q = tid; q < N * G; q += NT) {
                const int x = q / G, yl = q % G;
                fence_proxy_async_global();  // the acquire above precedes these reads
                bulk_g2s(sm + YG::off(q, 0), sv + ((long long)x * N + it.j * G + yl) * N, ROW_BYTES, &s_bar);
            }
            if (!wait_copies()) s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            // its rows are in shared memory: drop them from L2 unwritten, then
            // the slot may be overwritten
            twopass_discard_rows<TG>(sv, it.j, tid, NT);
            __syncthreads();
            if (tid == 0) red_release_gpu_add(&ctl->cnt[TWOPASS_RMAX + slot], 1u);
            // 2. x pass, straight to the output: line = (yl, z)
            cx<T> *gvol = out + it.vol * TG::V;
            for (int base = 0; base < LINES; base += WARPS * LS) {
                const int l = base + warp * LS + lw;
                const bool valid = l < LINES;
                const int yl = valid ? l / N : 0, z = l % N;
                const cx<T> *col = sm + YG::off(yl, z);
                cx<T> *o = gvol + (long long)(it.j * G + yl) * N + z;
                lane_split_line<N, P, LS, S, T>(
                    t, valid, [&](int x) { return col[x * G * PITCH]; },
                    [&](int x, cx<T> v) {
                        if constexpr (S > 0) v = cscale(v, scale);
                        store_out(o + (long long)x * N * N, v);
                    });
            }
            fence_proxy_async_smem();
            __syncthreads();
        }
    }
    if (copies_pending) mbar_wait_bounded(&s_bar, phase ^ 1u);

    if (tid == 0 && s_stop == 2) {
        report_error(err, DEV_ERR_DEP_TIMEOUT);
        atomicExch(&ctl->abort, 1u);
    }
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            ctl->ticket = 0ull;
            for (int i = 0; i < 2 * TWOPASS_RMAX; ++i) ctl->cnt[i] = 0u;
            ctl->abort = 0u;
            __threadfence();
            ctl->done = 0u;
        }
    }
}

// TWOPASS for N^3 with every line split into two thread-level stages
// (staged.cuh: 64 = 8 x 8 Cooley-Tukey, 45 = 5 x 9 Good-Thomas): one plane or
// one y-row per item, a task holds 5 to 9 points, so many warps fit an SM --
// where an N-point line in one thread spills (64) or leaves 8 warps per SM
// (45).  Rows are held at pitch P (odd for complex double: bank-conflict-free
// rows and columns; even for complex float, whose rows must start 16-byte
// aligned for the bulk copies) and moved by bulk copies.  The z pass runs in
// place, leaving each row in Line::slot order; the y pass's second stage
// stores into the scratch slot at the natural z; the row item's second stage
// streams the output.  Item control, L2 policies and the slot release as in
// k_twopass_regs.
template <class Line, typename T>
constexpr int staged_pitch() { return sizeof(T) == 8 ? (Line::N | 1) : ((Line::N + 2) & ~1); }

template <class Line, int S, int NT, int MINB, typename T = double>
__global__ void __launch_bounds__(NT, MINB)
    k_twopass_staged(const cx<T> *__restrict__ in, cx<T> *__restrict__ out, long long nvol, T scale,
                     int *err, unsigned char *work, int R, int D)
{
    pdl_begin();
    constexpr int N = Line::N, P = staged_pitch<Line, T>();
    static_assert((N * sizeof(cx<T>)) % 16 == 0 && (P * sizeof(cx<T>)) % 16 == 0,
                  "bulk row copies: 16-byte rows at 16-byte aligned shared-memory starts");
    using TG = TwoPassGeom<N, N, N, T, 1>;
    static_assert(NT % 32 == 0, "whole warps");
    constexpr uint32_t ROW_BYTES = (uint32_t)(N * sizeof(cx<T>));
    constexpr long long PLANE = (long long)N * N;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    __shared__ long long s_t;
    __shared__ int s_stop;
    __shared__ __align__(8) uint64_t s_bar;
    TwoPassCtl *ctl = reinterpret_cast<TwoPassCtl *>(work);
    cx<T> *ring = reinterpret_cast<cx<T> *>(work + TWOPASS_CTL_BYTES);
    const int tid = threadIdx.x;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;
    uint32_t phase = 0;
    bool copies_pending = false;
    long long next = 0;  // thread 0: the ticket taken ahead
    const uint64_t pol_first = l2_policy_evict_first(), pol_last = l2_policy_evict_last();
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        fence_mbar_init();
        next = (long long)atomicAdd(&ctl->ticket, 1ull);
    }
    auto wait_copies = [&]() {
        copies_pending = true;
        const bool ok = mbar_wait_bounded(&s_bar, phase);
        phase ^= 1u;
        if (ok) copies_pending = false;
        return ok;
    };
    auto rowaddr = [](int l, int e) { return l * P + e; };  // element e of row l
    auto coladdr = [](int l, int e) { return e * P + l; };  // element e of column l

    for (;;) {
        if (tid == 0) {
            const long long t = next;
            int stop = t >= total ? 1 : 0;
            if (!stop) {
                next = (long long)atomicAdd(&ctl->ticket, 1ull);
                const TwoPassItem it = twopass_decode(t, nvol, TG::NA, TG::NB, D);
                // a row item reads its slot: its plane items must be done first
                const unsigned target = (unsigned)TG::NA * (unsigned)(it.vol / R + 1);
                if (!it.plane && !wait_counter_geq(&ctl->cnt[it.vol % R], target, &ctl->abort)) stop = 2;
            }
            s_t = t;
            s_stop = stop;
        }
        __syncthreads();
        if (s_stop) break;
        const TwoPassItem it = twopass_decode(s_t, nvol, TG::NA, TG::NB, D);
        const int slot = (int)(it.vol % R);
        cx<T> *sv = ring + (long long)slot * TG::V;

        if (it.plane) {
            // 1. x-plane j of the input, one bulk copy per y-row (read once: evict_first)
            if (tid == 0) mbar_arrive_expect_tx(&s_bar, (uint32_t)N * ROW_BYTES);
            const cx<T> *rows = in + it.vol * TG::V + (long long)it.j * PLANE;
            for (int r = tid; r < N; r += NT)
                bulk_g2s_hint(sm + r * P, rows + (long long)r * N, ROW_BYTES, &s_bar, pol_first);
            // while the rows are in flight: the slot's previous volume must have
            // been read out before this item's y pass stores into it
            if (tid == 0) {
                const unsigned target = (unsigned)TG::NB * (unsigned)(it.vol / R);
                if (target > 0 && !wait_counter_geq(&ctl->cnt[TWOPASS_RMAX + slot], target, &ctl->abort))
                    s_stop = 2;
            }
            if (!wait_copies()) s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            // 2. z pass along the rows, in place (rows end in Line::slot order)
            for (int t = tid; t < N * Line::T1; t += NT) Line::template stage1<S, T>(sm, N, t, rowaddr);
            __syncthreads();
            for (int t = tid; t < N * Line::T2; t += NT)
                Line::template stage2<S, T>(sm, N, t, rowaddr,
                                            [&](int l, int k, cx<T> v) { sm[rowaddr(l, Line::slot(k))] = v; });
            __syncthreads();
            // 3. y pass along the columns; column p holds z = Line::at(p)
            for (int t = tid; t < N * Line::T1; t += NT) Line::template stage1<S, T>(sm, N, t, coladdr);
            __syncthreads();
            cx<T> *dst = sv + (long long)it.j * PLANE;
            for (int t = tid; t < N * Line::T2; t += NT)
                Line::template stage2<S, T>(sm, N, t, coladdr, [&](int p, int k, cx<T> v) {
                    cx<T> *o = dst + k * N + Line::at(p);
                    if constexpr (sizeof(T) == 8)
                        st_cg_hint(reinterpret_cast<double2 *>(o), make_double2(v.re, v.im), pol_last);
                    else
                        st_cg_hint(reinterpret_cast<float2 *>(o), make_float2(v.re, v.im), pol_last);
                });
            fence_proxy_async_smem();  // these reads before the next item's bulk copies
            __syncthreads();  // then one cumulative release publishes every thread's stores
            if (tid == 0) red_release_gpu_add(&ctl->cnt[slot], 1u);
        } else {
            // 1. y-row j of every x-plane of the slot (its plane items are done)
            if (tid == 0) mbar_arrive_expect_tx(&s_bar, (uint32_t)N * ROW_BYTES);
            for (int x = tid; x < N; x += NT) {
                fence_proxy_async_global();  // the acquire above precedes these reads
                bulk_g2s(sm + x * P, sv + ((long long)x * N + it.j) * N, ROW_BYTES, &s_bar);
            }
            if (!wait_copies()) s_stop = 2;
            __syncthreads();
            if (s_stop) break;
            // its rows are in shared memory: drop them from L2 unwritten, then
            // the slot may be overwritten
            twopass_discard_rows<TG>(sv, it.j, tid, NT);
            __syncthreads();
            if (tid == 0) red_release_gpu_add(&ctl->cnt[TWOPASS_RMAX + slot], 1u);
            // 2. x pass along the columns (column z), streamed to the output
            for (int t = tid; t < N * Line::T1; t += NT) Line::template stage1<S, T>(sm, N, t, coladdr);
            __syncthreads();
            cx<T> *gvol = out + it.vol * TG::V + (long long)it.j * N;
            for (int t = tid; t < N * Line::T2; t += NT)
                Line::template stage2<S, T>(sm, N, t, coladdr, [&](int z, int k, cx<T> v) {
                    if constexpr (S > 0) v = cscale(v, scale);
                    store_out(gvol + k * PLANE + z, v);
                });
            fence_proxy_async_smem();
            __syncthreads();
        }
    }
    // a bulk copy that timed out may still land: wait once more (bounded)
    if (copies_pending) mbar_wait_bounded(&s_bar, phase ^ 1u);

    if (tid == 0 && s_stop == 2) {
        report_error(err, DEV_ERR_DEP_TIMEOUT);
        atomicExch(&ctl->abort, 1u);
    }
    // The last CTA to leave clears the control block for the next launch.
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            ctl->ticket = 0ull;
            for (int i = 0; i < 2 * TWOPASS_RMAX; ++i) ctl->cnt[i] = 0u;
            ctl->abort = 0u;
            __threadfence();
            ctl->done = 0u;
        }
    }
}

int twopass_ring(const KernelEntry &e, long long grid, int *lag)
{
    // The lag covers up to twice the tickets the grid holds at once: kernels
    // that take their next ticket ahead (k_twopass_regs, k_twopass_staged) hold
    // two per CTA, and for the others too a lag of two grids' worth measured
    // faster on B200 (fewer row items arriving before their planes are done).
    // It is shortened, down to one grid's worth, while the ring would exceed
    // 64 MB, so that the ring stays in half of L2.
    const int na = e.n0 / e.vpc, nb = e.n1 / e.vpc;
    const long long vbytes = (long long)e.n0 * e.n1 * e.n2 * element_bytes(e.precision);
    long long held = 2 * grid;
    int r = twopass_ring_size(na, nb, held, lag);
    while (held > grid && (long long)r * vbytes > (64LL << 20)) {
        held = std::max(grid, held - (long long)(na + nb));
        r = twopass_ring_size(na, nb, held, lag);
    }
    return r;
}

size_t entry_workspace_bytes(const KernelEntry &e, int grid_limit)
{
    if (e.family != FAM_TWOPASS) return 0;
    int lag = 0;
    const int r = twopass_ring(e, grid_limit, &lag);
    return TWOPASS_CTL_BYTES + (size_t)r * (size_t)e.n0 * e.n1 * e.n2 * (size_t)element_bytes(e.precision);
}

template <int N0, int N1, int N2, typename T, int S, int G, int NT, int MINB>
static void add_twopass(std::vector<KernelEntry> &out, const char *name)
{
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_TWOPASS;
    e.vpc = G;
    e.threads = NT;
    e.smem = TwoPassGeom<N0, N1, N2, T, G>::SMEM;
    e.alg = 0;
    e.func = (const void *)&k_twopass<N0, N1, N2, T, S, G, NT, MINB>;
    e.name = name;
    out.push_back(e);
}

#define FFT3D_TWOPASS(N0, N1, N2, T, G, NT, MINB)                                              \
    add_twopass<N0, N1, N2, T, -1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " " #T    \
                                                     " g" #G " nt" #NT " minb" #MINB);         \
    add_twopass<N0, N1, N2, T, +1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " " #T    \
                                                     " g" #G " nt" #NT " minb" #MINB)

template <int N0, int N1, int N2, int S, int G, int NT, int MINB>
static void add_twopass_pipe(std::vector<KernelEntry> &out, const char *name)
{
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = FFT3D_B200_C128;
    e.sign = S;
    e.family = FAM_TWOPASS;  // same launch arguments and workspace as k_twopass
    e.alg = 2;
    e.vpc = G;
    e.threads = NT;
    e.smem = 2 * TwoPassGeom<N0, N1, N2, double, G>::SMEM;
    e.func = (const void *)&k_twopass_pipe<N0, N1, N2, S, G, NT, MINB>;
    e.name = name;
    out.push_back(e);
}

template <int N0, int N1, int N2, int S, int G, int NT, int MINB, bool XBULK = false,
          bool HINT = false, typename T = double, int PITCH = 0>
static void add_twopass_regs(std::vector<KernelEntry> &out, const char *name)
{
    using TG = TwoPassGeom<N0, N1, N2, T, G, PITCH>;
    using XG = typename TG::XG;
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_TWOPASS;  // same launch arguments and workspace as k_twopass
    e.alg = 8 + (XBULK ? 32 : 0) + (HINT ? 128 : 0);
    e.vpc = G;
    e.threads = NT;
    // plane items only, unless row items gather their rows into shared memory too
    e.smem = XBULK ? TG::SMEM : ((XG::PV * XG::EB) + 127) / 128 * 128;
    e.func = (const void *)&k_twopass_regs<N0, N1, N2, S, G, NT, MINB, XBULK, HINT, T, PITCH>;
    e.name = name;
    out.push_back(e);
}

// Passes straight between registers and L2, complex double: "regs" in the name.
#define FFT3D_TWOPASS_REGS(N0, N1, N2, G, NT, MINB)                                              \
    add_twopass_regs<N0, N1, N2, -1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " double g" #G \
                                                       " regs nt" #NT " minb" #MINB);              \
    add_twopass_regs<N0, N1, N2, +1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " double g" #G \
                                                       " regs nt" #NT " minb" #MINB)

// Lean control, bulk row gathers, L2 policies: input planes evict_first, ring stores
// evict_last ("bulkqh").
#define FFT3D_TWOPASS_BULKQH(N0, N1, N2, G, NT, MINB)                                            \
    add_twopass_regs<N0, N1, N2, -1, G, NT, MINB, true, true>(                             \
        out, "twopass " #N0 "x" #N1 "x" #N2 " double g" #G " bulkqh nt" #NT " minb" #MINB);      \
    add_twopass_regs<N0, N1, N2, +1, G, NT, MINB, true, true>(                             \
        out, "twopass " #N0 "x" #N1 "x" #N2 " double g" #G " bulkqh nt" #NT " minb" #MINB)
// bulkqh for complex float at an explicit even row pitch (bulk rows need
// 16-byte aligned shared-memory starts): "bulkqh" with "float" in the name.
#define FFT3D_TWOPASS_BULKQH_F(N0, N1, N2, G, NT, MINB, PITCH)                                    \
    add_twopass_regs<N0, N1, N2, -1, G, NT, MINB, true, true, float, PITCH>(                \
        out, "twopass " #N0 "x" #N1 "x" #N2 " float g" #G " bulkqh nt" #NT " minb" #MINB);        \
    add_twopass_regs<N0, N1, N2, +1, G, NT, MINB, true, true, float, PITCH>(                \
        out, "twopass " #N0 "x" #N1 "x" #N2 " float g" #G " bulkqh nt" #NT " minb" #MINB)

template <int N, int S, int G, int NT, int MINB, int P>
static void add_twopass_lanes(std::vector<KernelEntry> &out, const char *name)
{
    using TG = TwoPassGeom<N, N, N, double, G, (N | 1)>;
    KernelEntry e;
    e.n0 = e.n1 = e.n2 = N;
    e.precision = FFT3D_B200_C128;
    e.sign = S;
    e.family = FAM_TWOPASS;  // same launch arguments and workspace as k_twopass
    e.alg = 1024 + P;
    e.vpc = G;
    e.threads = NT;
    e.smem = TG::SMEM;
    e.func = (const void *)&k_twopass_lanes<N, S, G, NT, MINB, P>;
    e.name = name;
    out.push_back(e);
}

// Lines split over P lanes of a warp, lean control: "lanesP" in the name.
#define FFT3D_TWOPASS_LANES(N, G, NT, MINB, P)                                                    \
    add_twopass_lanes<N, -1, G, NT, MINB, P>(out, "twopass " #N "x" #N "x" #N " double g" #G      \
                                                  " lanes" #P " nt" #NT " minb" #MINB);          \
    add_twopass_lanes<N, +1, G, NT, MINB, P>(out, "twopass " #N "x" #N "x" #N " double g" #G      \
                                                  " lanes" #P " nt" #NT " minb" #MINB)

template <class Line, int S, int NT, int MINB, typename T = double>
static void add_twopass_staged(std::vector<KernelEntry> &out, const char *name)
{
    KernelEntry e;
    e.n0 = e.n1 = e.n2 = Line::N;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_TWOPASS;  // same launch arguments and workspace as k_twopass
    e.alg = 512;
    e.vpc = 1;
    e.threads = NT;
    e.smem = Line::N * staged_pitch<Line, T>() * (int)sizeof(cx<T>);
    e.func = (const void *)&k_twopass_staged<Line, S, NT, MINB, T>;
    e.name = name;
    out.push_back(e);
}

// Lines split into two stages: "ct" (64 = 8 x 8) or "pfa" (45 = 5 x 9) in the name.
#define FFT3D_TWOPASS_STAGED(LINE, N, T, KIND, NT, MINB)                                           \
    add_twopass_staged<LINE, -1, NT, MINB, T>(out, "twopass " #N "x" #N "x" #N " " #T " g1 " KIND  \
                                                   " nt" #NT " minb" #MINB);                        \
    add_twopass_staged<LINE, +1, NT, MINB, T>(out, "twopass " #N "x" #N "x" #N " " #T " g1 " KIND  \
                                                   " nt" #NT " minb" #MINB)

// Two-stage pipeline, complex double: "pipe" in the name.
#define FFT3D_TWOPASS_PIPE(N0, N1, N2, G, NT, MINB)                                              \
    add_twopass_pipe<N0, N1, N2, -1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " double g" #G \
                                                       " pipe nt" #NT " minb" #MINB);              \
    add_twopass_pipe<N0, N1, N2, +1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " double g" #G \
                                                       " pipe nt" #NT " minb" #MINB)

// The candidates the autotuner races.  Measured on B200 (forward, in the
// tuner's race): every variant kept here wins, or comes within a few per cent
// of the winner, at some batch size -- 4, 16 or 256 volumes of 36^3, 128 of
// 45^3, 64 of 64^3 -- or is the only kernel for its extent and precision.
void register_twopass_kernels(std::vector<KernelEntry> &out)
{
    // 36^3 complex double: one line per thread, lean control, bulk rows, L2
    // policies (256 volumes: 124 us); lines over 4 lanes (4 and 16 volumes)
    FFT3D_TWOPASS_BULKQH(36, 36, 36, 3, 128, 3);
    FFT3D_TWOPASS_BULKQH(36, 36, 36, 2, 96, 4);
    FFT3D_TWOPASS_LANES(36, 2, 288, 3, 4);
    FFT3D_TWOPASS_REGS(36, 36, 36, 2, 96, 3);
    FFT3D_TWOPASS_PIPE(36, 36, 36, 2, 96, 2);
    // 36^3 complex float at an explicit even row pitch of 38
    FFT3D_TWOPASS_BULKQH_F(36, 36, 36, 3, 128, 5, 38);
    FFT3D_TWOPASS_BULKQH_F(36, 36, 36, 2, 96, 6, 38);
    FFT3D_TWOPASS_BULKQH_F(36, 36, 36, 4, 160, 3, 38);
    // 45^3: complex double five planes per item; 45 = 5 x 9 staged lines
    FFT3D_TWOPASS_BULKQH(45, 45, 45, 5, 256, 1);
    FFT3D_TWOPASS_STAGED(LinePFA45, 45, double, "pfa", 128, 6);
    // 45^3 complex float (a 360-byte row cannot be a bulk copy): element copies
    // 30^3 complex128 (446 KB a volume), a test geometry of the reference
    FFT3D_TWOPASS(30, 30, 30, double, 3, 96, 4);
    FFT3D_TWOPASS(30, 30, 30, double, 5, 160, 3);
    FFT3D_TWOPASS(45, 45, 45, float, 5, 256, 2);
    FFT3D_TWOPASS(45, 45, 45, float, 3, 160, 3);
    // 64^3: 64 = 8 x 8 staged lines, one plane or y-row per item
    FFT3D_TWOPASS_STAGED(LineCT64, 64, double, "ct", 128, 3);
    FFT3D_TWOPASS_STAGED(LineCT64, 64, double, "ct", 256, 3);
    FFT3D_TWOPASS_STAGED(LineCT64, 64, float, "ct", 128, 6);
    FFT3D_TWOPASS_STAGED(LineCT64, 64, float, "ct", 256, 3);
    FFT3D_TWOPASS(64, 64, 64, float, 2, 128, 3);
    FFT3D_TWOPASS(64, 64, 64, float, 4, 256, 1);
}

}  // namespace fft3d

// stream_kernels.cu -- kernel family STREAM: persistent CTAs with an NSTAGE-deep
// shared-memory ring.
//
// Each CTA walks the volume groups (VPC volumes each) item = blockIdx.x +
// k*gridDim.x.  While the three passes of item k run out of stage k % NSTAGE, the
// loads of items k+1 .. k+NSTAGE-1 are already in flight into the other stages,
// so HBM reads overlap the arithmetic; the x pass writes results straight to HBM
// with coalesced streaming stores, so a stage is free again as soon as its last
// pass has read it.  NSTAGE = 1 with MINB = 2 puts two single-stage CTAs on an
// SM instead: one loads while the other computes.  BST variants ("bst") leave
// the x pass's results in the stage in natural layout and move the finished
// group to HBM with one bulk copy (TMA) issued by thread 0, so no thread waits on
// its output stores; the stage is refilled after the next item's z pass, once
// that copy has read it.  Natural layouts transform the x lines in place; padded
// and swizzled ones (one x line per thread) transform into registers and, after
// a barrier, store the lines at their natural places.
//
// Loaders:
//   BULK   (natural layout, odd n2): thread 0 issues one cp.async.bulk (TMA)
//          per item -- the group is one contiguous byte range -- completing on
//          the stage's mbarrier.  Items that are not 16-byte aligned in address
//          or size (complex64 tails of odd volumes) are copied by the threads.
//   ASYNC  (padded or XOR-swizzled layouts): every thread issues cp.async copies
//          of its elements straight into their layout slots.
// Every mbarrier wait is bounded (ptx.cuh); a timeout records an error code in
// the plan's device error word and the CTA leaves after a bounded drain.
#include "internal.h"
#include "ptx.cuh"
#include "volume.cuh"

namespace fft3d {

constexpr int LOADER_BULK = 0;
constexpr int LOADER_ASYNC = 1;

template <class G, int VPC, int NSTAGE>
struct StreamLayout {
    // stage size rounded to 128 bytes; NSTAGE mbarriers after the stages
    static constexpr int STAGE_BYTES = ((VPC * G::PV * G::EB) + 127) / 128 * 128;
    static constexpr int SMEM_BYTES = NSTAGE * STAGE_BYTES + 8 * NSTAGE;
};

// Threads copy element by element (synchronous), used for unaligned BULK items.
template <class G>
__device__ __forceinline__ void load_lsu(cx<typename G::T> *stage, const cx<typename G::T> *gin,
                                         int nel, int tid, int nt)
{
    for (int g = tid; g < nel; g += nt) stage_in<G>(stage, gin, g);
}

template <class G, int NT>
__device__ __forceinline__ void load_async(cx<typename G::T> *stage, const cx<typename G::T> *gin,
                                           int nel, int tid)
{
    for (int g = tid; g < nel; g += NT) {
        const int vol = g / G::V;
        const int rem = g - vol * G::V;
        const int r = vol * G::ROWS + rem / G::N2;
        const int z = rem % G::N2;
        if constexpr (G::EB == 16) cp_async_16(stage + G::off(r, z), gin + g);
        else cp_async_8(stage + G::off(r, z), gin + g);
    }
}

// Wait until at most `pending` cp.async groups of this thread are in flight.
__device__ __forceinline__ void cp_async_wait_pending(int pending)
{
    switch (pending) {
    case 0: cp_async_wait<0>(); break;
    case 1: cp_async_wait<1>(); break;
    case 2: cp_async_wait<2>(); break;
    default: cp_async_wait<3>(); break;
    }
}

template <class G, int S, int ALG, int VPC, int NT, int LOADER, int NSTAGE, int MINB, bool BST>
__global__ void __launch_bounds__(NT, MINB)
    k_stream(const cx<typename G::T> *__restrict__ in, cx<typename G::T> *__restrict__ out,
             long long nvol, typename G::T scale, int *err)
{
    static_assert(NSTAGE >= 1 && NSTAGE <= 4, "ring depth");
    static_assert(!BST || NSTAGE >= 2, "bulk stores need a ring at least two deep");
    static_assert(!BST || G::POL == 0 || VPC * G::N1 * G::N2 <= NT,
                  "padded or swizzled layouts re-lay one x line per thread");
    pdl_begin();
    using T = typename G::T;
    using SL = StreamLayout<G, VPC, NSTAGE>;
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + NSTAGE * SL::STAGE_BYTES);
    __shared__ int s_abort;
    auto stage = [&](int s) { return reinterpret_cast<cx<T> *>(smraw + s * SL::STAGE_BYTES); };

    const int tid = threadIdx.x;
    const long long nitems = (nvol + VPC - 1) / VPC;
    const long long stride = gridDim.x;
    if (tid == 0) {
        if constexpr (LOADER == LOADER_BULK) {
            for (int s = 0; s < NSTAGE; ++s) mbar_init(&bar[s], 1);
            fence_mbar_init();
        }
        s_abort = 0;
    }
    __syncthreads();

    // Issue the load of `item` into stage s.  For BULK, returns with the copy in
    // flight (or, for an unaligned item, done by the threads and arrived).
    // Both directions walk their items in order.  Starting an inverse on the
    // items a preceding forward wrote last (still partly in L2) -- walking them
    // from last to first, or from the last 32 MB of the batch and wrapping --
    // measured 0.6% slower over a forward + inverse step and 4-5% slower for an
    // inverse alone.
    auto phys = [&](long long item) { return item; };
    const uint64_t pol_first = l2_policy_evict_first();
    auto issue = [&](long long item, int s) {
        const long long v0 = phys(item) * VPC;
        const int nv = (int)((nvol - v0) < VPC ? (nvol - v0) : VPC);
        const cx<T> *gin = in + v0 * G::V;
        const int nel = nv * G::V;
        if constexpr (LOADER == LOADER_BULK) {
            const uint32_t bytes = (uint32_t)nel * (uint32_t)G::EB;
            const bool aligned = ((((uintptr_t)gin) | bytes) & 15u) == 0;
            if (aligned) {
                if (tid == 0) {  // read once: keep L2 for the output
                    mbar_arrive_expect_tx(&bar[s], bytes);
                    bulk_g2s_hint(stage(s), gin, bytes, &bar[s], pol_first);
                }
            } else {
                load_lsu<G>(stage(s), gin, nel, tid, NT);
                __syncthreads();
                if (tid == 0) mbar_arrive(&bar[s]);
            }
        } else {
            load_async<G, NT>(stage(s), gin, nel, tid);
            cp_async_commit();
        }
    };

    long long item = blockIdx.x;
    for (int j = 0; j < NSTAGE - 1; ++j)
        if (item + j * stride < nitems) issue(item + j * stride, j);
    int k = 0;
    for (; item < nitems; item += stride, ++k) {
        const int cur = k % NSTAGE;
        const long long ahead = item + (long long)(NSTAGE - 1) * stride;
        if constexpr (!BST)
            if (ahead < nitems) issue(ahead, (k + NSTAGE - 1) % NSTAGE);

        if constexpr (LOADER == LOADER_BULK) {
            if (!mbar_wait_bounded(&bar[cur], (uint32_t)((k / NSTAGE) & 1))) s_abort = 1;
        } else {
            int later = 0;  // groups committed after this item's (BST issues its look-ahead later)
            for (int j = 1; j < NSTAGE - (BST ? 1 : 0); ++j)
                if (item + j * stride < nitems) ++later;
            cp_async_wait_pending(later);
        }
        __syncthreads();
        if (s_abort) break;

        const long long v0 = phys(item) * VPC;
        const int nv = (int)((nvol - v0) < VPC ? (nvol - v0) : VPC);
        cx<T> *sm = stage(cur);
        for (int r = tid; r < nv * G::ROWS; r += NT) pass_z<G, S, ALG>(sm, r);
        if constexpr (BST)  // the stage refilled next held the previous item: its store has read it
            if (tid == 0) bulk_wait_read<0>();
        __syncthreads();
        if constexpr (BST)
            if (ahead < nitems) issue(ahead, (k + NSTAGE - 1) % NSTAGE);
        for (int l = tid; l < nv * G::N0 * G::N2; l += NT) pass_y<G, S, ALG>(sm, l);
        __syncthreads();
        cx<T> *gout = out + v0 * G::V;
        if constexpr (BST) {
            // x pass in place, then one bulk store of the group (plain L2 policy:
            // a following transform of this output finds its last part in L2)
            if constexpr (G::POL == 0) {
                for (int l = tid; l < nv * G::N1 * G::N2; l += NT) pass_x<G, S, ALG>(sm, l, scale);
            } else {
                cx<T> v[G::N0];
                const bool line = tid < nv * G::N1 * G::N2;
                if (line) pass_x_regs<G, S, ALG>(sm, tid, scale, v);
                __syncthreads();
                if (line) store_x_natural<G>(sm, tid, v);
            }
            fence_proxy_async_smem();
            __syncthreads();
            const uint32_t bytes = (uint32_t)(nv * G::V) * (uint32_t)G::EB;
            if (((((uintptr_t)gout) | bytes) & 15u) == 0) {
                if (tid == 0) {
                    bulk_s2g(gout, sm, bytes);
                    bulk_commit();
                }
            } else {
                for (int g = tid; g < nv * G::V; g += NT) gout[g] = sm[g];
                fence_proxy_async_smem();
            }
        } else {
            // plain stores: a following transform of this output finds its last part in L2
            for (int l = tid; l < nv * G::N1 * G::N2; l += NT) pass_x_out<G, S, ALG, true>(sm, l, gout, scale);
            if constexpr (LOADER == LOADER_BULK) fence_proxy_async_smem();
            __syncthreads();
        }
    }

    if (s_abort) {
        if (tid == 0) report_error(err, DEV_ERR_LOAD_TIMEOUT);
        // bounded drain of the stage that timed out and of the loads issued ahead of it
        if constexpr (LOADER == LOADER_BULK) {
            // BST issues an item's look-ahead load after its z pass: one fewer in flight
            for (int j = 0; j < NSTAGE - (BST ? 1 : 0); ++j)
                if (item + j * stride < nitems)
                    mbar_wait_bounded(&bar[(k + j) % NSTAGE], (uint32_t)(((k + j) / NSTAGE) & 1));
        } else {
            cp_async_wait<0>();
        }
    }
    if constexpr (BST)  // the stores read this CTA's shared memory until they complete
        if (tid == 0) bulk_wait<0>();
}

template <int N0, int N1, int N2, typename T, int S, int ALG, int VPC, int NT, int NSTAGE,
          int MINB, bool BST = false>
static void add_stream(std::vector<KernelEntry> &out, const char *name)
{
    using G = Geom<N0, N1, N2, T>;
    constexpr int LOADER = (G::POL == 0) ? LOADER_BULK : LOADER_ASYNC;
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_STREAM;
    e.alg = ALG;
    e.vpc = VPC;
    e.threads = NT;
    e.smem = StreamLayout<G, VPC, NSTAGE>::SMEM_BYTES;
    e.func = (const void *)&k_stream<G, S, ALG, VPC, NT, LOADER, NSTAGE, MINB, BST>;
    e.name = name;
    out.push_back(e);
}

#define FFT3D_STREAM(N0, N1, N2, T, ALG, VPC, NT, NST, MINB)                                      \
    add_stream<N0, N1, N2, T, -1, ALG, VPC, NT, NST, MINB>(                                       \
        out, "stream " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " st" #NST   \
             " minb" #MINB);                                                                      \
    add_stream<N0, N1, N2, T, +1, ALG, VPC, NT, NST, MINB>(                                       \
        out, "stream " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " st" #NST   \
             " minb" #MINB)

// The x pass in place and one bulk store per item (natural layouts, odd n2).
#define FFT3D_STREAM_BST(N0, N1, N2, T, ALG, VPC, NT, NST, MINB)                                  \
    add_stream<N0, N1, N2, T, -1, ALG, VPC, NT, NST, MINB, true>(                                 \
        out, "stream " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " st" #NST   \
             " minb" #MINB " bst");                                                               \
    add_stream<N0, N1, N2, T, +1, ALG, VPC, NT, NST, MINB, true>(                                 \
        out, "stream " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " st" #NST   \
             " minb" #MINB " bst")

void register_stream_kernels(std::vector<KernelEntry> &out)
{
    // complex double (ring must fit 227 KB per CTA, MINB CTAs per SM)
    FFT3D_STREAM(6, 6, 6, double, 0, 8, 288, 3, 1);
    FFT3D_STREAM(6, 6, 6, double, 0, 16, 576, 2, 1);
    FFT3D_STREAM(8, 8, 8, double, 0, 4, 256, 4, 1);
    FFT3D_STREAM(8, 8, 8, double, 0, 2, 128, 3, 2);
    FFT3D_STREAM(8, 8, 8, double, 0, 8, 512, 2, 1);
    FFT3D_STREAM(8, 8, 8, double, 0, 1, 64, 3, 8);   // one volume per item: even tails
    FFT3D_STREAM(8, 8, 8, double, 0, 1, 64, 4, 6);
    FFT3D_STREAM_BST(8, 8, 8, double, 0, 1, 64, 4, 6);
    FFT3D_STREAM(12, 12, 12, double, 0, 2, 288, 2, 1);
    FFT3D_STREAM(12, 12, 12, double, 0, 1, 160, 3, 2);
    FFT3D_STREAM(16, 16, 16, double, 0, 1, 256, 2, 1);
    FFT3D_STREAM(16, 16, 16, double, 0, 1, 256, 3, 1);
    FFT3D_STREAM_BST(16, 16, 16, double, 0, 1, 256, 3, 1);
    FFT3D_STREAM(17, 17, 17, double, 0, 1, 320, 2, 1);
    FFT3D_STREAM(17, 17, 17, double, 1, 1, 320, 2, 1);
    FFT3D_STREAM(17, 17, 17, double, 0, 1, 320, 1, 2);
    FFT3D_STREAM_BST(17, 17, 17, double, 0, 1, 320, 2, 1);
    FFT3D_STREAM_BST(17, 17, 17, double, 2, 1, 320, 2, 1);  // CRT cosine half
    FFT3D_STREAM(8, 8, 16, double, 0, 4, 512, 2, 1);
    FFT3D_STREAM(8, 8, 16, double, 0, 2, 256, 4, 1);
    FFT3D_STREAM(13, 13, 13, double, 0, 1, 192, 3, 2);
    FFT3D_STREAM(13, 13, 13, double, 0, 2, 352, 2, 1);
    FFT3D_STREAM_BST(13, 13, 13, double, 0, 1, 192, 3, 2);
    FFT3D_STREAM_BST(13, 13, 13, double, 0, 2, 352, 2, 1);
    // complex float
    FFT3D_STREAM(6, 6, 6, float, 0, 16, 576, 3, 1);
    FFT3D_STREAM(6, 6, 6, float, 0, 32, 1024, 2, 1);
    FFT3D_STREAM(8, 8, 8, float, 0, 8, 512, 4, 1);
    FFT3D_STREAM(8, 8, 8, float, 0, 16, 1024, 2, 1);
    FFT3D_STREAM(12, 12, 12, float, 0, 2, 288, 4, 1);
    FFT3D_STREAM(12, 12, 12, float, 0, 4, 576, 2, 1);
    FFT3D_STREAM(16, 16, 16, float, 0, 1, 256, 4, 1);
    FFT3D_STREAM_BST(16, 16, 16, float, 0, 1, 256, 4, 1);
    FFT3D_STREAM(16, 16, 16, float, 0, 2, 512, 2, 1);
    FFT3D_STREAM(17, 17, 17, float, 0, 2, 640, 2, 1);
    FFT3D_STREAM(17, 17, 17, float, 1, 2, 640, 2, 1);
    FFT3D_STREAM_BST(17, 17, 17, float, 0, 2, 640, 2, 1);
    FFT3D_STREAM_BST(17, 17, 17, float, 2, 2, 640, 2, 1);
    FFT3D_STREAM(8, 8, 16, float, 0, 4, 512, 4, 1);
    FFT3D_STREAM(8, 8, 16, float, 0, 8, 512, 2, 1);
    FFT3D_STREAM(16, 16, 32, float, 0, 1, 256, 2, 1);
    FFT3D_STREAM(16, 16, 32, float, 0, 1, 256, 3, 1);
    FFT3D_STREAM(13, 13, 13, float, 0, 2, 352, 3, 1);
    FFT3D_STREAM_BST(13, 13, 13, float, 0, 2, 352, 3, 1);
    FFT3D_STREAM(23, 23, 23, float, 0, 1, 288, 2, 1);
}

}  // namespace fft3d

// batch_kernel.cu -- one persistent kernel over a device descriptor list of work
// items of uneven geometry (extents, precision, direction).
//
// The host (batch.cu) cuts every segment into items of VPC volumes of one
// "kind" (a compiled geometry x precision x direction), sorts the items by
// bytes, largest first, and uploads them.  Each CTA of the persistent grid takes
// items with an atomic ticket, so large items start first and small ones fill
// the tail.  Shared memory is two halves: an item that fits a half is loaded
// with cp.async while the previous one is transformed out of the other half;
// larger items (24^3 and 16x16x32 complex double) use all of it.
//
// Two classes of the kernel share this code: class 0 carries every kind (320
// threads, one CTA per SM, 227 KB of shared memory); class 1 carries the
// complex64 kinds only (batch_kinds.h FFT3D_BATCH_KINDS_C64), whose lines need
// fewer registers, as two 256-thread CTAs per SM with half the shared memory
// each, items re-sized to match -- twice the resident warps for an all-complex64
// batch.
//
// 36^3 does not fit one SM.  In this kernel a single CTA transforms it in two
// phases through a per-CTA scratch volume in global memory: x-slabs (z and y
// passes) are written to scratch, then y-slabs are read back for the x pass and
// written to the output.  The scratch of one CTA stays in L2, so HBM traffic is
// still about one read and one write of the volume.  (The plain 36^3 path uses
// the cluster kernel instead, which needs no scratch.)
#include "internal.h"
#include "ptx.cuh"
#include "volume.cuh"
#include "batch_kinds.h"

namespace fft3d {

template <int CLS>
struct BatchClass;
template <>
struct BatchClass<0> {
    static constexpr int NT = 320, MINB = 1;
    // 227 KB is the per-CTA maximum on sm_100a, static shared memory included;
    // keep 128 bytes for this kernel's static variables.
    static constexpr int SMEM = 232448 - 128;
    static constexpr int HALF = (SMEM / 2) / 128 * 128;
};
template <>
struct BatchClass<1> {
    static constexpr int NT = 256, MINB = 2;
    // two CTAs in the SM's 228 KB, each with its 1 KB reserve and static variables
    static constexpr int SMEM = (233472 - 2 * 1024) / 2 - 256;
    static constexpr int HALF = (SMEM / 2) / 128 * 128;
};

// cp.async copy of nel elements into the layout of G (row = g / N2).
template <int NT, class G>
__device__ __forceinline__ void batch_load(cx<typename G::T> *sm, const cx<typename G::T> *gin,
                                           int nel)
{
    for (int g = threadIdx.x; g < nel; g += NT) {
        const int vol = g / G::V;
        const int rem = g - vol * G::V;
        cx<typename G::T> *dst = sm + G::off(vol * G::ROWS + rem / G::N2, rem % G::N2);
        if constexpr (G::EB == 16) cp_async_16(dst, gin + g);
        else cp_async_8(dst, gin + g);
    }
    cp_async_commit();
}

// Line route per extent: 17-point lines take the CRT form of the folded sum.
constexpr int batch_alg(int n) { return n == 17 ? ALG_CRT : ALG_DEFAULT; }

template <int NT, class G, int S>
__device__ __forceinline__ void batch_passes(cx<typename G::T> *sm, int nv,
                                             cx<typename G::T> *gout, typename G::T scale)
{
    const int tid = threadIdx.x;
    for (int r = tid; r < nv * G::ROWS; r += NT) pass_z<G, S, batch_alg(G::N2)>(sm, r);
    __syncthreads();
    for (int l = tid; l < nv * G::N0 * G::N2; l += NT) pass_y<G, S, batch_alg(G::N1)>(sm, l);
    __syncthreads();
    for (int l = tid; l < nv * G::N1 * G::N2; l += NT) pass_x_out<G, S, batch_alg(G::N0)>(sm, l, gout, scale);
}

// ---------------------------------------------------------------- two-phase large cube

// One L^3 volume by one CTA: NS x-slabs of PL planes through the z pass in
// shared memory and the y pass, stored from registers into the CTA's scratch
// volume (L2 only); then the x pass of all L*L lines straight out of scratch
// into registers and on to the output -- no staging copy and no barrier in the
// second phase.  The slabs are double-buffered: the next slab's planes load
// while the current one is transformed.  The CTA barrier at the end of each
// slab orders its scratch stores before the x pass's loads.
template <int NT, int L, typename T, int S, int PL>
__device__ __forceinline__ void big_cube(cx<T> *sm, const cx<T> *gin, cx<T> *gout, cx<T> *scratch, T scale)
{
    constexpr int NS = L / PL;
    static_assert(NS * PL == L, "slabs of PL planes");
    using XG = Geom<PL, L, L, T>;  // x-slab: PL planes of L x L
    const int tid = threadIdx.x;
    batch_load<NT, XG>(sm, gin, PL * L * L);
    for (int s = 0; s < NS; ++s) {
        cx<T> *buf = sm + (s & 1) * XG::PV;
        if (s + 1 < NS) {
            batch_load<NT, XG>(sm + ((s + 1) & 1) * XG::PV, gin + (long long)(s + 1) * PL * L * L, PL * L * L);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        for (int r = tid; r < PL * L; r += NT) pass_z<XG, S, ALG_DEFAULT>(buf, r);
        __syncthreads();
        for (int l = tid; l < PL * L; l += NT) pass_y_store_l2<XG, S>(buf, l, scratch, s * PL);
        __syncthreads();  // the slab's stores before the x pass; its buffer free again
    }
    for (int l = tid; l < L * L; l += NT) pass_x_load_l2<L, L, L, S, T>(scratch, l, gout, 0, scale);
}

// ---------------------------------------------------------------- dispatch

template <int NT, class G, int S>
__device__ __forceinline__ void run_kind_small(unsigned char *region, const BatchItem &it,
                                               const BatchSeg &sg)
{
    using T = typename G::T;
    cx<T> *gout = reinterpret_cast<cx<T> *>(sg.out) + it.v0 * G::V;
    batch_passes<NT, G, S>(reinterpret_cast<cx<T> *>(region), it.nv, gout, (T)sg.scale);
}

template <int NT, int N0, int N1, int N2, typename T, int BIG>
__device__ __forceinline__ void load_kind_any(unsigned char *region, const BatchItem &it,
                                              const BatchSeg &sg)
{
    if constexpr (BIG == 0) {
        using G = Geom<N0, N1, N2, T>;
        const cx<T> *gin = reinterpret_cast<const cx<T> *>(sg.in) + it.v0 * G::V;
        batch_load<NT, G>(reinterpret_cast<cx<T> *>(region), gin, it.nv * G::V);
    }
}

template <int NT, int N0, int N1, int N2, typename T, int S, int BIG>
__device__ __forceinline__ void run_kind_any(unsigned char *region, const BatchItem &it,
                                             const BatchSeg &sg, unsigned char *scratch)
{
    if constexpr (BIG > 0) {
        constexpr long long V = (long long)N0 * N1 * N2;
        const cx<T> *gin = reinterpret_cast<const cx<T> *>(sg.in) + it.v0 * V;
        cx<T> *gout = reinterpret_cast<cx<T> *>(sg.out) + it.v0 * V;
        big_cube<NT, N0, T, S, BIG>(reinterpret_cast<cx<T> *>(region), gin, gout,
                                    reinterpret_cast<cx<T> *>(scratch), (T)sg.scale);
    } else {
        run_kind_small<NT, Geom<N0, N1, N2, T>, S>(region, it, sg);
    }
}

// Issue the loads of an item (two-phase cubes load inside run_item).
template <int CLS>
__device__ __forceinline__ void issue_item_load(unsigned char *region, const BatchItem &it, const BatchSeg &sg)
{
    constexpr int NT = BatchClass<CLS>::NT;
#define FFT3D_BK_LOAD(ID, N0, N1, N2, T, S, VPC, SOLO, BIG) \
    case ID: load_kind_any<NT, N0, N1, N2, T, BIG>(region, it, sg); break;
    if constexpr (CLS == 0) {
        switch (it.kind) {
            FFT3D_BATCH_KINDS(FFT3D_BK_LOAD)
        default: break;
        }
    } else {
        switch (it.kind) {
            FFT3D_BATCH_KINDS_C64(FFT3D_BK_LOAD)
        default: break;
        }
    }
#undef FFT3D_BK_LOAD
}

template <int CLS>
__device__ __forceinline__ void run_item(unsigned char *region, const BatchItem &it, const BatchSeg &sg,
                                         unsigned char *scratch_bytes)
{
    constexpr int NT = BatchClass<CLS>::NT;
#define FFT3D_BK_RUN(ID, N0, N1, N2, T, S, VPC, SOLO, BIG) \
    case ID: run_kind_any<NT, N0, N1, N2, T, S, BIG>(region, it, sg, scratch_bytes); break;
    if constexpr (CLS == 0) {
        switch (it.kind) {
            FFT3D_BATCH_KINDS(FFT3D_BK_RUN)
        default: break;
        }
    } else {
        switch (it.kind) {
            FFT3D_BATCH_KINDS_C64(FFT3D_BK_RUN)
        default: break;
        }
    }
#undef FFT3D_BK_RUN
}

template <int CLS>
__global__ void __launch_bounds__(BatchClass<CLS>::NT, BatchClass<CLS>::MINB)
    k_batch(const BatchItem *__restrict__ items, int nitems, const BatchSeg *__restrict__ segs,
            unsigned int *ticket, unsigned char *scratch, long long scratch_per_cta,
            const unsigned char *__restrict__ solo_of_kind, int *err)
{
    constexpr int HALF = BatchClass<CLS>::HALF;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int s_next;
    (void)err;
    const int tid = threadIdx.x;
    unsigned char *my_scratch = scratch ? scratch + (long long)blockIdx.x * scratch_per_cta : nullptr;

    if (tid == 0) s_next = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    int cur = s_next;
    int off = 0;  // byte offset of the current item's region
    if (cur < nitems) {
        const BatchItem it = items[cur];
        issue_item_load<CLS>(smraw, it, segs[it.seg]);
    }
    while (cur < nitems) {
        const BatchItem it = items[cur];
        const bool solo = solo_of_kind[it.kind] != 0;
        __syncthreads();
        if (tid == 0) s_next = (int)atomicAdd(ticket, 1u);
        __syncthreads();
        const int next = s_next;
        bool pre = false;
        int noff = 0;
        if (!solo && next < nitems) {
            const BatchItem nt = items[next];
            if (!solo_of_kind[nt.kind]) {
                pre = true;
                noff = off == 0 ? HALF : 0;
                issue_item_load<CLS>(smraw + noff, nt, segs[nt.seg]);
            }
        }
        if (pre) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();
        run_item<CLS>(smraw + off, it, segs[it.seg], my_scratch);
        __syncthreads();
        if (!pre && next < nitems) {
            const BatchItem nt = items[next];
            noff = 0;
            issue_item_load<CLS>(smraw, nt, segs[nt.seg]);
        }
        cur = next;
        off = noff;
    }
    cp_async_wait<0>();
}

const void *batch_kernel_func() { return (const void *)&k_batch<0>; }
int batch_kernel_threads() { return BatchClass<0>::NT; }
int batch_kernel_smem() { return BatchClass<0>::SMEM; }
int batch_kernel_half() { return BatchClass<0>::HALF; }
const void *batch_c64_kernel_func() { return (const void *)&k_batch<1>; }
int batch_c64_kernel_threads() { return BatchClass<1>::NT; }
int batch_c64_kernel_smem() { return BatchClass<1>::SMEM; }
int batch_c64_kernel_half() { return BatchClass<1>::HALF; }

}  // namespace fft3d

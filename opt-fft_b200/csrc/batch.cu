// batch.cu -- descriptor-list batches of uneven geometry: host side.
//
// fft3d_b200_batch_create validates the caller's segments, maps each to a
// compiled kind of batch_kernel.cu, cuts it into items, orders the items largest
// first, uploads the descriptor list, sizes the persistent grid from occupancy,
// allocates the per-CTA scratch the two-phase 36^3 kinds need, and captures the
// ticket reset plus the launch in a CUDA graph.  fft3d_b200_batch_execute
// replays the graph on the caller's stream: one launch for the whole batch.
// A batch whose segments are all complex64 runs the complex64 class of the
// kernel (two CTAs per SM; FFT3D_BATCH_KINDS_C64), any other batch class 0
// (FFT3D_B200_BATCH_CLASS=0 in the environment forces class 0).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fft3d_b200.h"
#include "batch_kinds.h"
#include "internal.h"
#include "volume.cuh"

namespace fft3d {

struct KindInfo {
    int id, n0, n1, n2, prec, sign, vpc, solo, big;
    long long vol_elems;
    long long stage_bytes;
};

template <int N0, int N1, int N2, typename T, int VPC, int BIG>
constexpr long long kind_stage_bytes()
{
    if constexpr (BIG > 0) return 2LL * Geom<BIG, N1, N2, T>::PV * Geom<BIG, N1, N2, T>::EB;  // two slab buffers
    else return (long long)VPC * Geom<N0, N1, N2, T>::PV * Geom<N0, N1, N2, T>::EB;
}

static const KindInfo kKinds[] = {
#define FFT3D_BK_INFO(ID, N0, N1, N2, T, S, VPC, SOLO, BIG)                                   \
    {ID, N0, N1, N2, sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64, S, VPC, SOLO, BIG, \
     (long long)N0 * N1 * N2, kind_stage_bytes<N0, N1, N2, T, VPC, BIG>()},
    FFT3D_BATCH_KINDS(FFT3D_BK_INFO)
#undef FFT3D_BK_INFO
};

static const KindInfo kKindsC64[] = {
#define FFT3D_BK_INFO(ID, N0, N1, N2, T, S, VPC, SOLO, BIG)                                   \
    {ID, N0, N1, N2, sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64, S, VPC, SOLO, BIG, \
     (long long)N0 * N1 * N2, kind_stage_bytes<N0, N1, N2, T, VPC, BIG>()},
    FFT3D_BATCH_KINDS_C64(FFT3D_BK_INFO)
#undef FFT3D_BK_INFO
};

static const KindInfo *find_kind(int n0, int n1, int n2, int prec, int sign, int cls = 0)
{
    if (cls == 1) {
        for (const auto &k : kKindsC64)
            if (k.n0 == n0 && k.n1 == n1 && k.n2 == n2 && k.prec == prec && k.sign == sign) return &k;
        return nullptr;
    }
    for (const auto &k : kKinds)
        if (k.n0 == n0 && k.n1 == n1 && k.n2 == n2 && k.prec == prec && k.sign == sign) return &k;
    return nullptr;
}

// The kernel class a batch runs: its function, threads, shared memory, half.
struct BatchKernelClass {
    const void *func;
    int threads, smem, half;
};

static BatchKernelClass kernel_class(int cls)
{
    if (cls == 1)
        return {batch_c64_kernel_func(), batch_c64_kernel_threads(), batch_c64_kernel_smem(),
                batch_c64_kernel_half()};
    return {batch_kernel_func(), batch_kernel_threads(), batch_kernel_smem(), batch_kernel_half()};
}

int batch_kind_of(int n0, int n1, int n2, int precision, int sign, int *vpc, int *big,
                  long long *vol_elems, int *solo)
{
    const KindInfo *k = find_kind(n0, n1, n2, precision, sign);
    if (!k) return -1;
    if (vpc) *vpc = k->vpc;
    if (big) *big = k->big;
    if (vol_elems) *vol_elems = k->vol_elems;
    if (solo) *solo = (k->solo || k->big || k->stage_bytes > batch_kernel_half()) ? 1 : 0;
    return k->id;
}

}  // namespace fft3d

using namespace fft3d;

struct fft3d_b200_batch {
    int device = 0;
    std::vector<fft3d_b200_segment> segs;
    BatchItem *d_items = nullptr;
    BatchSeg *d_segs = nullptr;
    unsigned int *d_ticket = nullptr;
    unsigned char *d_solo = nullptr;
    unsigned char *d_scratch = nullptr;
    int *d_err = nullptr;
    long long scratch_per_cta = 0;
    int nitems = 0;
    int grid = 0;
    int cls = 0;  // kernel class (batch_kernel.cu)
    bool use_graph = false;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string describe;
    // per-segment strategy: one tuned plan per segment, parallel graph branches
    bool segments = false;
    std::vector<fft3d_b200_plan *> plans;  // one per segment (NULL for empty ones)
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    cudaGraph_t sgraph = nullptr;
    cudaGraphExec_t sexec = nullptr;
};

static void batch_free(fft3d_b200_batch *b)
{
    if (b->sexec) cudaGraphExecDestroy(b->sexec);
    if (b->sgraph) cudaGraphDestroy(b->sgraph);
    for (auto *p : b->plans)
        if (p) fft3d_b200_plan_destroy(p);
    for (auto st : b->branch) cudaStreamDestroy(st);
    for (auto ev : b->join) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap) cudaStreamDestroy(b->cap);
    cudaFree(b->d_items);
    cudaFree(b->d_segs);
    cudaFree(b->d_ticket);
    cudaFree(b->d_solo);
    cudaFree(b->d_scratch);
    cudaFree(b->d_err);
    delete b;
}

static cudaError_t batch_enqueue(fft3d_b200_batch *b, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(b->d_ticket, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    if (b->nitems == 0) return cudaSuccess;
    const BatchItem *items = b->d_items;
    int nitems = b->nitems;
    const BatchSeg *segs = b->d_segs;
    unsigned int *ticket = b->d_ticket;
    unsigned char *scratch = b->d_scratch;
    long long spc = b->scratch_per_cta;
    const unsigned char *solo = b->d_solo;
    int *err = b->d_err;
    void *args[] = {(void *)&items, (void *)&nitems, (void *)&segs,   (void *)&ticket,
                    (void *)&scratch, (void *)&spc,  (void *)&solo, (void *)&err};
    const BatchKernelClass kc = kernel_class(b->cls);
    return cudaLaunchKernel(kc.func, dim3(b->grid), dim3(kc.threads), args, (size_t)kc.smem, s);
}

// Per-segment strategy on stream s: fork to the branch streams, one tuned plan
// per segment (segments spread round-robin over the branches), join back on s.
static cudaError_t segments_enqueue(fft3d_b200_batch *b, cudaStream_t s)
{
    cudaError_t e = cudaEventRecord(b->fork, s);
    for (size_t k = 0; k < b->branch.size() && e == cudaSuccess; ++k)
        e = cudaStreamWaitEvent(b->branch[k], b->fork, 0);
    for (size_t i = 0; i < b->plans.size() && e == cudaSuccess; ++i) {
        if (!b->plans[i]) continue;
        const int st = fft3d_b200_execute(b->plans[i], b->segs[i].in, b->segs[i].out,
                                          b->branch[i % b->branch.size()]);
        if (st != FFT3D_B200_OK) e = cudaErrorLaunchFailure;
    }
    for (size_t k = 0; k < b->branch.size() && e == cudaSuccess; ++k) {
        e = cudaEventRecord(b->join[k], b->branch[k]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->join[k], 0);
    }
    return e;
}

// Mean time of `reps` runs of a strategy on s (after two warm-up runs): its
// graph when the batch replays graphs, its direct launches otherwise.
static float strategy_time_ms(fft3d_b200_batch *b, bool seg, cudaStream_t s, int reps)
{
    auto run = [&]() {
        if (b->use_graph) cudaGraphLaunch(seg ? b->sexec : b->exec, s);
        else if (seg) segments_enqueue(b, s);
        else batch_enqueue(b, s);
    };
    cudaEvent_t a, z;
    if (cudaEventCreate(&a) != cudaSuccess) return 1e30f;
    if (cudaEventCreate(&z) != cudaSuccess) {
        cudaEventDestroy(a);
        return 1e30f;
    }
    float best = 1e30f;
    for (int w = 0; w < 2; ++w) run();
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a, s);
        for (int i = 0; i < reps; ++i) run();
        cudaEventRecord(z, s);
        cudaEventSynchronize(z);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, z);
        best = std::min(best, ms / (float)reps);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    cudaGetLastError();
    return best;
}

extern "C" int fft3d_b200_batch_create(const fft3d_b200_segment *segs, int nseg, unsigned flags,
                                       int device, fft3d_b200_batch **out)
{
    if (!out) return FFT3D_B200_ERR_INVALID;
    *out = nullptr;
    if (nseg < 0 || (nseg > 0 && !segs)) return FFT3D_B200_ERR_INVALID;
    std::vector<BatchItem> items;
    std::vector<BatchSeg> dsegs;
    std::vector<unsigned char> solo(BATCH_NKINDS, 0);
    long long scratch_need = 0;
    bool persistent_ok = true;  // every segment has a kind of the persistent kernel
    // every segment complex64: the complex64 class of the kernel
    int cls = 1;
    for (int i = 0; i < nseg; ++i)
        if (segs[i].precision != FFT3D_B200_C64) cls = 0;
    if (const char *e = getenv("FFT3D_B200_BATCH_CLASS"))
        if (e[0] == '0') cls = 0;
    const BatchKernelClass kc = kernel_class(cls);
    for (const KindInfo &ki : kKinds) {
        const KindInfo *k = cls == 1 ? find_kind(ki.n0, ki.n1, ki.n2, ki.prec, ki.sign, 1) : &ki;
        if (!k) continue;
        if (k->stage_bytes > kc.smem) return FFT3D_B200_ERR_UNSUPPORTED;
        solo[k->id] = (unsigned char)(k->solo || k->big || k->stage_bytes > kc.half);
    }
    for (int i = 0; i < nseg; ++i) {
        const fft3d_b200_segment &s = segs[i];
        if (s.n0 < 1 || s.n1 < 1 || s.n2 < 1 || s.batch < 0) return FFT3D_B200_ERR_INVALID;
        if (s.direction != FFT3D_B200_FORWARD && s.direction != FFT3D_B200_BACKWARD)
            return FFT3D_B200_ERR_INVALID;
        if (s.precision != FFT3D_B200_C128 && s.precision != FFT3D_B200_C64)
            return FFT3D_B200_ERR_INVALID;
        const size_t eb = (size_t)element_bytes(s.precision);
        const size_t bytes = (size_t)s.batch * (size_t)s.n0 * (size_t)s.n1 * (size_t)s.n2 * eb;
        if (s.batch > 0) {
            if (!s.in || !s.out) return FFT3D_B200_ERR_INVALID;
            if (((uintptr_t)s.in % eb) || ((uintptr_t)s.out % eb)) return FFT3D_B200_ERR_ALIGN;
            const char *a = (const char *)s.in, *o = (const char *)s.out;
            if (a < o + bytes && o < a + bytes) return FFT3D_B200_ERR_OVERLAP;
        }
        const KindInfo *k = find_kind(s.n0, s.n1, s.n2, s.precision, s.direction, cls);
        if (!k) {
            // no persistent-kernel kind for this extent: the batch runs as one
            // tuned plan per segment (if the extent has a plan at all)
            if ((flags & FFT3D_B200_BATCH_PERSISTENT) || !fft3d_b200_supports(s.n0, s.n1, s.n2, s.precision))
                return FFT3D_B200_ERR_UNSUPPORTED;
            persistent_ok = false;
            continue;
        }
        BatchSeg d;
        d.in = s.in;
        d.out = s.out;
        d.scale = s.direction == FFT3D_B200_BACKWARD ? 1.0 / (double)k->vol_elems : 1.0;
        d.nvol = s.batch;
        d.kind = k->id;
        d.pad = 0;
        dsegs.push_back(d);
        for (long long v0 = 0; v0 < s.batch; v0 += k->vpc) {
            BatchItem it;
            it.kind = k->id;
            it.seg = i;
            it.v0 = v0;
            it.nv = (int)std::min<long long>(k->vpc, s.batch - v0);
            it.pad = 0;
            items.push_back(it);
        }
        if (k->big && s.batch > 0) scratch_need = std::max(scratch_need, (long long)(k->vol_elems * eb));
    }
    if (items.size() > 0x7fffffff) return FFT3D_B200_ERR_INVALID;
    // largest first: big items start early, small ones fill the tail
    std::stable_sort(items.begin(), items.end(), [&](const BatchItem &a, const BatchItem &b) {
        const KindInfo &ka = kKinds[a.kind], &kb = kKinds[b.kind];  // extents and precision
        const long long ca = (long long)a.nv * ka.vol_elems * (ka.prec == FFT3D_B200_C128 ? 16 : 8);
        const long long cb = (long long)b.nv * kb.vol_elems * (kb.prec == FFT3D_B200_C128 ? 16 : 8);
        return ca > cb;
    });

    int prev = -1;
    cudaGetDevice(&prev);
    if (device < 0) device = prev < 0 ? 0 : prev;
    if (cudaSetDevice(device) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    int st = ensure_device_tables(device);
    if (st) {
        if (prev >= 0) cudaSetDevice(prev);
        return st;
    }
    fft3d_b200_batch *b = new fft3d_b200_batch();
    b->device = device;
    b->segs.assign(segs, segs + nseg);
    b->nitems = (int)items.size();
    b->cls = cls;
    auto fail = [&](int code) {
        const cudaError_t ce = cudaGetLastError();
        if (getenv("FFT3D_B200_DEBUG"))
            fprintf(stderr, "fft3d_b200_batch_create: status %d (%s)\n", code, cudaGetErrorString(ce));
        batch_free(b);
        if (prev >= 0) cudaSetDevice(prev);
        return code;
    };
    if (!persistent_ok) {
        items.clear();
        dsegs.clear();
        scratch_need = 0;
        b->nitems = 0;
    }
    if (persistent_ok &&
        cudaFuncSetAttribute(kc.func, cudaFuncAttributeMaxDynamicSharedMemorySize, kc.smem) != cudaSuccess)
        return fail(FFT3D_B200_ERR_CUDA);
    int occ = 0, sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (persistent_ok &&
        (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kc.func, kc.threads, (size_t)kc.smem) != cudaSuccess ||
         occ < 1))
        return fail(FFT3D_B200_ERR_UNSUPPORTED);
    b->grid = std::max(1, std::min(occ * sms, std::max(1, b->nitems)));
    if (cudaMalloc(&b->d_items, std::max<size_t>(1, items.size()) * sizeof(BatchItem)) != cudaSuccess ||
        cudaMalloc(&b->d_segs, std::max<size_t>(1, dsegs.size()) * sizeof(BatchSeg)) != cudaSuccess ||
        cudaMalloc(&b->d_ticket, sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc(&b->d_solo, BATCH_NKINDS) != cudaSuccess ||
        cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess)
        return fail(FFT3D_B200_ERR_NOMEM);
    if (!items.empty() &&
        cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(FFT3D_B200_ERR_CUDA);
    if (!dsegs.empty() &&
        cudaMemcpy(b->d_segs, dsegs.data(), dsegs.size() * sizeof(BatchSeg), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(FFT3D_B200_ERR_CUDA);
    if (cudaMemcpy(b->d_solo, solo.data(), BATCH_NKINDS, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(b->d_err, 0, sizeof(int)) != cudaSuccess)
        return fail(FFT3D_B200_ERR_CUDA);
    if (scratch_need > 0) {
        b->scratch_per_cta = (scratch_need + 255) / 256 * 256;
        if (cudaMalloc(&b->d_scratch, (size_t)b->scratch_per_cta * b->grid) != cudaSuccess)
            return fail(FFT3D_B200_ERR_NOMEM);
    }
    b->use_graph = !(flags & FFT3D_B200_FLAG_NO_GRAPH);
    if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess)
        return fail(FFT3D_B200_ERR_CUDA);
    if (b->use_graph && persistent_ok) {
        if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return fail(FFT3D_B200_ERR_CUDA);
        cudaError_t le = batch_enqueue(b, b->cap);
        cudaError_t ee = cudaStreamEndCapture(b->cap, &b->graph);
        if (le != cudaSuccess || ee != cudaSuccess) return fail(FFT3D_B200_ERR_CUDA);
        if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) return fail(FFT3D_B200_ERR_CUDA);
    }
    // The per-segment strategy: built unless the persistent kernel is pinned
    // (or timing is off), then timed against the persistent launch.
    const bool want_seg = !persistent_ok || (flags & FFT3D_B200_BATCH_SEGMENTS) ||
                          !(flags & (FFT3D_B200_BATCH_PERSISTENT | FFT3D_B200_FLAG_NO_TUNE));
    float t_persist = -1.f, t_seg = -1.f;
    bool plans_ok = want_seg && nseg > 0;
    if (plans_ok) {
        b->plans.assign(nseg, nullptr);
        for (int i = 0; i < nseg && plans_ok; ++i) {
            if (segs[i].batch <= 0) continue;
            fft3d_b200_desc d;
            d.n0 = segs[i].n0;
            d.n1 = segs[i].n1;
            d.n2 = segs[i].n2;
            d.batch = segs[i].batch;
            d.direction = segs[i].direction;
            d.precision = segs[i].precision;
            d.flags = 0;
            d.device = device;
            plans_ok = fft3d_b200_plan_create(&d, &b->plans[i]) == FFT3D_B200_OK;
        }
        if (!plans_ok) {  // a geometry without a plan: the persistent kernel only
            if ((flags & FFT3D_B200_BATCH_SEGMENTS) || !persistent_ok) return fail(FFT3D_B200_ERR_UNSUPPORTED);
            for (auto *pl : b->plans)
                if (pl) fft3d_b200_plan_destroy(pl);
            b->plans.clear();
            cudaGetLastError();
        }
    }
    if (plans_ok) {
        const int nbr = std::max(1, std::min(nseg, 16));
        b->branch.assign(nbr, nullptr);
        b->join.assign(nbr, nullptr);
        for (int k = 0; k < nbr; ++k)
            if (cudaStreamCreateWithFlags(&b->branch[k], cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) != cudaSuccess)
                return fail(FFT3D_B200_ERR_CUDA);
        if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
            return fail(FFT3D_B200_ERR_CUDA);
        if (b->use_graph) {
            if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
                return fail(FFT3D_B200_ERR_CUDA);
            cudaError_t le = segments_enqueue(b, b->cap);
            cudaError_t ee = cudaStreamEndCapture(b->cap, &b->sgraph);
            if (le != cudaSuccess || ee != cudaSuccess) return fail(FFT3D_B200_ERR_CUDA);
            if (cudaGraphInstantiate(&b->sexec, b->sgraph, 0) != cudaSuccess) return fail(FFT3D_B200_ERR_CUDA);
        }
        b->segments = true;
        if (!(flags & FFT3D_B200_BATCH_SEGMENTS) && persistent_ok) {
            // the race, on the batch's own buffers
            t_seg = strategy_time_ms(b, true, b->cap, 5);
            t_persist = strategy_time_ms(b, false, b->cap, 5);
            b->segments = t_seg < t_persist;
        }
        if (cudaStreamSynchronize(b->cap) != cudaSuccess) return fail(FFT3D_B200_ERR_CUDA);
    }
    char buf[400];
    if (b->segments) {
        snprintf(buf, sizeof buf,
                 "batch: %d segments, one tuned plan per segment on %zu parallel branches, %s",
                 nseg, b->branch.size(), b->use_graph ? "CUDA graph" : "direct launches");
    } else {
        snprintf(buf, sizeof buf, "batch: %d segments, %d items, grid %d x %d threads (%s kernel), %s%s",
                 nseg, b->nitems, b->grid, kernel_class(b->cls).threads,
                 b->cls == 1 ? "complex64" : "all-kinds", b->use_graph ? "CUDA graph" : "direct launch",
                 b->d_scratch ? ", two-phase scratch" : "");
    }
    b->describe = buf;
    if (t_seg >= 0.f) {
        snprintf(buf, sizeof buf, " (timed: per-segment %.1f us, persistent %.1f us)", t_seg * 1e3f,
                 t_persist * 1e3f);
        b->describe += buf;
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    *out = b;
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_batch_execute(fft3d_b200_batch *b, void *stream)
{
    if (!b) return FFT3D_B200_ERR_INVALID;
    cudaError_t e;
    if (b->segments) {
        if (b->use_graph) e = cudaGraphLaunch(b->sexec, (cudaStream_t)stream);
        else e = segments_enqueue(b, (cudaStream_t)stream);
    } else if (b->use_graph) {
        e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    } else {
        e = batch_enqueue(b, (cudaStream_t)stream);
    }
    return e == cudaSuccess ? FFT3D_B200_OK : FFT3D_B200_ERR_CUDA;
}

extern "C" void fft3d_b200_batch_destroy(fft3d_b200_batch *b)
{
    if (!b) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    batch_free(b);
    if (prev >= 0) cudaSetDevice(prev);
}

extern "C" const char *fft3d_b200_batch_describe(const fft3d_b200_batch *b)
{
    return b ? b->describe.c_str() : "";
}

// batch_noalloc.cu -- the descriptor-list batch with no device allocation at all.
//
// Who needs this: code that may not call cudaMalloc.  A host application that
// has handed all device memory to its own pool allocator (a framework's caching
// allocator, a serving engine that reserves HBM up front) cannot let a library
// allocate behind its back; a latency-critical loop cannot afford cudaMalloc /
// cudaFree, which may synchronise the device and can fail under memory pressure;
// some plugin hosts simply forbid it.  fft3d_b200_batch_create allocates the
// device descriptor list, the work ticket and the error word, so those callers
// cannot use it.
//
// fft3d_b200_batch_execute_noalloc runs the same persistent batch kernel
// (batch_kernel.cu) with all of that scratch in one file-scope static
// __device__ array (g_noalloc below, NOALLOC_BYTES, about 540 KB) that every GPU
// loading this library keeps until the process exits.  Limits: at most
// NOALLOC_MAX_SEGS segments and NOALLOC_MAX_ITEMS work items per call, and no
// 36^3 segments (their two-phase route needs per-CTA scratch far larger than
// this array); beyond them the call returns FFT3D_B200_ERR_BUDGET and enqueues
// nothing.
//
// Host code may not use g_noalloc's name as an address: on the host it is only a
// stand-in for the device symbol.  The first call on each device (with that
// device current) looks the address up with cudaGetSymbolAddress and caches it;
// make that first call before any stream capture.  Every call reuses the same
// array: it copies the call's descriptors in and resets the ticket to zero on
// the caller's stream.  Host threads that call on the same stream are serialised
// from the first copy to the launch, so each launch reads its own descriptors;
// calls that overlap on the GPU (different streams) race on the array and must
// be ordered by the caller.  The descriptors are copied from the caller's stack,
// so a stream that is being captured is refused (FFT3D_B200_ERR_INVALID): a
// replayed copy would read stack memory that no longer holds them.
// fft3d_b200_noalloc_check synchronises a stream and reports the launch's
// status and the array's device error word.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fft3d_b200.h"
#include "batch_kinds.h"
#include "internal.h"

namespace fft3d {

constexpr int NOALLOC_MAX_ITEMS = 16384;
constexpr int NOALLOC_MAX_SEGS = 256;
constexpr size_t NOALLOC_ITEMS_OFF = 0;
constexpr size_t NOALLOC_SEGS_OFF = NOALLOC_ITEMS_OFF + sizeof(BatchItem) * NOALLOC_MAX_ITEMS;
constexpr size_t NOALLOC_TICKET_OFF = (NOALLOC_SEGS_OFF + sizeof(BatchSeg) * NOALLOC_MAX_SEGS + 255) / 256 * 256;
constexpr size_t NOALLOC_ERR_OFF = NOALLOC_TICKET_OFF + 256;
constexpr size_t NOALLOC_SOLO_OFF = NOALLOC_ERR_OFF + 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_SOLO_OFF + 256;

static __device__ __align__(256) unsigned char g_noalloc[NOALLOC_BYTES];

struct NoAllocDevice {
    unsigned char *base = nullptr;  // device address of g_noalloc on this device
    int grid = 0;
};

static std::mutex g_noalloc_mu;        // first-time set-up
static std::mutex g_noalloc_enqueue_mu;  // descriptor copies through the launch
static NoAllocDevice g_noalloc_dev[64];

// Once per device, with the device current: the symbol's device address, the
// kernel's shared-memory attribute, the grid size, the twiddle tables.
static int noalloc_setup(int device, NoAllocDevice *out)
{
    if (device < 0 || device >= 64) return FFT3D_B200_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice &d = g_noalloc_dev[device];
    if (!d.base) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc) != cudaSuccess || !p) {
            cudaGetLastError();
            return FFT3D_B200_ERR_CUDA;
        }
        const int st = ensure_device_tables(device);
        if (st) return st;
        if (cudaFuncSetAttribute(batch_kernel_func(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 batch_kernel_smem()) != cudaSuccess) {
            cudaGetLastError();
            return FFT3D_B200_ERR_CUDA;
        }
        int occ = 0, sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel_func(),
                                                          batch_kernel_threads(),
                                                          (size_t)batch_kernel_smem()) != cudaSuccess ||
            occ < 1) {
            cudaGetLastError();
            return FFT3D_B200_ERR_UNSUPPORTED;
        }
        d.grid = occ * sms;
        d.base = (unsigned char *)p;
    }
    *out = d;
    return FFT3D_B200_OK;
}

}  // namespace fft3d

using namespace fft3d;

extern "C" int fft3d_b200_batch_execute_noalloc(const fft3d_b200_segment *segs, int nseg,
                                                void *stream)
{
    if (nseg < 0 || (nseg > 0 && !segs)) return FFT3D_B200_ERR_INVALID;
    if (nseg > NOALLOC_MAX_SEGS) return FFT3D_B200_ERR_BUDGET;
    // Validate and describe every segment (stack memory only).
    BatchSeg dsegs[NOALLOC_MAX_SEGS];
    int vpc[NOALLOC_MAX_SEGS];
    int order[NOALLOC_MAX_SEGS];
    long long cost[NOALLOC_MAX_SEGS];
    long long nitems = 0;
    for (int i = 0; i < nseg; ++i) {
        const fft3d_b200_segment &s = segs[i];
        if (s.n0 < 1 || s.n1 < 1 || s.n2 < 1 || s.batch < 0) return FFT3D_B200_ERR_INVALID;
        if ((s.direction != FFT3D_B200_FORWARD && s.direction != FFT3D_B200_BACKWARD) ||
            (s.precision != FFT3D_B200_C128 && s.precision != FFT3D_B200_C64))
            return FFT3D_B200_ERR_INVALID;
        int big = 0;
        long long ve = 0;
        const int kind = batch_kind_of(s.n0, s.n1, s.n2, s.precision, s.direction, &vpc[i], &big, &ve,
                                       nullptr);
        if (kind < 0) return FFT3D_B200_ERR_UNSUPPORTED;
        if (big && s.batch > 0) return FFT3D_B200_ERR_BUDGET;  // needs per-CTA scratch
        // before any product with the batch: a segment alone above the item
        // limit is refused, so the sums and byte counts below cannot overflow
        if (s.batch > (long long)NOALLOC_MAX_ITEMS * vpc[i]) return FFT3D_B200_ERR_BUDGET;
        const size_t eb = (size_t)element_bytes(s.precision);
        const size_t bytes = (size_t)s.batch * (size_t)ve * eb;
        if (s.batch > 0) {
            if (!s.in || !s.out) return FFT3D_B200_ERR_INVALID;
            if (((uintptr_t)s.in % eb) || ((uintptr_t)s.out % eb)) return FFT3D_B200_ERR_ALIGN;
            const char *a = (const char *)s.in, *o = (const char *)s.out;
            if (a < o + bytes && o < a + bytes) return FFT3D_B200_ERR_OVERLAP;
        }
        dsegs[i].in = s.in;
        dsegs[i].out = s.out;
        dsegs[i].scale = s.direction == FFT3D_B200_BACKWARD ? 1.0 / (double)ve : 1.0;
        dsegs[i].nvol = s.batch;
        dsegs[i].kind = kind;
        dsegs[i].pad = 0;
        nitems += (s.batch + vpc[i] - 1) / vpc[i];
        cost[i] = (long long)vpc[i] * ve * (long long)eb;  // bytes of a full item
        order[i] = i;
    }
    if (nitems > NOALLOC_MAX_ITEMS) return FFT3D_B200_ERR_BUDGET;
    // largest items first, segment by segment (insertion sort, stable)
    for (int i = 1; i < nseg; ++i) {
        const int o = order[i];
        int j = i - 1;
        while (j >= 0 && cost[order[j]] < cost[o]) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = o;
    }

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        return FFT3D_B200_ERR_INVALID;
    }
    if (cap != cudaStreamCaptureStatusNone) return FFT3D_B200_ERR_INVALID;
    NoAllocDevice nd;
    int st = noalloc_setup(device, &nd);
    if (st) return st;
    std::lock_guard<std::mutex> enqueue_lock(g_noalloc_enqueue_mu);
    BatchItem *d_items = (BatchItem *)(nd.base + NOALLOC_ITEMS_OFF);
    BatchSeg *d_segs = (BatchSeg *)(nd.base + NOALLOC_SEGS_OFF);
    unsigned int *d_ticket = (unsigned int *)(nd.base + NOALLOC_TICKET_OFF);
    int *d_err = (int *)(nd.base + NOALLOC_ERR_OFF);
    unsigned char *d_solo = nd.base + NOALLOC_SOLO_OFF;

    // Descriptors go through a small stack buffer; copies from pageable memory
    // return once the source has been read, so the buffer can be refilled.
    BatchItem chunk[256];
    int filled = 0;
    long long written = 0;
    for (int oi = 0; oi < nseg; ++oi) {
        const int i = order[oi];
        for (long long v0 = 0; v0 < segs[i].batch; v0 += vpc[i]) {
            BatchItem &it = chunk[filled++];
            it.kind = dsegs[i].kind;
            it.seg = i;
            it.v0 = v0;
            it.nv = (int)((segs[i].batch - v0) < vpc[i] ? (segs[i].batch - v0) : vpc[i]);
            it.pad = 0;
            if (filled == 256) {
                if (cudaMemcpyAsync(d_items + written, chunk, sizeof chunk, cudaMemcpyHostToDevice, s) !=
                    cudaSuccess)
                    return FFT3D_B200_ERR_CUDA;
                written += filled;
                filled = 0;
            }
        }
    }
    if (filled && cudaMemcpyAsync(d_items + written, chunk, filled * sizeof(BatchItem),
                                  cudaMemcpyHostToDevice, s) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    unsigned char solo[BATCH_NKINDS];
    for (int k = 0; k < BATCH_NKINDS; ++k) solo[k] = 0;
    for (int i = 0; i < nseg; ++i) {
        int so = 0;
        batch_kind_of(segs[i].n0, segs[i].n1, segs[i].n2, segs[i].precision, segs[i].direction,
                      nullptr, nullptr, nullptr, &so);
        solo[dsegs[i].kind] = (unsigned char)so;
    }
    if ((nseg > 0 &&
         cudaMemcpyAsync(d_segs, dsegs, nseg * sizeof(BatchSeg), cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        cudaMemcpyAsync(d_solo, solo, sizeof solo, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(d_ticket, 0, sizeof(unsigned int), s) != cudaSuccess ||
        cudaMemsetAsync(d_err, 0, sizeof(int), s) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    if (nitems == 0) return FFT3D_B200_OK;

    const BatchItem *items = d_items;
    int n = (int)nitems;
    const BatchSeg *dsp = d_segs;
    unsigned char *scratch = nullptr;
    long long spc = 0;
    const unsigned char *solo_p = d_solo;
    int grid = nd.grid < n ? nd.grid : n;
    void *args[] = {(void *)&items, (void *)&n,       (void *)&dsp,    (void *)&d_ticket,
                    (void *)&scratch, (void *)&spc, (void *)&solo_p, (void *)&d_err};
    if (cudaLaunchKernel(batch_kernel_func(), dim3(grid), dim3(batch_kernel_threads()), args,
                         (size_t)batch_kernel_smem(), s) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_noalloc_check(void *stream)
{
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    NoAllocDevice nd;
    const int st = noalloc_setup(device, &nd);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    int v = 0;
    const int *d_err = (const int *)(nd.base + NOALLOC_ERR_OFF);
    if (cudaMemcpyAsync(&v, d_err, sizeof v, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    return v == 0 ? FFT3D_B200_OK : FFT3D_B200_ERR_TIMEOUT;
}

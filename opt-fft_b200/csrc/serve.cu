// serve.cu -- continuous-batching request server over the persistent batch kernel.
//
// Requests (fft3d_b200_segment: geometry, direction, precision, volumes, device
// in/out pointers) are submitted from any host thread and queue FIFO.  A server
// thread admits them against an HBM budget (the in+out bytes of all requests
// admitted and not yet finished may not exceed it), coalesces every admitted
// request into one descriptor list, and launches the persistent batch kernel
// (batch_kernel.cu) on one of `max_inflight` streams.  Requests that arrive
// while batches are running are admitted as soon as a stream slot and budget are
// free, so their work overlaps the running batches on the device.  Completion is
// detected with one event per launch; latency is completion minus submission,
// on the host clock, and p50 / p99 are reported with throughput.
//
// Each stream slot owns device-resident descriptor buffers, a ticket, and the
// per-CTA scratch of the two-phase 36^3 route, allocated once at creation; the
// hot loop allocates nothing on the device.
//
// A request whose extent is not one of the persistent kernel's kinds (any
// other compiled extent) is launched on its own with its tuned kernel, on the
// same stream as the batch (a scratch-ring kernel with the slot's workspace).
//
// Baseline mode (FFT3D_B200_SERVE_PLAIN): every request is launched on its own,
// as soon as it is admitted, with the tuned per-geometry kernel of its kind --
// one launch per request.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/fft3d_b200.h"
#include "batch_kinds.h"
#include "internal.h"

namespace fft3d {

static double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

constexpr int SERVE_MAX_ITEMS = 65536;
constexpr int SERVE_MAX_SEGS = 8192;

struct ServeReq {
    fft3d_b200_segment seg;
    unsigned long long ticket;
    double t_submit;
    size_t bytes;
    int kind, vpc, big;
    long long vol_elems;
    long long nitems;
};

struct ServeSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    BatchItem *d_items = nullptr;
    BatchSeg *d_segs = nullptr;
    unsigned int *d_ticket = nullptr;
    unsigned char *d_solo = nullptr;
    unsigned char *d_scratch = nullptr;
    int *d_err = nullptr;
    BatchItem *h_items = nullptr;  // pinned staging
    BatchSeg *h_segs = nullptr;
    void *d_work = nullptr;        // workspace of scratch-ring kernels, grown on demand
    size_t work_bytes = 0;
    bool busy = false;
    std::vector<ServeReq> reqs;
    size_t bytes = 0;
};

}  // namespace fft3d

using namespace fft3d;

struct fft3d_b200_server {
    int device = 0;
    unsigned flags = 0;
    size_t budget = 0;
    size_t used = 0;
    size_t peak_used = 0;
    int grid = 0;
    long long scratch_per_cta = 0;
    std::vector<ServeSlot> slots;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<ServeReq> pending;
    std::atomic<long long> npending{0};  // pending.size(), readable without the lock
    std::deque<unsigned long long> completed;
    unsigned long long next_ticket = 1;
    unsigned long long submitted = 0, finished = 0;
    std::atomic<bool> stop{false};
    std::thread thr;
    int status = FFT3D_B200_OK;
    // statistics
    std::vector<double> lat;
    std::vector<unsigned long long> lat_ticket;  // ticket of each lat entry
    long long volumes = 0, batches = 0, batched_requests = 0;
    double t_first = 0, t_last = 0;
};

// Plain mode, and extents without a persistent-kernel kind: the per-geometry
// kernel the autotuner picks for this request's volume count (memoised by batch
// size class) among the kernels that need no workspace -- they run on many
// slots at once -- or, for an extent that has none (45^3, 64^3, complex128
// 30^3), among its scratch-ring kernels; and its persistent-grid limit.
static const KernelEntry *plain_entry(fft3d_b200_server *s, const ServeReq &r, int *grid)
{
    const KernelEntry *e = tuned_entry(s->device, r.seg.n0, r.seg.n1, r.seg.n2, r.seg.precision,
                                       r.seg.direction, r.seg.batch);
    if (!e)
        e = tuned_entry(s->device, r.seg.n0, r.seg.n1, r.seg.n2, r.seg.precision, r.seg.direction,
                        r.seg.batch, true);
    if (!e) return nullptr;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    *grid = entry_occupancy(*e, s->device) * sms;
    return e;
}

// One request by its own tuned kernel on the slot's stream; a scratch-ring
// kernel gets the slot's workspace (grown, and its control block zeroed, on
// first need; every launch leaves the block zero again).  The workspace is
// allocated and freed in stream order on the slot's stream, so growing it
// synchronises neither the device nor the other slots.
static int launch_request(fft3d_b200_server *s, ServeSlot &slot, const ServeReq &r)
{
    int grid = 0;
    const KernelEntry *e = plain_entry(s, r, &grid);
    if (!e) return FFT3D_B200_ERR_UNSUPPORTED;
    const size_t wb = entry_workspace_bytes(*e, grid);
    if (wb > slot.work_bytes) {
        if (slot.d_work && cudaFreeAsync(slot.d_work, slot.stream) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
        slot.d_work = nullptr;
        slot.work_bytes = 0;
        if (cudaMallocAsync(&slot.d_work, wb, slot.stream) != cudaSuccess) return FFT3D_B200_ERR_NOMEM;
        if (cudaMemsetAsync(slot.d_work, 0, TWOPASS_CTL_BYTES, slot.stream) != cudaSuccess)
            return FFT3D_B200_ERR_CUDA;
        slot.work_bytes = wb;
    }
    const double scale = r.seg.direction == FFT3D_B200_BACKWARD ? 1.0 / (double)r.vol_elems : 1.0;
    if (launch_entry(*e, r.seg.in, r.seg.out, r.seg.batch, scale, slot.stream, grid, slot.d_err,
                     wb ? slot.d_work : nullptr) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    return FFT3D_B200_OK;
}

// Launch every request of `slot` as one persistent batch (or, in plain mode,
// one launch per request) and record the slot's completion event.
static int launch_slot(fft3d_b200_server *s, ServeSlot &slot)
{
    cudaStream_t st = slot.stream;
    if (s->flags & FFT3D_B200_SERVE_PLAIN) {
        for (const ServeReq &r : slot.reqs)
            if (const int e = launch_request(s, slot, r)) return e;
    } else {
        // requests whose extent is not a kind of the persistent kernel: one
        // tuned launch each on the slot's stream, beside the batch launch
        for (const ServeReq &r : slot.reqs)
            if (r.kind < 0)
                if (const int e = launch_request(s, slot, r)) return e;
        // descriptors: requests are segments; items largest first
        int nseg = (int)slot.reqs.size();
        std::vector<int> order(nseg);
        for (int i = 0; i < nseg; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            const ServeReq &x = slot.reqs[a], &y = slot.reqs[b];
            const long long cx = x.vpc * x.vol_elems * (x.seg.precision == FFT3D_B200_C128 ? 16 : 8);
            const long long cy = y.vpc * y.vol_elems * (y.seg.precision == FFT3D_B200_C128 ? 16 : 8);
            return cx > cy;
        });
        int n = 0;
        unsigned char solo[BATCH_NKINDS];
        std::memset(solo, 0, sizeof solo);
        for (int i = 0; i < nseg; ++i) {
            const ServeReq &r = slot.reqs[i];
            BatchSeg &d = slot.h_segs[i];
            d.in = r.seg.in;
            d.out = r.seg.out;
            d.scale = r.seg.direction == FFT3D_B200_BACKWARD ? 1.0 / (double)r.vol_elems : 1.0;
            d.nvol = r.seg.batch;
            d.kind = r.kind < 0 ? 0 : r.kind;
            d.pad = 0;
            if (r.kind < 0) {
                d.nvol = 0;  // launched on its own above; no item refers to it
                continue;
            }
            int so = 0;
            batch_kind_of(r.seg.n0, r.seg.n1, r.seg.n2, r.seg.precision, r.seg.direction, nullptr,
                          nullptr, nullptr, &so);
            solo[r.kind] = (unsigned char)so;
        }
        for (int oi = 0; oi < nseg; ++oi) {
            const int i = order[oi];
            const ServeReq &r = slot.reqs[i];
            if (r.kind < 0) continue;
            for (long long v0 = 0; v0 < r.seg.batch; v0 += r.vpc) {
                BatchItem &it = slot.h_items[n++];
                it.kind = r.kind;
                it.seg = i;
                it.v0 = v0;
                it.nv = (int)std::min<long long>(r.vpc, r.seg.batch - v0);
                it.pad = 0;
            }
        }
        if (n > 0 &&
            (cudaMemcpyAsync(slot.d_items, slot.h_items, (size_t)n * sizeof(BatchItem),
                             cudaMemcpyHostToDevice, st) != cudaSuccess ||
             cudaMemcpyAsync(slot.d_segs, slot.h_segs, (size_t)nseg * sizeof(BatchSeg),
                             cudaMemcpyHostToDevice, st) != cudaSuccess ||
             cudaMemcpyAsync(slot.d_solo, solo, sizeof solo, cudaMemcpyHostToDevice, st) != cudaSuccess ||
             cudaMemsetAsync(slot.d_ticket, 0, sizeof(unsigned int), st) != cudaSuccess))
            return FFT3D_B200_ERR_CUDA;
        const BatchItem *items = slot.d_items;
        const BatchSeg *segs = slot.d_segs;
        unsigned int *ticket = slot.d_ticket;
        unsigned char *scratch = slot.d_scratch;
        long long spc = s->scratch_per_cta;
        const unsigned char *so = slot.d_solo;
        int *err = slot.d_err;
        int grid = std::min(s->grid, n);
        void *args[] = {(void *)&items, (void *)&n,       (void *)&segs, (void *)&ticket,
                        (void *)&scratch, (void *)&spc, (void *)&so,   (void *)&err};
        if (n > 0 && cudaLaunchKernel(batch_kernel_func(), dim3(grid), dim3(batch_kernel_threads()), args,
                                      (size_t)batch_kernel_smem(), st) != cudaSuccess)
            return FFT3D_B200_ERR_CUDA;
    }
    if (cudaEventRecord(slot.done, st) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    return FFT3D_B200_OK;
}

static void server_loop(fft3d_b200_server *s)
{
    cudaSetDevice(s->device);
    const bool plain = (s->flags & FFT3D_B200_SERVE_PLAIN) != 0;
    std::vector<ServeSlot *> to_launch;
    bool blocked = false;  // the queue's head waits for a slot or for budget
    while (true) {
        // Without the lock (only this thread changes the slots): is there work --
        // a launch that finished, or a request that may be admitted?  While
        // launches are in flight the thread polls (a sleep would round up to
        // the kernel's timer slack, tens of microseconds); idle, it waits for a
        // submission.  Submitters take the lock only to queue.
        bool in_flight = false, finished = false;
        for (ServeSlot &slot : s->slots) {
            if (!slot.busy) continue;
            in_flight = true;
            if (!finished && cudaEventQuery(slot.done) != cudaErrorNotReady) finished = true;
        }
        const bool admissible = !blocked && s->npending.load(std::memory_order_acquire) > 0;
        if (!finished && !admissible && !s->stop.load()) {
            if (in_flight) {
                std::this_thread::yield();
            } else {
                std::unique_lock<std::mutex> lk(s->mu);
                if (s->pending.empty() && !s->stop) s->cv.wait_for(lk, std::chrono::milliseconds(1));
                blocked = false;
            }
            continue;
        }
        std::unique_lock<std::mutex> lk(s->mu);
        // retire finished launches
        for (ServeSlot &slot : s->slots) {
            if (!slot.busy) continue;
            const cudaError_t q = cudaEventQuery(slot.done);
            if (q == cudaErrorNotReady) continue;
            const double t = now_s();
            if (q != cudaSuccess) s->status = FFT3D_B200_ERR_CUDA;
            for (const ServeReq &r : slot.reqs) {
                s->lat.push_back(t - r.t_submit);
                s->lat_ticket.push_back(r.ticket);
                s->completed.push_back(r.ticket);
                s->volumes += r.seg.batch;
                ++s->finished;
            }
            s->t_last = t;
            s->used -= slot.bytes;
            slot.reqs.clear();
            slot.bytes = 0;
            slot.busy = false;
        }
        // admit pending requests, FIFO, into free slots
        to_launch.clear();
        for (ServeSlot &slot : s->slots) {
            if (s->pending.empty()) break;
            if (slot.busy) continue;
            long long items = 0;
            // plain mode launches one request per slot use; batching takes all that fit
            while (!s->pending.empty()) {
                const ServeReq &r = s->pending.front();
                if (s->used + r.bytes > s->budget) break;
                if ((int)slot.reqs.size() + 1 > SERVE_MAX_SEGS || items + r.nitems > SERVE_MAX_ITEMS) break;
                if (plain && !slot.reqs.empty()) break;
                items += r.nitems;
                s->used += r.bytes;
                slot.bytes += r.bytes;
                slot.reqs.push_back(r);
                s->pending.pop_front();
                s->npending.fetch_sub(1, std::memory_order_relaxed);
            }
            if (slot.reqs.empty()) break;  // head of queue waits for budget
            s->peak_used = std::max(s->peak_used, s->used);
            slot.busy = true;
            ++s->batches;
            s->batched_requests += (long long)slot.reqs.size();
            to_launch.push_back(&slot);
        }
        // requests left queued wait for a launch to finish (a slot or budget)
        blocked = !s->pending.empty();
        s->cv.notify_all();
        bool any_busy = false;
        for (const ServeSlot &slot : s->slots) any_busy |= slot.busy;
        if (s->stop && s->pending.empty() && !any_busy) break;
        // descriptors and launches outside the lock: submitters are not held up;
        // the slots are this thread's own until they are retired above
        lk.unlock();
        for (ServeSlot *slot : to_launch) {
            const int st = launch_slot(s, *slot);
            if (st) {
                std::lock_guard<std::mutex> g(s->mu);
                s->status = st;
            }
        }
    }
}

static void server_free(fft3d_b200_server *s)
{
    for (ServeSlot &slot : s->slots) {
        if (slot.d_work) {  // stream-ordered, before the stream goes
            cudaFreeAsync(slot.d_work, slot.stream);
            cudaStreamSynchronize(slot.stream);
        }
        if (slot.stream) cudaStreamDestroy(slot.stream);
        if (slot.done) cudaEventDestroy(slot.done);
        cudaFree(slot.d_items);
        cudaFree(slot.d_segs);
        cudaFree(slot.d_ticket);
        cudaFree(slot.d_solo);
        cudaFree(slot.d_scratch);
        cudaFree(slot.d_err);
        if (slot.h_items) cudaFreeHost(slot.h_items);
        if (slot.h_segs) cudaFreeHost(slot.h_segs);
    }
    delete s;
}

extern "C" int fft3d_b200_server_create(size_t hbm_budget_bytes, int max_inflight, unsigned flags,
                                        int device, fft3d_b200_server **out)
{
    if (!out || max_inflight < 1 || max_inflight > 64 || hbm_budget_bytes == 0)
        return FFT3D_B200_ERR_INVALID;
    *out = nullptr;
    int prev = -1;
    cudaGetDevice(&prev);
    if (device < 0) device = prev < 0 ? 0 : prev;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return FFT3D_B200_ERR_CUDA;
    }
    int st = ensure_device_tables(device);
    if (st) return st;
    fft3d_b200_server *s = new fft3d_b200_server();
    s->device = device;
    s->flags = flags;
    s->budget = hbm_budget_bytes;
    auto fail = [&](int code) {
        cudaGetLastError();
        server_free(s);
        if (prev >= 0) cudaSetDevice(prev);
        return code;
    };
    if (cudaFuncSetAttribute(batch_kernel_func(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             batch_kernel_smem()) != cudaSuccess)
        return fail(FFT3D_B200_ERR_CUDA);
    int occ = 0, sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel_func(), batch_kernel_threads(),
                                                      (size_t)batch_kernel_smem()) != cudaSuccess ||
        occ < 1)
        return fail(FFT3D_B200_ERR_UNSUPPORTED);
    s->grid = occ * sms;
    s->scratch_per_cta = (long long)36 * 36 * 36 * 16;  // the largest two-phase volume
    s->slots.resize((size_t)max_inflight);
    for (ServeSlot &slot : s->slots) {
        if (cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc(&slot.d_err, sizeof(int)) != cudaSuccess ||
            cudaMemset(slot.d_err, 0, sizeof(int)) != cudaSuccess)
            return fail(FFT3D_B200_ERR_NOMEM);
        if (!(flags & FFT3D_B200_SERVE_PLAIN)) {
            if (cudaMalloc(&slot.d_items, sizeof(BatchItem) * SERVE_MAX_ITEMS) != cudaSuccess ||
                cudaMalloc(&slot.d_segs, sizeof(BatchSeg) * SERVE_MAX_SEGS) != cudaSuccess ||
                cudaMalloc(&slot.d_ticket, sizeof(unsigned int)) != cudaSuccess ||
                cudaMalloc(&slot.d_solo, BATCH_NKINDS) != cudaSuccess ||
                cudaMalloc(&slot.d_scratch, (size_t)s->scratch_per_cta * s->grid) != cudaSuccess ||
                cudaHostAlloc(&slot.h_items, sizeof(BatchItem) * SERVE_MAX_ITEMS, 0) != cudaSuccess ||
                cudaHostAlloc(&slot.h_segs, sizeof(BatchSeg) * SERVE_MAX_SEGS, 0) != cudaSuccess)
                return fail(FFT3D_B200_ERR_NOMEM);
        }
    }
    s->thr = std::thread(server_loop, s);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    *out = s;
    return FFT3D_B200_OK;
}

// Queue one request; its latency counts from t_arrival (< 0: now, under the lock).
static int server_submit_at(fft3d_b200_server *s, const fft3d_b200_segment *req,
                            unsigned long long *ticket, double t_arrival)
{
    if (!s || !req) return FFT3D_B200_ERR_INVALID;
    const fft3d_b200_segment &q = *req;
    if (q.n0 < 1 || q.n1 < 1 || q.n2 < 1 || q.batch < 1 || !q.in || !q.out)
        return FFT3D_B200_ERR_INVALID;
    if ((q.direction != FFT3D_B200_FORWARD && q.direction != FFT3D_B200_BACKWARD) ||
        (q.precision != FFT3D_B200_C128 && q.precision != FFT3D_B200_C64))
        return FFT3D_B200_ERR_INVALID;
    ServeReq r;
    r.seg = q;
    r.kind = batch_kind_of(q.n0, q.n1, q.n2, q.precision, q.direction, &r.vpc, &r.big,
                           &r.vol_elems, nullptr);
    if (r.kind < 0) {
        // not a kind of the persistent kernel: served by its own tuned launch
        if (!fft3d_b200_supports(q.n0, q.n1, q.n2, q.precision)) return FFT3D_B200_ERR_UNSUPPORTED;
        r.vpc = 1;
        r.big = 0;
        r.vol_elems = (long long)q.n0 * q.n1 * q.n2;
    }
    const size_t eb = (size_t)element_bytes(q.precision);
    r.bytes = 2 * (size_t)q.batch * (size_t)r.vol_elems * eb;
    if (((uintptr_t)q.in % eb) || ((uintptr_t)q.out % eb)) return FFT3D_B200_ERR_ALIGN;
    const char *a = (const char *)q.in, *o = (const char *)q.out;
    if (a < o + r.bytes / 2 && o < a + r.bytes / 2) return FFT3D_B200_ERR_OVERLAP;
    if (r.bytes > s->budget) return FFT3D_B200_ERR_BUDGET;
    r.nitems = r.kind < 0 ? 0 : (q.batch + r.vpc - 1) / r.vpc;
    if (r.nitems > SERVE_MAX_ITEMS) return FFT3D_B200_ERR_BUDGET;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r.ticket = s->next_ticket++;
        r.t_submit = t_arrival >= 0.0 ? t_arrival : now_s();
        if (s->submitted == 0) s->t_first = r.t_submit;
        ++s->submitted;
        s->pending.push_back(r);
        s->npending.fetch_add(1, std::memory_order_release);
    }
    s->cv.notify_all();
    if (ticket) *ticket = r.ticket;
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_server_submit(fft3d_b200_server *s, const fft3d_b200_segment *req,
                                        unsigned long long *ticket)
{
    return server_submit_at(s, req, ticket, -1.0);
}

// Requests with arrival times: latency counts from the scheduled arrival, so a
// submission delayed behind the server (queueing in the client) is charged to
// the request, as an open-loop load generator must.
extern "C" int fft3d_b200_server_submit_many(fft3d_b200_server *s, const fft3d_b200_segment *reqs,
                                             const double *arrival_s, int n,
                                             unsigned long long *tickets)
{
    if (!s || n < 0 || (n > 0 && !reqs)) return FFT3D_B200_ERR_INVALID;
    const double t0 = now_s();
    for (int k = 0; k < n; ++k) {
        double t_arr = -1.0;
        if (arrival_s) {
            t_arr = t0 + arrival_s[k];
            while (now_s() < t_arr) {
            }
        }
        const int st = server_submit_at(s, &reqs[k], tickets ? &tickets[k] : nullptr, t_arr);
        if (st) return st;
    }
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_server_poll(fft3d_b200_server *s, unsigned long long *tickets, int max)
{
    if (!s || max < 0 || (max > 0 && !tickets)) return FFT3D_B200_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    int n = 0;
    while (n < max && !s->completed.empty()) {
        tickets[n++] = s->completed.front();
        s->completed.pop_front();
    }
    return n;
}

extern "C" int fft3d_b200_server_drain(fft3d_b200_server *s, double timeout_s)
{
    if (!s) return FFT3D_B200_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    const double t_end = now_s() + timeout_s;
    while (s->finished < s->submitted) {
        if (now_s() > t_end) return FFT3D_B200_ERR_TIMEOUT;
        s->cv.wait_for(lk, std::chrono::milliseconds(1));
    }
    return s->status;
}

extern "C" int fft3d_b200_server_get_stats(fft3d_b200_server *s, fft3d_b200_server_stats *out)
{
    if (!s || !out) return FFT3D_B200_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof *out);
    out->requests = (long long)s->finished;
    out->volumes = s->volumes;
    out->launches = s->batches;
    out->mean_requests_per_launch = s->batches ? (double)s->batched_requests / (double)s->batches : 0.0;
    out->peak_admitted_bytes = (long long)s->peak_used;
    if (!s->lat.empty()) {
        std::vector<double> l = s->lat;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) {
            size_t i = (size_t)(p * (double)(l.size() - 1) + 0.5);
            return l[std::min(i, l.size() - 1)];
        };
        out->p50_s = pct(0.50);
        out->p99_s = pct(0.99);
        out->max_s = l.back();
        double sum = 0;
        for (double v : l) sum += v;
        out->mean_s = sum / (double)l.size();
        const double span = s->t_last - s->t_first;
        out->volumes_per_s = span > 0 ? (double)s->volumes / span : 0.0;
        out->span_s = span;
    }
    return s->status;
}

extern "C" long long fft3d_b200_server_latencies(fft3d_b200_server *s, unsigned long long *tickets,
                                                double *latency_s, long long max)
{
    if (!s || max < 0 || (max > 0 && (!tickets || !latency_s))) return FFT3D_B200_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    const long long n = std::min<long long>(max, (long long)s->lat.size());
    for (long long k = 0; k < n; ++k) {
        tickets[k] = s->lat_ticket[(size_t)k];
        latency_s[k] = s->lat[(size_t)k];
    }
    return n;
}

extern "C" void fft3d_b200_server_destroy(fft3d_b200_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->thr.joinable()) s->thr.join();
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    server_free(s);
    if (prev >= 0) cudaSetDevice(prev);
}

/* fft3d_b200.h -- extension API of the B200 batched 3D complex FFT.
 *
 * The six symbols of the reference contract are unchanged and live in
 * fft3d_api.h (host pointers) and fft3d_gpu_api.h (device pointers).  This header
 * adds what that contract cannot express (it is forward-only, cubes only,
 * complex double only, with void returns):
 *
 *   - anisotropic n0 x n1 x n2 extents       (python/fft3d.py:360-371 handles any shape)
 *   - direction: forward, or backward with 1/V (python/fft3d.py:402-423)
 *   - precision: complex128, complex64 in FP32 (python/fft3d.py:368-371 keeps c64 I/O)
 *   - status-returning execute on a caller stream, and host-pointer execute
 *   - descriptor-list batches of uneven geometry run by one persistent launch
 *
 * Layout everywhere: element (b, i0, i1, i2) at ((b*n0 + i0)*n1 + i1)*n2 + i2,
 * interleaved complex, batch slowest (bench/geom/fft3d_api.h:14-18).
 * All transforms are out-of-place; `in` is never written.
 */
#ifndef FFT3D_B200_H
#define FFT3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  0 is success; every failure is negative. */
#define FFT3D_B200_OK 0
#define FFT3D_B200_ERR_INVALID (-1)     /* null pointer, non-positive extent, bad enum */
#define FFT3D_B200_ERR_UNSUPPORTED (-2) /* geometry / precision this build has no kernel for */
#define FFT3D_B200_ERR_ALIGN (-3)       /* buffer not aligned to its element size */
#define FFT3D_B200_ERR_CUDA (-4)        /* a CUDA runtime call failed (fault, launch error) */
#define FFT3D_B200_ERR_NOMEM (-5)       /* device or pinned-host allocation failed */
#define FFT3D_B200_ERR_TIMEOUT (-6)     /* a bounded device-side wait ran out */
#define FFT3D_B200_ERR_BUDGET (-7)      /* request larger than the admission budget */
#define FFT3D_B200_ERR_OVERLAP (-8)     /* in and out overlap; transforms are out-of-place */
#define FFT3D_B200_ERR_BUSY (-9)        /* server queue full; retry later */
#define FFT3D_B200_ERR_PEER (-10)       /* multi-GPU: two listed devices cannot reach each other */

#define FFT3D_B200_FORWARD (-1)  /* exp(-2*pi*i k.j/n), unnormalised */
#define FFT3D_B200_BACKWARD (+1) /* exp(+2*pi*i k.j/n), scaled by 1/(n0*n1*n2) */

#define FFT3D_B200_C128 0 /* complex double in, complex double out, FP64 arithmetic */
#define FFT3D_B200_C64 1  /* complex float in and out, FP32 arithmetic */

/* Plan flags. */
#define FFT3D_B200_FLAG_NO_TUNE 0x1u   /* take the default kernel instead of timing candidates */
#define FFT3D_B200_FLAG_NO_GRAPH 0x2u  /* batches: launch directly instead of replaying a CUDA graph */
#define FFT3D_B200_BATCH_PERSISTENT 0x4u /* batches: always the one persistent descriptor-list kernel */
#define FFT3D_B200_BATCH_SEGMENTS 0x8u   /* batches: always one tuned plan per segment */

typedef struct fft3d_b200_plan fft3d_b200_plan;

typedef struct {
    int n0, n1, n2;      /* extents; n2 is the fastest-varying axis */
    long long batch;     /* number of volumes, >= 0 */
    int direction;       /* FFT3D_B200_FORWARD or FFT3D_B200_BACKWARD */
    int precision;       /* FFT3D_B200_C128 or FFT3D_B200_C64 */
    unsigned flags;      /* FFT3D_B200_FLAG_* */
    int device;          /* CUDA device ordinal; -1 = the current device */
} fft3d_b200_desc;

/* Nonzero when this build has a kernel for the geometry and precision. */
int fft3d_b200_supports(int n0, int n1, int n2, int precision);

/* Create a plan: twiddle and Rader tables, kernel choice (timed candidates unless
 * FFT3D_B200_FLAG_NO_TUNE), staging for host-pointer execution.  Returns a status;
 * *out is NULL on failure. */
int fft3d_b200_plan_create(const fft3d_b200_desc *desc, fft3d_b200_plan **out);

void fft3d_b200_plan_destroy(fft3d_b200_plan *plan);

/* Transform device-resident data on `stream` (a cudaStream_t; NULL = the legacy
 * default stream).  Asynchronous: returns once the work is enqueued.  `in` and
 * `out` must be distinct device buffers of batch*n0*n1*n2 elements aligned to the
 * element size.  On any stream but the legacy default one the kernel is launched
 * with programmatic dependent launch: its CTAs may be placed while the previous
 * kernel of the stream drains, and wait for that kernel to complete before their
 * first global memory access (stream order is kept; FFT3D_B200_PDL=0 in the
 * environment launches in plain stream order). */
int fft3d_b200_execute(fft3d_b200_plan *plan, const void *d_in, void *d_out, void *stream);

/* Transform host data: copies in, transforms, copies out, and returns when `out`
 * holds the result.  Page-locked buffers are transferred directly; pageable ones
 * through the plan's pinned staging, in overlapped chunks.  Chunks are whole
 * volumes, at most about 1/8 of the batch (4..64 MB), with smaller chunks first
 * and last; FFT3D_B200_HOST_CHUNK_MB=<n> in the environment (read when a plan
 * first transfers host data) sets the largest chunk instead. */
int fft3d_b200_execute_host(fft3d_b200_plan *plan, const void *h_in, void *h_out);

/* Run plans[0], plans[1], ... back to back on the device between ONE host-to-device
 * copy of h_in and ONE device-to-host copy into h_out (e.g. a forward and a
 * backward plan for a round trip).  All plans must have the same geometry,
 * precision and batch. */
int fft3d_b200_execute_host_chain(fft3d_b200_plan *const *plans, int nplans, const void *h_in,
                                  void *h_out);

/* Names of the compiled kernel variants for a geometry, precision and direction
 * (the autotuner's candidates).  Writes up to `max` names and returns the count. */
int fft3d_b200_variants(int n0, int n1, int n2, int precision, int direction, const char **names,
                        int max);

/* Like fft3d_b200_plan_create, but use the named variant instead of tuning. */
int fft3d_b200_plan_create_variant(const fft3d_b200_desc *desc, const char *variant,
                                   fft3d_b200_plan **out);

/* Wait for the plan's device work and report a device-side failure recorded
 * since the last check (FFT3D_B200_ERR_TIMEOUT when a bounded wait ran out). */
int fft3d_b200_plan_check(fft3d_b200_plan *plan);

/* Test hook, no counterpart in the reference: make the next device-pointer
 * execute of a plan whose kernel keeps a scratch ring (TWOPASS variants) skip
 * the first volume's plane items, so its dependent waits run out.  The launch
 * ends by itself after the bounded wait (about 2 s), fft3d_b200_plan_check then
 * reports FFT3D_B200_ERR_TIMEOUT, and later executes run normally.  Returns
 * FFT3D_B200_ERR_UNSUPPORTED for other kernels. */
int fft3d_b200_debug_stall_next_execute(fft3d_b200_plan *plan);

/* Human-readable description of the kernel configuration the plan selected. */
const char *fft3d_b200_plan_describe(const fft3d_b200_plan *plan);

/* Number of kernel launches one execute of this plan issues. */
int fft3d_b200_plan_launches(const fft3d_b200_plan *plan);

/* Status of the most recent call into the reference-contract entry points
 * (fft3d_execute / fft3d_gpu_execute return void) on this host thread. */
int fft3d_b200_last_status(void);

const char *fft3d_b200_status_string(int status);

/* ---------------------------------------------------------------- plan wisdom
 *
 * The autotuner's choices -- device type (name, compute capability, SM count),
 * extents, precision, direction and batch-size class -> kernel variant -- kept
 * per process and saved to / loaded from a text file, so that later processes
 * on the same kind of GPU skip the plan-time timing race.  Replaces the
 * reference's per-create race (bench/geom/best/fft3d_best.c:148-193) by the
 * persisted per-host form bench/gen/PANEL_BRIEF.md:12-20 asks for; no
 * counterpart function exists in the reference.
 *
 * With FFT3D_B200_WISDOM=<path> set, the file is read at the first plan
 * creation and rewritten after each new choice.  Entries for device types not
 * present are kept; entries naming variants this build lacks are ignored. */

/* Write the choices made or imported so far; entries written, or an error code. */
int fft3d_b200_wisdom_export(const char *path);

/* Merge a wisdom file into this process's choices; entries taken, or an error code. */
int fft3d_b200_wisdom_import(const char *path);

/* Drop every remembered choice (plans created afterwards time their candidates again). */
void fft3d_b200_wisdom_forget(void);

/* ---------------------------------------------------------------- 4D lattices (L^3 x T)
 *
 * The 4D DFT over (t, x, y, z) of `desc->batch` lattices of nt x n0 x n1 x n2
 * points, element (b, t, x, y, z) at (((b*nt + t)*n0 + x)*n1 + y)*n2 + z: the
 * asymmetric L^3 x T extents the reference names as the lattice-QCD target
 * (docs/EXTENSIONS.md:55-64) and has no kernel for.  desc->n0..n2, direction,
 * precision, flags and device are those of the 3D part; the inverse is scaled by
 * 1/(nt*n0*n1*n2).  Supported: any 3D geometry this build has and
 * nt in {2, 4, 6, 8, 12, 16, 17, 24, 32, 36, 48, 64}.  No counterpart exists in
 * the reference. */

typedef struct fft3d_b200_plan4d fft3d_b200_plan4d;

/* Nonzero when nt x n0 x n1 x n2 lattices are supported in this precision. */
int fft3d_b200_plan4d_supports(int nt, int n0, int n1, int n2, int precision);

int fft3d_b200_plan4d_create(int nt, const fft3d_b200_desc *desc, fft3d_b200_plan4d **out);

/* Device pointers, distinct buffers of batch*nt*n0*n1*n2 elements; asynchronous. */
int fft3d_b200_plan4d_execute(fft3d_b200_plan4d *plan, const void *d_in, void *d_out, void *stream);

void fft3d_b200_plan4d_destroy(fft3d_b200_plan4d *plan);

const char *fft3d_b200_plan4d_describe(const fft3d_b200_plan4d *plan);

/* ---------------------------------------------------------------- batches of uneven geometry */

typedef struct {
    int n0, n1, n2;      /* extents of every volume of the segment */
    int direction;       /* FFT3D_B200_FORWARD / FFT3D_B200_BACKWARD */
    int precision;       /* FFT3D_B200_C128 / FFT3D_B200_C64 */
    long long batch;     /* volumes in the segment */
    const void *in;      /* device pointer */
    void *out;           /* device pointer */
} fft3d_b200_segment;

typedef struct fft3d_b200_batch fft3d_b200_batch;

/* Build a batch over `nseg` segments.  Two launch strategies exist:
 *   persistent -- one kernel walks a device descriptor list of work items of
 *                 every segment (one launch for the whole batch);
 *   segments   -- one autotuned plan per segment, the launches captured as
 *                 parallel branches of one CUDA graph.
 * By default both are built and timed on the batch's own buffers and the faster
 * is kept: batch_create runs the batch a few times and so writes the segments'
 * output buffers.  FFT3D_B200_BATCH_PERSISTENT / FFT3D_B200_BATCH_SEGMENTS pick
 * one without timing; FFT3D_B200_FLAG_NO_TUNE takes the persistent kernel.
 * Unless FFT3D_B200_FLAG_NO_GRAPH, the launches are replayed from a CUDA graph.
 * With the persistent kernel every volume's result is bit-identical alone and in
 * any mix; with per-segment plans a segment's kernel is chosen for its size. */
int fft3d_b200_batch_create(const fft3d_b200_segment *segs, int nseg, unsigned flags, int device,
                            fft3d_b200_batch **out);

/* Run every segment of the batch on `stream` (one graph launch). */
int fft3d_b200_batch_execute(fft3d_b200_batch *batch, void *stream);

void fft3d_b200_batch_destroy(fft3d_b200_batch *batch);

const char *fft3d_b200_batch_describe(const fft3d_b200_batch *batch);

/* ---------------------------------------------------------------- chains */

/* The reference's chain workloads (docs/GRADER.md, bench/geom/best/ours_chain.c:36-53):
 * m forward transforms, each followed by a pointwise step. */
#define FFT3D_B200_CHAIN_UNITARY 1 /* state <- FFT(state) * V^(-1/2) */
#define FFT3D_B200_CHAIN_MAP 2     /* z = FFT(state) + c;  state <- z / (1 + |z|) */

typedef struct fft3d_b200_chain fft3d_b200_chain;

/* A chain over `batch` volumes; for CHAIN_MAP, `d_c` is the constant field
 * (device pointer, same shape and precision as the state). */
int fft3d_b200_chain_create(int n0, int n1, int n2, long long batch, int precision, int kind,
                            const void *d_c, int device, fft3d_b200_chain **out);

/* Run `steps` chain steps from d_x0, leaving the end state in d_out (one launch;
 * each volume stays in one CTA's shared memory for the whole chain). */
int fft3d_b200_chain_run(fft3d_b200_chain *chain, const void *d_x0, void *d_out, long long steps,
                         void *stream);

void fft3d_b200_chain_destroy(fft3d_b200_chain *chain);

/* ---------------------------------------------------------------- serving */

typedef struct fft3d_b200_server fft3d_b200_server;

#define FFT3D_B200_SERVE_PLAIN 0x1u /* baseline: one launch per request, no coalescing */

typedef struct {
    long long requests;         /* finished */
    long long volumes;          /* finished */
    long long launches;         /* batch launches (plain mode: request launches) */
    double mean_requests_per_launch;
    long long peak_admitted_bytes; /* high-water mark of admitted in+out bytes */
    double p50_s, p99_s, mean_s, max_s; /* submit-to-completion latency */
    double volumes_per_s;       /* finished volumes / (last completion - first submission) */
    double span_s;
} fft3d_b200_server_stats;

/* Start a continuous-batching server on `device`: requests (segments with device
 * in/out pointers) are admitted while the in+out bytes of unfinished requests
 * stay within `hbm_budget_bytes`, coalesced into persistent batch launches on up
 * to `max_inflight` concurrent streams, and completed asynchronously. */
int fft3d_b200_server_create(size_t hbm_budget_bytes, int max_inflight, unsigned flags, int device,
                             fft3d_b200_server **out);

/* Queue one request (thread-safe).  FFT3D_B200_ERR_BUDGET if it alone exceeds
 * the budget.  `ticket` identifies it in fft3d_b200_server_poll.  Extents of the
 * persistent batch kernel are coalesced; any other extent with a kernel that
 * compiled extent is served by its own tuned launch in the same slot (a
 * kernel with a scratch ring -- 45^3, 64^3, complex128 30^3 -- with the slot's
 * workspace, allocated on first need); an extent without a kernel is refused
 * with FFT3D_B200_ERR_UNSUPPORTED. */
int fft3d_b200_server_submit(fft3d_b200_server *server, const fft3d_b200_segment *request,
                             unsigned long long *ticket);

/* Load generator: submit requests[k] at arrival_s[k] seconds after the call
 * starts (busy-waiting between arrivals; NULL arrival_s = all at once), from the
 * calling thread.  Returns after the last submission; tickets (optional) get the
 * request tickets.  Stops at the first refused request and returns its status. */
int fft3d_b200_server_submit_many(fft3d_b200_server *server, const fft3d_b200_segment *requests,
                                  const double *arrival_s, int n, unsigned long long *tickets);

/* Tickets of requests finished since the last poll, in completion order; returns
 * how many were written (<= max). */
int fft3d_b200_server_poll(fft3d_b200_server *server, unsigned long long *tickets, int max);

/* Wait until every submitted request has finished (FFT3D_B200_ERR_TIMEOUT after
 * `timeout_s` seconds). */
int fft3d_b200_server_drain(fft3d_b200_server *server, double timeout_s);

/* Latency percentiles and throughput of everything finished so far. */
int fft3d_b200_server_get_stats(fft3d_b200_server *server, fft3d_b200_server_stats *stats);

/* Per-request latencies of the first `max` finished requests, in completion
 * order: tickets[k] finished latency_s[k] seconds after its submission (host
 * clock).  Returns how many were written (a negative status on bad arguments),
 * so a caller can take percentiles over a steady-state window of the stream. */
long long fft3d_b200_server_latencies(fft3d_b200_server *server, unsigned long long *tickets,
                                      double *latency_s, long long max);

void fft3d_b200_server_destroy(fft3d_b200_server *server);

/* Run the segments as one persistent batch launch on `stream` WITHOUT allocating
 * any device memory -- no counterpart in the reference.  For callers that may
 * not call cudaMalloc (an application whose pool allocator owns all device
 * memory, a latency-critical loop that cannot pay cudaMalloc's implicit
 * synchronisation, a plugin host that forbids allocation): the descriptor list,
 * work ticket and error word live in one static device array of about 540 KB
 * that the library holds on every GPU that loads it.  Limits: at most 256
 * segments and 16384 work items per call, and no 36^3 segments (their two-phase
 * route needs more scratch than the array holds); beyond these it returns
 * FFT3D_B200_ERR_BUDGET and enqueues nothing.  The first call on a device looks
 * up the array's device address (make it before any stream capture).  Calls
 * share the array and reset its ticket on their stream: host threads calling
 * on the same stream are serialised, but calls that overlap on the GPU
 * (different streams) race, so order them (one stream, or events).  The
 * descriptors are copied from the call's stack memory, so while `stream` is
 * being captured the call returns FFT3D_B200_ERR_INVALID and enqueues nothing. */
int fft3d_b200_batch_execute_noalloc(const fft3d_b200_segment *segs, int nseg, void *stream);

/* Status of the allocation-free launches enqueued on `stream` -- no counterpart
 * in the reference.  Synchronises `stream`; FFT3D_B200_ERR_CUDA if a launch
 * failed, FFT3D_B200_ERR_TIMEOUT if the shared array's device error word is
 * set, else FFT3D_B200_OK.  Allocates nothing. */
int fft3d_b200_noalloc_check(void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FFT3D_B200_H */

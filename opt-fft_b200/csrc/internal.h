// internal.h -- shared declarations of the library (not installed).
#pragma once

#include <cuda_runtime.h>

#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/fft3d_b200.h"

namespace fft3d {

void ensure_host_tables();
int ensure_device_tables(int device);
// Set the calling thread's fft3d_b200_last_status() and return the code.
int record_status(int s);

// Kernel family of a registry entry.
enum Family : int {
    FAM_VOLUME = 0,   // one CTA transforms VPC whole volumes held in its shared memory
    FAM_CLUSTER = 1,  // a thread-block cluster shares one volume through distributed smem
    FAM_STREAM = 2,   // persistent CTAs, two-stage pipeline: load of the next group in flight
    FAM_TWOPASS = 3,  // persistent CTAs, plane and row passes through an L2-resident scratch ring
};

// TWOPASS workspace: a control block (ticket, exit count, abort flag, per-slot
// completion counters) followed by a ring of R scratch volumes.
constexpr int TWOPASS_RMAX = 128;
constexpr size_t TWOPASS_CTL_BYTES = 4096;
struct TwoPassCtl {
    unsigned long long ticket;          // next work item
    unsigned done;                      // CTAs that have left
    unsigned abort;                     // set by a CTA whose wait timed out
    unsigned cnt[2 * TWOPASS_RMAX];     // [s]: plane items done on slot s; [RMAX + s]: row items
};
static_assert(sizeof(TwoPassCtl) <= TWOPASS_CTL_BYTES, "control block");

// One compiled kernel variant.  The plan's autotuner times the entries that
// match its geometry, precision and direction and keeps the fastest.
struct KernelEntry {
    int n0, n1, n2;
    int precision;      // FFT3D_B200_C128 / FFT3D_B200_C64
    int sign;           // -1 forward, +1 backward
    int family;
    int alg;            // codelet variant for extent 17 (0 folded direct, 1 Rader-FFT16)
    int vpc;            // volumes per CTA (VOLUME) / CTAs per cluster (CLUSTER) /
                        // planes (and rows) per work item (TWOPASS)
    int threads;        // threads per CTA
    int smem;           // dynamic shared memory bytes per CTA
    const void *func;   // __global__ function
    const char *name;
};

// Registry of every compiled variant (defined by the kernel translation units).
const std::vector<KernelEntry> &registry();
void register_kernels(std::vector<KernelEntry> &out);          // volume_kernels.cu
void register_stream_kernels(std::vector<KernelEntry> &out);   // stream_kernels.cu
void register_direct_kernels(std::vector<KernelEntry> &out);   // direct_kernels.cu
void register_tc_kernels(std::vector<KernelEntry> &out);       // tc_kernels.cu
int tc_tables_upload();                                         // split-BF16 DFT matrices
void register_cluster_kernels(std::vector<KernelEntry> &out);  // cluster_kernels.cu
void register_twopass_kernels(std::vector<KernelEntry> &out);  // twopass_kernels.cu

// TWOPASS ring geometry for a launch of `grid` CTAs: returns the ring size R
// (scratch volumes) and sets *lag to D, the distance in steps between the
// plane items and the row items of one volume in the ticket order (D < R).
int twopass_ring(const KernelEntry &e, long long grid, int *lag);

// Device workspace a launch of `e` with up to `grid_limit` CTAs needs (0 for
// every family but TWOPASS).  The control block must be zero before the first
// launch; each launch leaves it zero again.
size_t entry_workspace_bytes(const KernelEntry &e, int grid_limit);

// Launch `e` over `nvol` volumes.  scale multiplies every output (1/V for inverse).
// Persistent families use at most `grid_limit` CTAs; `err` is the device error word;
// `work` is the entry's workspace (entry_workspace_bytes), required for TWOPASS.
// Launches that share one workspace must be ordered (one stream).
cudaError_t launch_entry(const KernelEntry &e, const void *in, void *out, long long nvol,
                         double scale, cudaStream_t stream, int grid_limit, int *err,
                         void *work = nullptr);

// CTAs of `e` that fit on one SM (0 if it cannot launch); sets attributes on first use.
int entry_occupancy(const KernelEntry &e, int device);

int element_bytes(int precision);

// The autotuner's choice for a geometry at a batch size (memoised per batch
// bucket like plan creation); nullptr if the geometry has no kernel.  Without
// `workspace_ok` it chooses among the kernels that need no workspace (a caller
// that launches on several streams at once and holds none); with it, among all
// of them, as plan creation does -- the caller then passes a workspace of
// entry_workspace_bytes to launch_entry.
const KernelEntry *tuned_entry(int device, int n0, int n1, int n2, int precision, int sign,
                               long long batch, bool workspace_ok = false);

}  // namespace fft3d

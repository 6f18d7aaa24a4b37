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

// Kernel family of a registry entry.
enum Family : int {
    FAM_VOLUME = 0,   // one CTA transforms VPC whole volumes held in its shared memory
    FAM_CLUSTER = 1,  // a thread-block cluster shares one volume through distributed smem
    FAM_STREAM = 2,   // persistent CTAs, two-stage pipeline: load of the next group in flight
};

// One compiled kernel variant.  The plan's autotuner times the entries that
// match its geometry, precision and direction and keeps the fastest.
struct KernelEntry {
    int n0, n1, n2;
    int precision;      // FFT3D_B200_C128 / FFT3D_B200_C64
    int sign;           // -1 forward, +1 backward
    int family;
    int alg;            // codelet variant for extent 17 (0 folded direct, 1 Rader-FFT16)
    int vpc;            // volumes per CTA (VOLUME) / CTAs per cluster (CLUSTER)
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

// Launch `e` over `nvol` volumes.  scale multiplies every output (1/V for inverse).
// Persistent families use at most `grid_limit` CTAs; `err` is the device error word.
cudaError_t launch_entry(const KernelEntry &e, const void *in, void *out, long long nvol,
                         double scale, cudaStream_t stream, int grid_limit, int *err);

// CTAs of `e` that fit on one SM (0 if it cannot launch); sets attributes on first use.
int entry_occupancy(const KernelEntry &e, int device);

int element_bytes(int precision);

// The autotuner's choice for a geometry at a batch size (memoised per batch
// bucket like plan creation); nullptr if the geometry has no kernel.
const KernelEntry *tuned_entry(int device, int n0, int n1, int n2, int precision, int sign,
                               long long batch);

}  // namespace fft3d

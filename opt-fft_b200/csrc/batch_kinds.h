// batch_kinds.h -- the geometries the descriptor-list batch kernel is compiled
// for, and the device descriptors it walks.
#pragma once

#include <stdint.h>

namespace fft3d {

// One work item: `nv` volumes of segment `seg`, starting at volume `v0`.
struct BatchItem {
    int kind;
    int seg;
    long long v0;
    int nv;
    int pad;
};

// One segment of the caller's batch (device pointers).
struct BatchSeg {
    const void *in;
    void *out;
    double scale;  // 1 forward, 1/V backward
    long long nvol;
    int kind;
    int pad;
};

// X(id, n0, n1, n2, real type, sign, volumes per item, solo, big-cube slab planes)
//   solo: the item needs all of shared memory (no prefetch around it)
//   big:  0, or the slab thickness of the two-phase path for cubes beyond one SM
//         (two slab buffers in shared memory)
#define FFT3D_BATCH_KINDS(X)                         \
    X(0, 6, 6, 6, double, -1, 28, 0, 0)              \
    X(1, 6, 6, 6, double, +1, 28, 0, 0)              \
    X(2, 8, 8, 8, double, -1, 14, 0, 0)               \
    X(3, 8, 8, 8, double, +1, 14, 0, 0)               \
    X(4, 12, 12, 12, double, -1, 3, 0, 0)            \
    X(5, 12, 12, 12, double, +1, 3, 0, 0)            \
    X(6, 16, 16, 16, double, -1, 1, 0, 0)            \
    X(7, 16, 16, 16, double, +1, 1, 0, 0)            \
    X(8, 17, 17, 17, double, -1, 1, 0, 0)            \
    X(9, 17, 17, 17, double, +1, 1, 0, 0)            \
    X(10, 24, 24, 24, double, -1, 1, 1, 0)           \
    X(11, 24, 24, 24, double, +1, 1, 1, 0)           \
    X(12, 36, 36, 36, double, -1, 1, 1, 4)           \
    X(13, 36, 36, 36, double, +1, 1, 1, 4)           \
    X(14, 8, 8, 16, double, -1, 7, 0, 0)             \
    X(15, 8, 8, 16, double, +1, 7, 0, 0)             \
    X(16, 16, 16, 32, double, -1, 1, 1, 0)           \
    X(17, 16, 16, 32, double, +1, 1, 1, 0)           \
    X(18, 6, 6, 6, float, -1, 57, 0, 0)              \
    X(19, 6, 6, 6, float, +1, 57, 0, 0)              \
    X(20, 8, 8, 8, float, -1, 25, 0, 0)               \
    X(21, 8, 8, 8, float, +1, 25, 0, 0)               \
    X(22, 12, 12, 12, float, -1, 7, 0, 0)            \
    X(23, 12, 12, 12, float, +1, 7, 0, 0)            \
    X(24, 16, 16, 16, float, -1, 3, 0, 0)            \
    X(25, 16, 16, 16, float, +1, 3, 0, 0)            \
    X(26, 17, 17, 17, float, -1, 2, 0, 0)            \
    X(27, 17, 17, 17, float, +1, 2, 0, 0)            \
    X(28, 24, 24, 24, float, -1, 1, 0, 0)            \
    X(29, 24, 24, 24, float, +1, 1, 0, 0)            \
    X(30, 36, 36, 36, float, -1, 1, 1, 6)            \
    X(31, 36, 36, 36, float, +1, 1, 1, 6)            \
    X(32, 8, 8, 16, float, -1, 14, 0, 0)              \
    X(33, 8, 8, 16, float, +1, 14, 0, 0)              \
    X(34, 16, 16, 32, float, -1, 1, 0, 0)            \
    X(35, 16, 16, 32, float, +1, 1, 0, 0)

constexpr int BATCH_NKINDS = 36;

// The complex64 kinds for the class-1 kernel (two CTAs per SM, half the shared
// memory each): the same ids, volumes per item re-sized for a 57 KB half; a
// 24^3 volume (115,200 bytes with its row padding) takes a CTA's whole share.
#define FFT3D_BATCH_KINDS_C64(X)                     \
    X(18, 6, 6, 6, float, -1, 28, 0, 0)              \
    X(19, 6, 6, 6, float, +1, 28, 0, 0)              \
    X(20, 8, 8, 8, float, -1, 12, 0, 0)              \
    X(21, 8, 8, 8, float, +1, 12, 0, 0)              \
    X(22, 12, 12, 12, float, -1, 3, 0, 0)            \
    X(23, 12, 12, 12, float, +1, 3, 0, 0)            \
    X(24, 16, 16, 16, float, -1, 1, 0, 0)            \
    X(25, 16, 16, 16, float, +1, 1, 0, 0)            \
    X(26, 17, 17, 17, float, -1, 1, 0, 0)            \
    X(27, 17, 17, 17, float, +1, 1, 0, 0)            \
    X(28, 24, 24, 24, float, -1, 1, 1, 0)            \
    X(29, 24, 24, 24, float, +1, 1, 1, 0)            \
    X(30, 36, 36, 36, float, -1, 1, 1, 4)            \
    X(31, 36, 36, 36, float, +1, 1, 1, 4)            \
    X(32, 8, 8, 16, float, -1, 7, 0, 0)              \
    X(33, 8, 8, 16, float, +1, 7, 0, 0)              \
    X(34, 16, 16, 32, float, -1, 1, 1, 0)            \
    X(35, 16, 16, 32, float, +1, 1, 1, 0)

// Kind lookup for the host side (batch.cu): returns the kind id or -1, and the
// kind's volumes per item, two-phase flag, volume size, and whether its items
// need all of shared memory.
int batch_kind_of(int n0, int n1, int n2, int precision, int sign, int *vpc, int *big,
                  long long *vol_elems, int *solo);

const void *batch_kernel_func();
int batch_kernel_threads();
int batch_kernel_smem();
int batch_kernel_half();
// the complex64 class (FFT3D_BATCH_KINDS_C64)
const void *batch_c64_kernel_func();
int batch_c64_kernel_threads();
int batch_c64_kernel_smem();
int batch_c64_kernel_half();

}  // namespace fft3d

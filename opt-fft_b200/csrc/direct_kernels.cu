// direct_kernels.cu -- kernel family DIRECT: the z pass reads HBM directly.
//
// z-lines are contiguous in the reference layout, so each thread streams its
// line's N2 points from HBM with back-to-back vector loads straight into
// registers, transforms it, and writes it once into the shared-memory layout;
// the y pass runs in shared memory and the x pass writes to HBM with coalesced
// streaming stores.  Shared-memory traffic per volume drops from six volume
// copies (stage in, z, y, x) to four, and there is no staging copy to wait for:
// latency is hidden by running several small CTAs per SM.
#include "internal.h"
#include "ptx.cuh"
#include "volume.cuh"

namespace fft3d {

template <class G, int S, int ALG, int VPC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_direct(const cx<typename G::T> *__restrict__ in, cx<typename G::T> *__restrict__ out,
             long long nvol, typename G::T scale)
{
    pdl_begin();
    using T = typename G::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    const long long v0 = (long long)blockIdx.x * VPC;
    const long long left = nvol - v0;
    const int nv = left < VPC ? (int)left : VPC;
    const cx<T> *gin = in + v0 * G::V;
    cx<T> *gout = out + v0 * G::V;
    const int tid = threadIdx.x;
    for (int r = tid; r < nv * G::ROWS; r += NT) pass_z_from_global<G, S, ALG>(sm, gin, r);
    __syncthreads();
    for (int l = tid; l < nv * G::N0 * G::N2; l += NT) pass_y<G, S, ALG>(sm, l);
    __syncthreads();
    for (int l = tid; l < nv * G::N1 * G::N2; l += NT) pass_x_out<G, S, ALG>(sm, l, gout, scale);
}

template <int N0, int N1, int N2, typename T, int S, int ALG, int VPC, int NT, int MINB>
static void add_direct(std::vector<KernelEntry> &out, const char *name)
{
    using G = Geom<N0, N1, N2, T>;
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_VOLUME;  // same launch shape as the VOLUME family
    e.alg = ALG;
    e.vpc = VPC;
    e.threads = NT;
    e.smem = VPC * G::PV * G::EB;
    e.func = (const void *)&k_direct<G, S, ALG, VPC, NT, MINB>;
    e.name = name;
    out.push_back(e);
}

#define FFT3D_DIRECT(N0, N1, N2, T, ALG, VPC, NT, MINB)                                       \
    add_direct<N0, N1, N2, T, -1, ALG, VPC, NT, MINB>(                                        \
        out, "direct " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " minb" #MINB); \
    add_direct<N0, N1, N2, T, +1, ALG, VPC, NT, MINB>(                                        \
        out, "direct " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " minb" #MINB)

// DIRECT, pipelined across items ("directp"): persistent CTAs, one item of
// VPC volumes at a time.  Each thread owns z-lines r = q*NT + tid of the item;
// right after the z pass has put the current item into shared memory, the
// thread starts loading its lines of the CTA's next item into the same
// registers, and only uses them after the current item's y and x passes -- so
// the HBM reads of one item overlap the arithmetic of the previous one, even
// when a single item fills an SM's shared memory (16x16x32 complex double,
// 131 KB).
template <class G, int S, int VPC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_direct_pipe(const cx<typename G::T> *__restrict__ in, cx<typename G::T> *__restrict__ out,
                  long long nvol, typename G::T scale, int *err)
{
    pdl_begin();
    (void)err;
    using T = typename G::T;
    constexpr int RPT = (VPC * G::ROWS + NT - 1) / NT;  // z-lines per thread
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    const int tid = threadIdx.x;
    const long long nitems = (nvol + VPC - 1) / VPC;
    long long item = blockIdx.x;
    if (item >= nitems) return;
    auto vols = [&](long long it) {
        const long long left = nvol - it * VPC;
        return left < VPC ? (int)left : VPC;
    };
    cx<T> v[RPT][G::N2];
    auto load = [&](long long it) {
        const cx<T> *g = in + it * VPC * G::V;
        const int nr = vols(it) * G::ROWS;
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            const int r = q * NT + tid;
            if (r < nr)
#pragma unroll
                for (int j = 0; j < G::N2; ++j) v[q][j] = load_in(g + (long long)r * G::N2 + j);
        }
    };
    load(item);
    for (; item < nitems; item += gridDim.x) {
        const int nv = vols(item);
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            const int r = q * NT + tid;
            if (r < nv * G::ROWS) {
                dft<G::N2, S, T>(v[q]);
#pragma unroll
                for (int j = 0; j < G::N2; ++j) sm[G::off(r, j)] = v[q][j];
            }
        }
        __syncthreads();
        if (item + gridDim.x < nitems) load(item + gridDim.x);  // consumed at the next z pass
        for (int l = tid; l < nv * G::N0 * G::N2; l += NT) pass_y<G, S, ALG_DEFAULT>(sm, l);
        __syncthreads();
        cx<T> *gout = out + item * VPC * G::V;
        for (int l = tid; l < nv * G::N1 * G::N2; l += NT) pass_x_out<G, S, ALG_DEFAULT>(sm, l, gout, scale);
        __syncthreads();  // shared memory is rewritten by the next z pass
    }
}

template <int N0, int N1, int N2, typename T, int S, int VPC, int NT, int MINB>
static void add_direct_pipe(std::vector<KernelEntry> &out, const char *name)
{
    using G = Geom<N0, N1, N2, T>;
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_STREAM;  // persistent launch over items of vpc volumes: (in, out, nvol, scale, err)
    e.alg = 0;
    e.vpc = VPC;
    e.threads = NT;
    e.smem = VPC * G::PV * G::EB;
    e.func = (const void *)&k_direct_pipe<G, S, VPC, NT, MINB>;
    e.name = name;
    out.push_back(e);
}

#define FFT3D_DIRECT_PIPE(N0, N1, N2, T, VPC, NT, MINB)                                            \
    add_direct_pipe<N0, N1, N2, T, -1, VPC, NT, MINB>(                                             \
        out, "directp " #N0 "x" #N1 "x" #N2 " " #T " vpc" #VPC " nt" #NT " minb" #MINB);           \
    add_direct_pipe<N0, N1, N2, T, +1, VPC, NT, MINB>(                                             \
        out, "directp " #N0 "x" #N1 "x" #N2 " " #T " vpc" #VPC " nt" #NT " minb" #MINB)

void register_direct_kernels(std::vector<KernelEntry> &out)
{
    // complex double
    FFT3D_DIRECT(6, 6, 6, double, 0, 8, 288, 3);
    FFT3D_DIRECT(8, 8, 8, double, 0, 4, 256, 3);
    FFT3D_DIRECT(8, 8, 8, double, 0, 2, 128, 6);
    FFT3D_DIRECT(12, 12, 12, double, 0, 1, 160, 4);
    FFT3D_DIRECT(12, 12, 12, double, 0, 2, 288, 2);
    FFT3D_DIRECT(16, 16, 16, double, 0, 1, 256, 2);
    FFT3D_DIRECT(17, 17, 17, double, 0, 1, 320, 2);
    FFT3D_DIRECT(17, 17, 17, double, 0, 1, 320, 1);
    FFT3D_DIRECT(24, 24, 24, double, 0, 1, 288, 1);
    FFT3D_DIRECT(8, 8, 16, double, 0, 2, 256, 2);
    FFT3D_DIRECT(16, 16, 32, double, 0, 1, 256, 1);
    // pipelined through registers
    FFT3D_DIRECT_PIPE(16, 16, 32, double, 1, 256, 1);
    FFT3D_DIRECT_PIPE(16, 16, 16, double, 1, 256, 1);
    FFT3D_DIRECT_PIPE(17, 17, 17, double, 1, 320, 1);
    FFT3D_DIRECT_PIPE(12, 12, 12, double, 2, 288, 1);
    FFT3D_DIRECT_PIPE(8, 8, 8, double, 4, 256, 2);
    // complex float
    FFT3D_DIRECT(6, 6, 6, float, 0, 16, 576, 2);
    FFT3D_DIRECT(8, 8, 8, float, 0, 8, 512, 2);
    FFT3D_DIRECT(8, 8, 8, float, 0, 4, 256, 4);
    FFT3D_DIRECT(12, 12, 12, float, 0, 2, 288, 3);
    FFT3D_DIRECT(16, 16, 16, float, 0, 2, 512, 2);
    FFT3D_DIRECT(16, 16, 16, float, 0, 1, 256, 4);
    FFT3D_DIRECT(17, 17, 17, float, 0, 2, 640, 1);
    FFT3D_DIRECT(17, 17, 17, float, 0, 1, 320, 3);
    FFT3D_DIRECT(24, 24, 24, float, 0, 1, 576, 1);
    FFT3D_DIRECT(8, 8, 16, float, 0, 4, 512, 2);
    FFT3D_DIRECT(16, 16, 32, float, 0, 1, 512, 1);
    // pipelined through registers
    FFT3D_DIRECT_PIPE(6, 6, 6, float, 16, 576, 1);
    FFT3D_DIRECT_PIPE(8, 8, 8, float, 4, 256, 3);
    FFT3D_DIRECT_PIPE(8, 8, 8, float, 8, 512, 2);
    FFT3D_DIRECT_PIPE(12, 12, 12, float, 2, 288, 3);
    FFT3D_DIRECT_PIPE(16, 16, 16, float, 1, 256, 3);
    FFT3D_DIRECT_PIPE(17, 17, 17, float, 1, 320, 2);
    FFT3D_DIRECT_PIPE(24, 24, 24, float, 1, 576, 1);
    FFT3D_DIRECT_PIPE(8, 8, 16, float, 8, 512, 2);
    FFT3D_DIRECT_PIPE(16, 16, 32, float, 1, 512, 1);
}

}  // namespace fft3d

// volume_kernels.cu -- kernel family VOLUME: one CTA transforms VPC whole volumes.
//
// Per CTA: the CTA's VPC volumes are read from HBM once with coalesced vector
// loads into the bank-conflict-free shared-memory layout of volume.cuh; the z and
// y passes run shared memory -> registers -> shared memory, one line per thread;
// the x pass reads shared memory and writes each result line straight to HBM with
// coalesced streaming stores, so each volume is written once.  This is the
// row-column structure of python/fft3d.py:349-399 and of the fused A100 kernels of
// the reference (bench/gpu/impl_4/L17_dmma.cu:36-38), laid out for sm_100a.
#include "internal.h"
#include "ptx.cuh"
#include "volume.cuh"

namespace fft3d {

template <class G, int S, int ALG, int VPC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_volume(const cx<typename G::T> *__restrict__ in, cx<typename G::T> *__restrict__ out,
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

    const int nel = nv * G::V;
    for (int g = tid; g < nel; g += NT) stage_in<G>(sm, gin, g);
    __syncthreads();
    for (int r = tid; r < nv * G::ROWS; r += NT) pass_z<G, S, ALG>(sm, r);
    __syncthreads();
    for (int l = tid; l < nv * G::N0 * G::N2; l += NT) pass_y<G, S, ALG>(sm, l);
    __syncthreads();
    for (int l = tid; l < nv * G::N1 * G::N2; l += NT) pass_x_out<G, S, ALG>(sm, l, gout, scale);
}

template <int N0, int N1, int N2, typename T, int S, int ALG, int VPC, int NT, int MINB>
static void add_volume(std::vector<KernelEntry> &out, const char *name)
{
    using G = Geom<N0, N1, N2, T>;
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_VOLUME;
    e.alg = ALG;
    e.vpc = VPC;
    e.threads = NT;
    e.smem = VPC * G::PV * G::EB;
    e.func = (const void *)&k_volume<G, S, ALG, VPC, NT, MINB>;
    e.name = name;
    out.push_back(e);
}

// Both directions of one variant.
#define FFT3D_VOL(N0, N1, N2, T, ALG, VPC, NT, MINB)                                              \
    add_volume<N0, N1, N2, T, -1, ALG, VPC, NT, MINB>(                                            \
        out, "volume " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " minb" #MINB); \
    add_volume<N0, N1, N2, T, +1, ALG, VPC, NT, MINB>(                                            \
        out, "volume " #N0 "x" #N1 "x" #N2 " " #T " alg" #ALG " vpc" #VPC " nt" #NT " minb" #MINB)

void register_kernels(std::vector<KernelEntry> &out)
{
    // complex double
    FFT3D_VOL(6, 6, 6, double, 0, 16, 256, 1);
    FFT3D_VOL(8, 8, 8, double, 0, 8, 256, 1);
    FFT3D_VOL(8, 8, 8, double, 0, 16, 512, 1);
    FFT3D_VOL(12, 12, 12, double, 0, 2, 288, 1);
    FFT3D_VOL(16, 16, 16, double, 0, 1, 256, 1);
    FFT3D_VOL(17, 17, 17, double, 0, 1, 320, 1);
    FFT3D_VOL(17, 17, 17, double, 1, 1, 320, 1);
    FFT3D_VOL(24, 24, 24, double, 0, 1, 288, 1);
    FFT3D_VOL(8, 8, 16, double, 0, 8, 512, 1);
    FFT3D_VOL(16, 16, 32, double, 0, 1, 256, 1);
    FFT3D_VOL(13, 13, 13, double, 0, 2, 352, 1);
    FFT3D_VOL(23, 23, 23, double, 0, 1, 288, 1);
    // complex float
    FFT3D_VOL(6, 6, 6, float, 0, 32, 512, 1);
    FFT3D_VOL(8, 8, 8, float, 0, 16, 512, 1);
    FFT3D_VOL(12, 12, 12, float, 0, 4, 576, 1);
    FFT3D_VOL(16, 16, 16, float, 0, 2, 512, 1);
    FFT3D_VOL(17, 17, 17, float, 0, 2, 608, 1);
    FFT3D_VOL(24, 24, 24, float, 0, 1, 576, 1);
    FFT3D_VOL(8, 8, 16, float, 0, 16, 1024, 1);
    FFT3D_VOL(16, 16, 32, float, 0, 1, 512, 1);
    FFT3D_VOL(13, 13, 13, float, 0, 4, 704, 1);
    FFT3D_VOL(23, 23, 23, float, 0, 1, 544, 1);

    // The other extents of the reference's oracle and tests
    // (python/test_fft3d.py:25-36): small cubes, 10^3, 15^3 and anisotropic
    // volumes, degenerate axes of length 1 included.  One CTA per group of
    // volumes; about 256-700 threads and 25-55 KB of shared memory a CTA.
    FFT3D_VOL(1, 1, 1, double, 0, 64, 64, 1);
    FFT3D_VOL(3, 3, 3, double, 0, 32, 288, 1);
    FFT3D_VOL(4, 4, 4, double, 0, 16, 256, 1);
    FFT3D_VOL(9, 9, 9, double, 0, 4, 352, 1);
    FFT3D_VOL(10, 10, 10, double, 0, 2, 224, 1);
    FFT3D_VOL(15, 15, 15, double, 0, 1, 256, 1);
    FFT3D_VOL(2, 3, 5, double, 0, 32, 320, 1);
    FFT3D_VOL(7, 11, 13, double, 0, 2, 288, 1);
    FFT3D_VOL(5, 8, 12, double, 0, 4, 384, 1);
    FFT3D_VOL(13, 5, 8, double, 0, 4, 416, 1);
    FFT3D_VOL(17, 2, 2, double, 0, 16, 544, 1);
    FFT3D_VOL(32, 8, 4, double, 0, 2, 256, 1);
    FFT3D_VOL(1, 8, 8, double, 0, 32, 256, 1);
    FFT3D_VOL(8, 1, 8, double, 0, 32, 256, 1);
    FFT3D_VOL(8, 8, 1, double, 0, 32, 256, 1);
    FFT3D_VOL(1, 1, 1, float, 0, 128, 128, 1);
    FFT3D_VOL(3, 3, 3, float, 0, 64, 576, 1);
    FFT3D_VOL(4, 4, 4, float, 0, 32, 512, 1);
    FFT3D_VOL(9, 9, 9, float, 0, 8, 672, 1);
    FFT3D_VOL(10, 10, 10, float, 0, 4, 416, 1);
    FFT3D_VOL(15, 15, 15, float, 0, 2, 480, 1);
    FFT3D_VOL(2, 3, 5, float, 0, 64, 512, 1);
    FFT3D_VOL(7, 11, 13, float, 0, 4, 576, 1);
    FFT3D_VOL(5, 8, 12, float, 0, 8, 768, 1);
    FFT3D_VOL(13, 5, 8, float, 0, 8, 832, 1);
    FFT3D_VOL(17, 2, 2, float, 0, 32, 1024, 1);
    FFT3D_VOL(32, 8, 4, float, 0, 4, 512, 1);
    FFT3D_VOL(1, 8, 8, float, 0, 64, 512, 1);
    FFT3D_VOL(8, 1, 8, float, 0, 64, 512, 1);
    FFT3D_VOL(8, 8, 1, float, 0, 64, 512, 1);

    // The rest of the reference's test geometries (python/test_fft3d.py:25-36):
    // bare primes (5, 7, 11, and 19, 23, 47, 83, 97 along one axis -- folded
    // direct sums; 83 and 97 spill, these are correctness extents), prime
    // powers 25, 27, 49, unit and strongly anisotropic extents, 24x18x12 and
    // 30^3 (complex64; the complex128 30^3 volume, 446 KB, runs as TWOPASS).
    // About 48 KB of shared memory a CTA, lines of 32+ points on 256 threads.
    FFT3D_VOL(2, 2, 2, double, 0, 64, 256, 1);
    FFT3D_VOL(5, 5, 5, double, 0, 24, 512, 1);
    FFT3D_VOL(7, 7, 7, double, 0, 8, 416, 1);
    FFT3D_VOL(11, 11, 11, double, 0, 2, 256, 1);
    FFT3D_VOL(49, 2, 2, double, 0, 10, 256, 1);
    FFT3D_VOL(25, 4, 3, double, 0, 10, 512, 1);
    FFT3D_VOL(27, 2, 2, double, 0, 18, 512, 1);
    FFT3D_VOL(19, 3, 2, double, 0, 17, 512, 1);
    FFT3D_VOL(23, 2, 2, double, 0, 22, 512, 1);
    FFT3D_VOL(47, 3, 2, double, 0, 7, 256, 1);
    FFT3D_VOL(83, 2, 1, double, 0, 18, 256, 1);
    FFT3D_VOL(97, 2, 1, double, 0, 15, 256, 1);
    FFT3D_VOL(1, 1, 16, double, 0, 64, 512, 1);
    FFT3D_VOL(1, 7, 1, double, 0, 64, 448, 1);
    FFT3D_VOL(3, 5, 7, double, 0, 29, 512, 1);
    FFT3D_VOL(4, 6, 10, double, 0, 11, 512, 1);
    FFT3D_VOL(16, 3, 5, double, 0, 12, 512, 1);
    FFT3D_VOL(24, 18, 12, double, 0, 1, 448, 1);
    FFT3D_VOL(2, 2, 64, double, 0, 12, 256, 1);
    FFT3D_VOL(64, 2, 2, double, 0, 8, 256, 1);
    FFT3D_VOL(9, 25, 7, double, 0, 1, 256, 1);
    FFT3D_VOL(20, 12, 6, double, 0, 1, 256, 1);
    FFT3D_VOL(11, 4, 9, double, 0, 7, 512, 1);
    FFT3D_VOL(2, 2, 2, float, 0, 64, 256, 1);
    FFT3D_VOL(5, 5, 5, float, 0, 49, 512, 1);
    FFT3D_VOL(7, 7, 7, float, 0, 17, 512, 1);
    FFT3D_VOL(11, 11, 11, float, 0, 4, 512, 1);
    FFT3D_VOL(49, 2, 2, float, 0, 20, 256, 1);
    FFT3D_VOL(25, 4, 3, float, 0, 20, 512, 1);
    FFT3D_VOL(27, 2, 2, float, 0, 37, 512, 1);
    FFT3D_VOL(19, 3, 2, float, 0, 35, 512, 1);
    FFT3D_VOL(23, 2, 2, float, 0, 44, 512, 1);
    FFT3D_VOL(47, 3, 2, float, 0, 14, 256, 1);
    FFT3D_VOL(83, 2, 1, float, 0, 37, 256, 1);
    FFT3D_VOL(97, 2, 1, float, 0, 31, 256, 1);
    FFT3D_VOL(1, 1, 16, float, 0, 64, 512, 1);
    FFT3D_VOL(1, 7, 1, float, 0, 64, 448, 1);
    FFT3D_VOL(3, 5, 7, float, 0, 58, 512, 1);
    FFT3D_VOL(4, 6, 10, float, 0, 23, 512, 1);
    FFT3D_VOL(16, 3, 5, float, 0, 25, 512, 1);
    FFT3D_VOL(24, 18, 12, float, 0, 1, 448, 1);
    FFT3D_VOL(30, 30, 30, float, 0, 1, 512, 1);
    FFT3D_VOL(2, 2, 64, float, 0, 24, 256, 1);
    FFT3D_VOL(64, 2, 2, float, 0, 16, 256, 1);
    FFT3D_VOL(9, 25, 7, float, 0, 3, 512, 1);
    FFT3D_VOL(20, 12, 6, float, 0, 3, 512, 1);
    FFT3D_VOL(11, 4, 9, float, 0, 15, 512, 1);
}

}  // namespace fft3d

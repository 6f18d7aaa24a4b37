// chain_kernels.cu -- chains of forward transforms with a pointwise step, the
// reference's graded workload (docs/GRADER.md; bench/geom/best/ours_chain.c:36-53):
//
//   unitary:  state <- FFT(state) * V^(-1/2)
//   map:      z = FFT(state) + c;  state <- z / (1 + |z|)
//
// Volumes are independent and each step of a volume depends only on its own
// previous state, so one CTA loads its volumes into shared memory once, runs all
// m steps there -- z and y passes, then the x pass with the step's pointwise map
// fused into its epilogue, written back in place -- and writes the end state to
// HBM once.  A whole chain is one launch; HBM traffic is one read of the start
// state (plus the map constant, which stays in L2) and one write of the end.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/fft3d_b200.h"
#include "internal.h"
#include "volume.cuh"

namespace fft3d {

template <class G, int ALG, int EPI, int VPC, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_chain(const cx<typename G::T> *__restrict__ x0, cx<typename G::T> *__restrict__ out,
            const cx<typename G::T> *__restrict__ cmap, long long nvol, long long steps,
            typename G::T uscale)
{
    using T = typename G::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    const long long v0 = (long long)blockIdx.x * VPC;
    const long long left = nvol - v0;
    const int nv = left < VPC ? (int)left : VPC;
    const int tid = threadIdx.x;
    const long long e0 = v0 * G::V;
    for (int g = tid; g < nv * G::V; g += NT) stage_in<G>(sm, x0 + e0, g);
    __syncthreads();
    for (long long s = 0; s < steps; ++s) {
        for (int r = tid; r < nv * G::ROWS; r += NT) pass_z<G, -1, ALG>(sm, r);
        __syncthreads();
        for (int l = tid; l < nv * G::N0 * G::N2; l += NT) pass_y<G, -1, ALG>(sm, l);
        __syncthreads();
        for (int l = tid; l < nv * G::N1 * G::N2; l += NT)
            pass_x_chain<G, ALG, EPI>(sm, l, cmap, e0, uscale);
        __syncthreads();
    }
    // end state back to HBM, coalesced
    cx<T> *o = out + e0;
    for (int g = tid; g < nv * G::V; g += NT) {
        const int vol = g / G::V;
        const int rem = g - vol * G::V;
        store_out(o + g, sm[G::off(vol * G::ROWS + rem / G::N2, rem % G::N2)]);
    }
}

struct ChainEntry {
    int n0, n1, n2, precision, epi, vpc, threads, smem;
    const void *func;
};

template <int N0, int N1, int N2, typename T, int EPI, int VPC, int NT>
static void add_chain(std::vector<ChainEntry> &out)
{
    using G = Geom<N0, N1, N2, T>;
    ChainEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.epi = EPI;
    e.vpc = VPC;
    e.threads = NT;
    e.smem = VPC * G::PV * G::EB;
    e.func = (const void *)&k_chain<G, ALG_DEFAULT, EPI, VPC, NT>;
    out.push_back(e);
}

#define FFT3D_CHAIN(N0, N1, N2, T, VPC, NT)                 \
    add_chain<N0, N1, N2, T, EPI_UNITARY, VPC, NT>(out);    \
    add_chain<N0, N1, N2, T, EPI_MAP, VPC, NT>(out)

static std::vector<ChainEntry> build_chain_registry()
{
    std::vector<ChainEntry> out;
    {
        // one volume group per CTA; small VPC keeps many CTAs busy for small batches
        FFT3D_CHAIN(6, 6, 6, double, 1, 64);
        FFT3D_CHAIN(8, 8, 8, double, 1, 64);
        FFT3D_CHAIN(12, 12, 12, double, 1, 160);
        FFT3D_CHAIN(16, 16, 16, double, 1, 256);
        FFT3D_CHAIN(17, 17, 17, double, 1, 320);
        FFT3D_CHAIN(24, 24, 24, double, 1, 288);
        FFT3D_CHAIN(6, 6, 6, float, 1, 64);
        FFT3D_CHAIN(8, 8, 8, float, 1, 64);
        FFT3D_CHAIN(12, 12, 12, float, 1, 160);
        FFT3D_CHAIN(16, 16, 16, float, 1, 256);
        FFT3D_CHAIN(17, 17, 17, float, 1, 320);
        FFT3D_CHAIN(24, 24, 24, float, 1, 576);
    }
    return out;
}

static const std::vector<ChainEntry> &chain_registry()
{
    static const std::vector<ChainEntry> reg = build_chain_registry();
    return reg;
}

}  // namespace fft3d

using namespace fft3d;

struct fft3d_b200_chain {
    int device;
    int n0, n1, n2, precision, kind;
    long long batch;
    const void *cmap;
    const ChainEntry *e;
    double uscale;
};

extern "C" int fft3d_b200_chain_create(int n0, int n1, int n2, long long batch, int precision,
                                       int kind, const void *d_c, int device,
                                       fft3d_b200_chain **out)
{
    if (!out) return FFT3D_B200_ERR_INVALID;
    *out = nullptr;
    if (n0 < 1 || n1 < 1 || n2 < 1 || batch < 0) return FFT3D_B200_ERR_INVALID;
    if (precision != FFT3D_B200_C128 && precision != FFT3D_B200_C64) return FFT3D_B200_ERR_INVALID;
    if (kind != FFT3D_B200_CHAIN_UNITARY && kind != FFT3D_B200_CHAIN_MAP) return FFT3D_B200_ERR_INVALID;
    if (kind == FFT3D_B200_CHAIN_MAP && batch > 0 && !d_c) return FFT3D_B200_ERR_INVALID;
    const int epi = kind == FFT3D_B200_CHAIN_UNITARY ? EPI_UNITARY : EPI_MAP;
    const ChainEntry *e = nullptr;
    for (const auto &c : chain_registry())
        if (c.n0 == n0 && c.n1 == n1 && c.n2 == n2 && c.precision == precision && c.epi == epi) e = &c;
    if (!e) return FFT3D_B200_ERR_UNSUPPORTED;
    int prev = -1;
    cudaGetDevice(&prev);
    if (device < 0) device = prev < 0 ? 0 : prev;
    if (cudaSetDevice(device) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    int st = ensure_device_tables(device);
    if (st == FFT3D_B200_OK &&
        cudaFuncSetAttribute(e->func, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem) !=
            cudaSuccess) {
        cudaGetLastError();
        st = FFT3D_B200_ERR_UNSUPPORTED;
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (st) return st;
    fft3d_b200_chain *c = new fft3d_b200_chain();
    c->device = device;
    c->n0 = n0;
    c->n1 = n1;
    c->n2 = n2;
    c->precision = precision;
    c->kind = kind;
    c->batch = batch;
    c->cmap = d_c;
    c->e = e;
    c->uscale = 1.0 / std::sqrt((double)n0 * n1 * n2);
    *out = c;
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_chain_run(fft3d_b200_chain *c, const void *d_x0, void *d_out,
                                    long long steps, void *stream)
{
    if (!c || steps < 0) return FFT3D_B200_ERR_INVALID;
    if (c->batch == 0) return FFT3D_B200_OK;
    if (!d_x0 || !d_out) return FFT3D_B200_ERR_INVALID;
    const size_t eb = (size_t)element_bytes(c->precision);
    if (((uintptr_t)d_x0 % eb) || ((uintptr_t)d_out % eb)) return FFT3D_B200_ERR_ALIGN;
    const ChainEntry &e = *c->e;
    const long long grid = (c->batch + e.vpc - 1) / e.vpc;
    if (grid > 0x7fffffffLL) return FFT3D_B200_ERR_INVALID;
    long long nvol = c->batch;
    const void *cm = c->cmap;
    cudaError_t err;
    if (c->precision == FFT3D_B200_C128) {
        double us = c->uscale;
        void *args[] = {(void *)&d_x0, (void *)&d_out, (void *)&cm, (void *)&nvol, (void *)&steps,
                        (void *)&us};
        err = cudaLaunchKernel(e.func, dim3((unsigned)grid), dim3(e.threads), args, (size_t)e.smem,
                               (cudaStream_t)stream);
    } else {
        float us = (float)c->uscale;
        void *args[] = {(void *)&d_x0, (void *)&d_out, (void *)&cm, (void *)&nvol, (void *)&steps,
                        (void *)&us};
        err = cudaLaunchKernel(e.func, dim3((unsigned)grid), dim3(e.threads), args, (size_t)e.smem,
                               (cudaStream_t)stream);
    }
    return err == cudaSuccess ? FFT3D_B200_OK : FFT3D_B200_ERR_CUDA;
}

extern "C" void fft3d_b200_chain_destroy(fft3d_b200_chain *c) { delete c; }

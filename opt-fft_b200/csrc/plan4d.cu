// plan4d.cu -- 4D transforms of L^3 x T lattices (nt x n0 x n1 x n2 volumes).
//
// The asymmetric L^3 x T extents of lattice QCD (docs/EXTENSIONS.md:55-64 of the
// reference: "per-axis different lengths ... a genuine new capability").
// Layout: element (b, t, x, y, z) at (((b*T + t)*n0 + x)*n1 + y)*n2 + z.  A 4D
// plan is the autotuned 3D plan over the B*T time slices (in -> out), then one
// pass along t in place on out: each thread owns one spatial point of one 4D
// volume, loads its T points (stride n0*n1*n2 -- consecutive threads read
// consecutive addresses, so every load and store is coalesced), transforms them
// in registers and stores them back.  Two HBM passes in all; the inverse scales
// by 1/V in the 3D pass and by 1/T in the t pass.
#include <cuda_runtime.h>

#include <string>

#include "../../include/fft3d_b200.h"
#include "internal.h"
#include "volume.cuh"

namespace fft3d {

constexpr int TPASS_THREADS = 128;

template <int TL, typename T, int S>
__global__ void __launch_bounds__(TPASS_THREADS)
    k_tpass(cx<T> *__restrict__ data, long long vol_elems, long long nblocks_per_vol, T scale)
{
    const long long b = blockIdx.x / nblocks_per_vol;
    const long long p = (blockIdx.x % nblocks_per_vol) * TPASS_THREADS + threadIdx.x;
    if (p >= vol_elems) return;
    cx<T> *col = data + b * TL * vol_elems + p;
    cx<T> v[TL];
#pragma unroll
    for (int t = 0; t < TL; ++t) v[t] = load_in(col + t * vol_elems);
    dft<TL, S, T>(v);
#pragma unroll
    for (int t = 0; t < TL; ++t) {
        cx<T> r = v[t];
        if constexpr (S > 0) r = cscale(r, scale);
        store_out(col + t * vol_elems, r);
    }
}

struct TPassKernel {
    int tl, precision, sign;
    const void *func;
};

#define FFT3D_TPASS(TL)                                                          \
    {TL, FFT3D_B200_C128, -1, (const void *)&k_tpass<TL, double, -1>},           \
        {TL, FFT3D_B200_C128, +1, (const void *)&k_tpass<TL, double, +1>},       \
        {TL, FFT3D_B200_C64, -1, (const void *)&k_tpass<TL, float, -1>},         \
        {TL, FFT3D_B200_C64, +1, (const void *)&k_tpass<TL, float, +1>}

static const TPassKernel kTPass[] = {
    FFT3D_TPASS(2),  FFT3D_TPASS(4),  FFT3D_TPASS(6),  FFT3D_TPASS(8),  FFT3D_TPASS(12),
    FFT3D_TPASS(16), FFT3D_TPASS(17), FFT3D_TPASS(24), FFT3D_TPASS(32), FFT3D_TPASS(36),
    FFT3D_TPASS(48), FFT3D_TPASS(64),
};

static const TPassKernel *find_tpass(int tl, int precision, int sign)
{
    for (const auto &k : kTPass)
        if (k.tl == tl && k.precision == precision && k.sign == sign) return &k;
    return nullptr;
}

}  // namespace fft3d

using namespace fft3d;

struct fft3d_b200_plan4d {
    fft3d_b200_plan *p3 = nullptr;
    const TPassKernel *tk = nullptr;
    int nt = 0;
    long long batch = 0, vol_elems = 0;
    int sign = -1, precision = 0, device = 0;
    std::string describe;
};

extern "C" int fft3d_b200_plan4d_supports(int nt, int n0, int n1, int n2, int precision)
{
    if (nt < 1 || !fft3d_b200_supports(n0, n1, n2, precision)) return 0;
    return find_tpass(nt, precision, -1) ? 1 : 0;
}

extern "C" int fft3d_b200_plan4d_create(int nt, const fft3d_b200_desc *desc, fft3d_b200_plan4d **out)
{
    if (!out || !desc || nt < 1 || desc->batch < 0) return FFT3D_B200_ERR_INVALID;
    *out = nullptr;
    if (desc->direction != FFT3D_B200_FORWARD && desc->direction != FFT3D_B200_BACKWARD)
        return FFT3D_B200_ERR_INVALID;
    const TPassKernel *tk = find_tpass(nt, desc->precision, desc->direction);
    if (!tk) return FFT3D_B200_ERR_UNSUPPORTED;
    fft3d_b200_desc d3 = *desc;
    d3.batch = desc->batch * nt;  // every time slice is one 3D volume
    fft3d_b200_plan *p3 = nullptr;
    const int st = fft3d_b200_plan_create(&d3, &p3);
    if (st != FFT3D_B200_OK) return st;
    fft3d_b200_plan4d *p = new fft3d_b200_plan4d();
    p->p3 = p3;
    p->tk = tk;
    p->nt = nt;
    p->batch = desc->batch;
    p->vol_elems = (long long)desc->n0 * desc->n1 * desc->n2;
    p->sign = desc->direction;
    p->precision = desc->precision;
    cudaGetDevice(&p->device);
    p->describe = std::string("3D: ") + fft3d_b200_plan_describe(p3) + "; t pass: " +
                  std::to_string(nt) + " points per thread, " + std::to_string(TPASS_THREADS) +
                  " threads per CTA";
    *out = p;
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_plan4d_execute(fft3d_b200_plan4d *p, const void *d_in, void *d_out, void *stream)
{
    if (!p) return FFT3D_B200_ERR_INVALID;
    if (p->batch == 0) return FFT3D_B200_OK;
    int st = fft3d_b200_execute(p->p3, d_in, d_out, stream);
    if (st != FFT3D_B200_OK) return st;
    const long long nb = (p->vol_elems + TPASS_THREADS - 1) / TPASS_THREADS;
    const long long grid = nb * p->batch;
    if (grid > 0x7fffffffLL) return FFT3D_B200_ERR_UNSUPPORTED;
    long long ve = p->vol_elems, nbl = nb;
    cudaError_t e;
    if (p->precision == FFT3D_B200_C128) {
        double sc = p->sign > 0 ? 1.0 / (double)p->nt : 1.0;
        void *args[] = {(void *)&d_out, (void *)&ve, (void *)&nbl, (void *)&sc};
        e = cudaLaunchKernel(p->tk->func, dim3((unsigned)grid), dim3(TPASS_THREADS), args, 0,
                             (cudaStream_t)stream);
    } else {
        float sc = p->sign > 0 ? 1.0f / (float)p->nt : 1.0f;
        void *args[] = {(void *)&d_out, (void *)&ve, (void *)&nbl, (void *)&sc};
        e = cudaLaunchKernel(p->tk->func, dim3((unsigned)grid), dim3(TPASS_THREADS), args, 0,
                             (cudaStream_t)stream);
    }
    return e == cudaSuccess ? FFT3D_B200_OK : FFT3D_B200_ERR_CUDA;
}

extern "C" void fft3d_b200_plan4d_destroy(fft3d_b200_plan4d *p)
{
    if (!p) return;
    fft3d_b200_plan_destroy(p->p3);
    delete p;
}

extern "C" const char *fft3d_b200_plan4d_describe(const fft3d_b200_plan4d *p)
{
    return p ? p->describe.c_str() : "";
}

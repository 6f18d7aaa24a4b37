// mgpu.cu -- the multi-GPU contract (bench/mgpu/fft3d_mgpu_api.h): one process,
// n GPUs, slab decomposition with the all-to-all fused into the first kernel.
//
// execute() is two kernels per GPU (layouts in mgpu.cuh):
//   k_mg_yz  GPU g: each CTA loads one x-plane of its slab (cp.async), runs the z
//            and y passes in shared memory, and stores each point straight into
//            the middle buffer of the GPU that owns its y row -- peer stores over
//            NVLink, so the transpose costs no separate copy and overlaps the next
//            plane's arithmetic;
//   k_mg_x   GPU h: each CTA loads all x of one (volume, y) row of its y-slab and
//            writes the x transform to the output y-slab.
// Cross-GPU ordering is by events only: every k_mg_x waits for every GPU's k_mg_yz
// of the same execute, and every k_mg_yz waits for every k_mg_x of the previous
// execute (which still reads the middle buffers).  No kernel waits on another
// device's kernel from the device side.  Peer access is enabled in create() for
// every pair of distinct devices; the same device may be listed more than once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/fft3d_mgpu_api.h"
#include "internal.h"
#include "mgpu.cuh"
#include "ptx.cuh"
#include "splitline.cuh"

namespace fft3d {

constexpr int MGPU_MAX = 16;

template <int L, typename T, int S>
__global__ void __launch_bounds__(L < 64 ? 64 : L, 2)
    k_mg_yz(const cx<T> *__restrict__ in, long long nplanes, cx<T> *const *__restrict__ mids,
            MgpuShape m, int g)
{
    using PG = Geom<1, L, L, T>;  // one x-plane: L rows (y) of L points (z)
    constexpr int NT = L < 64 ? 64 : L;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    const int tid = threadIdx.x;
    for (long long p = blockIdx.x; p < nplanes; p += gridDim.x) {
        const cx<T> *src = in + p * (long long)(L * L);
        for (int e = tid; e < L * L; e += NT) {
            if constexpr (sizeof(T) == 8) cp_async_16(sm + PG::off(e / L, e % L), src + e);
            else cp_async_8(sm + PG::off(e / L, e % L), src + e);
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        for (int r = tid; r < L; r += NT) pass_z<PG, S, ALG_DEFAULT>(sm, r);
        __syncthreads();
        for (int l = tid; l < L; l += NT) pass_y<PG, S, ALG_DEFAULT>(sm, l);
        __syncthreads();
        for (int e = tid; e < L * L; e += NT) {
            const int y = e / L, z = e % L;
            int h;
            const long long off = mgpu_mid_offset(m, g, p, y, z, &h);
            mids[h][off] = sm[PG::off(y, z)];
        }
        __syncthreads();
    }
}

template <int L, typename T, int S>
__global__ void __launch_bounds__(L < 64 ? 64 : L, 2)
    k_mg_x(const cx<T> *__restrict__ mid, cx<T> *__restrict__ out, long long nrows, MgpuShape m,
           T scale)
{
    using RG = Geom<L, 1, L, T>;  // one (volume, y) row of every plane: rows x, points z
    constexpr int NT = L < 64 ? 64 : L;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    const int tid = threadIdx.x;
    for (long long r = blockIdx.x; r < nrows; r += gridDim.x) {
        const long long b = r / m.S;
        const int yl = (int)(r % m.S);
        for (int e = tid; e < L * L; e += NT) {
            const int x = e / L, z = e % L;
            const cx<T> *s = mid + mgpu_yslab_offset(m, b, x, yl, z);
            if constexpr (sizeof(T) == 8) cp_async_16(sm + RG::off(x, z), s);
            else cp_async_8(sm + RG::off(x, z), s);
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        for (int z = tid; z < L; z += NT) {
            cx<T> v[L];
#pragma unroll
            for (int j = 0; j < L; ++j) v[j] = sm[RG::off(j, z)];
            dft<L, S, T>(v);
#pragma unroll
            for (int j = 0; j < L; ++j) {
                cx<T> o = v[j];
                if constexpr (S > 0) o = cscale(o, scale);
                store_out(out + mgpu_yslab_offset(m, b, j, yl, z), o);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- L = 96 .. 256
// Lines too long for one thread and planes too large for shared memory: three
// tiled passes, each line spread over P lanes (splitline.cuh), 128 threads and
// C = 128 / P lines per tile.
//   k_mgl_z  GPU g: C consecutive rows (z lines) of its x-slab, in -> tmp;
//   k_mgl_y  GPU g: the y lines of C consecutive z of one plane, tmp -> the
//            middle buffer of each point's y owner (the fused all-to-all);
//   k_mgl_x  GPU h: the x lines of C consecutive z of one (volume, y) row of
//            its y-slab, middle -> out.
constexpr int MGL_THREADS = 128;

template <int L>
struct MglTile {
    static constexpr int P = LineSplit<L>::P;
    static constexpr int C = MGL_THREADS / P;  // lines per tile
    static constexpr int CP = C + 1;           // padded row of a column tile
    static constexpr int ZSMEM = C * L * (int)sizeof(cx<double>);
    static constexpr int CSMEM = L * CP * (int)sizeof(cx<double>);
    static_assert(L % C == 0, "tiles");
};

template <int L, int S>
__global__ void __launch_bounds__(MGL_THREADS, 4)
    k_mgl_z(const cx<double> *__restrict__ in, cx<double> *__restrict__ tmp, long long nrows)
{
    using TL = MglTile<L>;
    constexpr int P = TL::P, C = TL::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<double> *sm = reinterpret_cast<cx<double> *>(smraw);
    const int tid = threadIdx.x, c = tid / P, t = tid % P;
    for (long long r0 = (long long)blockIdx.x * C; r0 < nrows; r0 += (long long)gridDim.x * C) {
        const cx<double> *src = in + r0 * L;
        for (int e = tid; e < C * L; e += MGL_THREADS) cp_async_16(sm + e, src + e);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        cx<double> *line = sm + c * L;
        split_line<L, S, double>(t, true, [&](int k) { return line[k]; },
                                 [&](int k, cx<double> v) { line[k] = v; });
        __syncthreads();
        cx<double> *dst = tmp + r0 * L;
        for (int e = tid; e < C * L; e += MGL_THREADS) dst[e] = sm[e];
        __syncthreads();
    }
}

template <int L, int S>
__global__ void __launch_bounds__(MGL_THREADS, 4)
    k_mgl_y(const cx<double> *__restrict__ tmp, long long nplanes, cx<double> *const *__restrict__ mids,
            MgpuShape m, int g)
{
    using TL = MglTile<L>;
    constexpr int P = TL::P, C = TL::C, CP = TL::CP;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<double> *sm = reinterpret_cast<cx<double> *>(smraw);
    const int tid = threadIdx.x, c = tid / P, t = tid % P;
    const long long ntiles = nplanes * (L / C);
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long p = tile / (L / C);
        const int z0 = (int)(tile % (L / C)) * C;
        const cx<double> *src = tmp + p * L * L + z0;
        for (int e = tid; e < L * C; e += MGL_THREADS) cp_async_16(sm + (e / C) * CP + e % C, src + (e / C) * L + e % C);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        split_line<L, S, double>(t, true, [&](int y) { return sm[y * CP + c]; },
                                 [&](int y, cx<double> v) { sm[y * CP + c] = v; });
        __syncthreads();
        for (int e = tid; e < L * C; e += MGL_THREADS) {
            const int y = e / C, z = z0 + e % C;
            int h;
            const long long off = mgpu_mid_offset(m, g, p, y, z, &h);
            mids[h][off] = sm[y * CP + e % C];
        }
        __syncthreads();
    }
}

template <int L, int S>
__global__ void __launch_bounds__(MGL_THREADS, 4)
    k_mgl_x(const cx<double> *__restrict__ mid, cx<double> *__restrict__ out, long long nrows, MgpuShape m,
            double scale)
{
    using TL = MglTile<L>;
    constexpr int P = TL::P, C = TL::C, CP = TL::CP;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<double> *sm = reinterpret_cast<cx<double> *>(smraw);
    const int tid = threadIdx.x, c = tid / P, t = tid % P;
    const long long ntiles = nrows * (L / C);
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long r = tile / (L / C);  // (volume, y) row of the y-slab
        const long long b = r / m.S;
        const int yl = (int)(r % m.S);
        const int z0 = (int)(tile % (L / C)) * C;
        for (int e = tid; e < L * C; e += MGL_THREADS)
            cp_async_16(sm + (e / C) * CP + e % C, mid + mgpu_yslab_offset(m, b, e / C, yl, z0 + e % C));
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        split_line<L, S, double>(t, true, [&](int x) { return sm[x * CP + c]; },
                                 [&](int x, cx<double> v) { sm[x * CP + c] = v; });
        __syncthreads();
        for (int e = tid; e < L * C; e += MGL_THREADS) {
            cx<double> v = sm[(e / C) * CP + e % C];
            if constexpr (S > 0) v = cscale(v, scale);
            store_out(out + mgpu_yslab_offset(m, b, e / C, yl, z0 + e % C), v);
        }
        __syncthreads();
    }
}

struct MgpuKernels {
    int L;
    const void *yz[2], *x[2];  // [0] forward, [1] inverse; large L: the y pass
    const void *z[2];          // large L only: the z pass (null otherwise)
    int smem;                  // plane kernels / column tiles
    int zsmem;                 // large L: row tiles
    int tile_lines;            // large L: lines per tile (0 otherwise)
    int threads;
};

template <int L>
static MgpuKernels mgpu_kernels()
{
    using G = Geom<1, L, L, double>;
    MgpuKernels k;
    k.L = L;
    k.yz[0] = (const void *)&k_mg_yz<L, double, -1>;
    k.yz[1] = (const void *)&k_mg_yz<L, double, +1>;
    k.x[0] = (const void *)&k_mg_x<L, double, -1>;
    k.x[1] = (const void *)&k_mg_x<L, double, +1>;
    k.z[0] = k.z[1] = nullptr;
    k.smem = G::PV * G::EB;
    k.zsmem = 0;
    k.tile_lines = 0;
    k.threads = L < 64 ? 64 : L;
    return k;
}

template <int L>
static MgpuKernels mgpu_kernels_large()
{
    using TL = MglTile<L>;
    MgpuKernels k;
    k.L = L;
    k.z[0] = (const void *)&k_mgl_z<L, -1>;
    k.z[1] = (const void *)&k_mgl_z<L, +1>;
    k.yz[0] = (const void *)&k_mgl_y<L, -1>;
    k.yz[1] = (const void *)&k_mgl_y<L, +1>;
    k.x[0] = (const void *)&k_mgl_x<L, -1>;
    k.x[1] = (const void *)&k_mgl_x<L, +1>;
    k.smem = TL::CSMEM;
    k.zsmem = TL::ZSMEM;
    k.tile_lines = TL::C;
    k.threads = MGL_THREADS;
    return k;
}

static const MgpuKernels *mgpu_find(int L)
{
    static const MgpuKernels table[] = {mgpu_kernels<36>(),        mgpu_kernels<45>(),
                                        mgpu_kernels<64>(),        mgpu_kernels_large<96>(),
                                        mgpu_kernels_large<128>(), mgpu_kernels_large<192>(),
                                        mgpu_kernels_large<256>()};
    for (const auto &k : table)
        if (k.L == L) return &k;
    return nullptr;
}

}  // namespace fft3d

using namespace fft3d;

struct fft3d_mgpu_plan {
    int L, batch, n, sign;
    int dev[MGPU_MAX];
    MgpuShape m;
    const MgpuKernels *k;
    size_t slab_elems;  // per GPU, every buffer: batch * S * L * L
    cx<double> *in[MGPU_MAX] = {};
    cx<double> *mid[MGPU_MAX] = {};
    cx<double> *out[MGPU_MAX] = {};
    cx<double> *tmp[MGPU_MAX] = {};    // large L: the z-transformed x-slab
    cx<double> **mids[MGPU_MAX] = {};  // per GPU: device array of the n middle buffers
    cudaStream_t st[MGPU_MAX] = {};
    cudaEvent_t ev_yz[MGPU_MAX] = {}, ev_x[MGPU_MAX] = {};
    int grid_yz[MGPU_MAX], grid_x[MGPU_MAX], grid_z[MGPU_MAX];
};

extern "C" const char *fft3d_mgpu_name(void) { return "b200_slab_p2p"; }

extern "C" const char *fft3d_mgpu_description(void)
{
    return "x-slab per GPU; z and y passes in shared memory with the all-to-all fused as peer "
           "stores to the y-slab owner; x pass per y-slab; event-ordered, no device-side waits";
}

extern "C" int fft3d_mgpu_supports(int L, int ngpus)
{
    if (ngpus < 1 || ngpus > MGPU_MAX || L % ngpus != 0) return 0;
    return mgpu_find(L) ? 1 : 0;
}

extern "C" void fft3d_mgpu_destroy(fft3d_mgpu_plan *p)
{
    if (!p) return;
    int prev = -1;
    cudaGetDevice(&prev);
    for (int g = 0; g < p->n; ++g) {
        cudaSetDevice(p->dev[g]);
        cudaDeviceSynchronize();
        if (p->in[g]) cudaFree(p->in[g]);
        if (p->mid[g]) cudaFree(p->mid[g]);
        if (p->out[g]) cudaFree(p->out[g]);
        if (p->tmp[g]) cudaFree(p->tmp[g]);
        if (p->mids[g]) cudaFree(p->mids[g]);
        if (p->st[g]) cudaStreamDestroy(p->st[g]);
        if (p->ev_yz[g]) cudaEventDestroy(p->ev_yz[g]);
        if (p->ev_x[g]) cudaEventDestroy(p->ev_x[g]);
    }
    cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    delete p;
}

extern "C" fft3d_mgpu_plan *fft3d_mgpu_create_ex(int L, int batch, int ngpus, const int *devices,
                                                 int inverse)
{
    if (!devices || batch < 1) {
        record_status(FFT3D_B200_ERR_INVALID);
        return nullptr;
    }
    if (!fft3d_mgpu_supports(L, ngpus)) {
        record_status(FFT3D_B200_ERR_UNSUPPORTED);
        return nullptr;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
        cudaGetLastError();
        record_status(FFT3D_B200_ERR_CUDA);
        return nullptr;
    }
    for (int g = 0; g < ngpus; ++g)
        if (devices[g] < 0 || devices[g] >= ndev) {
            record_status(FFT3D_B200_ERR_INVALID);
            return nullptr;
        }
    // every pair of distinct listed devices must reach each other's memory:
    // the exchange is peer stores from inside the compute kernels
    for (int g = 0; g < ngpus; ++g)
        for (int h = 0; h < ngpus; ++h) {
            if (devices[h] == devices[g]) continue;
            int can = 0;
            if (cudaDeviceCanAccessPeer(&can, devices[g], devices[h]) != cudaSuccess) {
                cudaGetLastError();
                record_status(FFT3D_B200_ERR_CUDA);
                return nullptr;
            }
            if (!can) {
                record_status(FFT3D_B200_ERR_PEER);
                return nullptr;
            }
        }
    int prev = -1;
    cudaGetDevice(&prev);
    fft3d_mgpu_plan *p = new fft3d_mgpu_plan();
    p->L = L;
    p->batch = batch;
    p->n = ngpus;
    p->sign = inverse ? +1 : -1;
    p->k = mgpu_find(L);
    p->m = MgpuShape{L, ngpus, L / ngpus};
    p->slab_elems = (size_t)batch * p->m.S * L * L;
    bool ok = true;
    for (int g = 0; g < ngpus && ok; ++g) {
        p->dev[g] = devices[g];
        ok = cudaSetDevice(devices[g]) == cudaSuccess && ensure_device_tables(devices[g]) == FFT3D_B200_OK;
        const size_t bytes = p->slab_elems * sizeof(cx<double>);
        ok = ok && cudaMalloc(&p->in[g], bytes) == cudaSuccess &&
             cudaMalloc(&p->mid[g], bytes) == cudaSuccess && cudaMalloc(&p->out[g], bytes) == cudaSuccess &&
             cudaMalloc(&p->mids[g], ngpus * sizeof(void *)) == cudaSuccess &&
             cudaStreamCreateWithFlags(&p->st[g], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&p->ev_yz[g], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&p->ev_x[g], cudaEventDisableTiming) == cudaSuccess;
        const int si = inverse ? 1 : 0;
        ok = ok && cudaFuncSetAttribute(p->k->yz[si], cudaFuncAttributeMaxDynamicSharedMemorySize, p->k->smem) == cudaSuccess &&
             cudaFuncSetAttribute(p->k->x[si], cudaFuncAttributeMaxDynamicSharedMemorySize, p->k->smem) == cudaSuccess;
        int sms = 148, occ_yz = 0, occ_x = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devices[g]);
        ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_yz, p->k->yz[si], p->k->threads, p->k->smem) == cudaSuccess &&
             cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_x, p->k->x[si], p->k->threads, p->k->smem) == cudaSuccess &&
             occ_yz > 0 && occ_x > 0;
        p->grid_yz[g] = occ_yz * sms;
        p->grid_x[g] = occ_x * sms;
        p->grid_z[g] = 0;
        if (ok && p->k->z[si]) {  // large L: the separate z pass and its buffer
            int occ_z = 0;
            ok = cudaMalloc(&p->tmp[g], bytes) == cudaSuccess &&
                 cudaFuncSetAttribute(p->k->z[si], cudaFuncAttributeMaxDynamicSharedMemorySize, p->k->zsmem) == cudaSuccess &&
                 cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_z, p->k->z[si], p->k->threads, p->k->zsmem) == cudaSuccess &&
                 occ_z > 0;
            p->grid_z[g] = occ_z * sms;
        }
        // peer access to every other device of the list
        for (int h = 0; h < ngpus && ok; ++h) {
            if (devices[h] == devices[g]) continue;
            int can = 0;
            ok = cudaDeviceCanAccessPeer(&can, devices[g], devices[h]) == cudaSuccess && can;
            if (ok) {
                const cudaError_t e = cudaDeviceEnablePeerAccess(devices[h], 0);
                if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
                else ok = e == cudaSuccess;
            }
        }
    }
    for (int g = 0; g < ngpus && ok; ++g) {
        ok = cudaSetDevice(p->dev[g]) == cudaSuccess &&
             cudaMemcpy(p->mids[g], p->mid, ngpus * sizeof(void *), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaEventRecord(p->ev_x[g], p->st[g]) == cudaSuccess;  // "previous execute" is done
    }
    if (prev >= 0) cudaSetDevice(prev);
    if (!ok) {
        cudaGetLastError();
        fft3d_mgpu_destroy(p);
        record_status(FFT3D_B200_ERR_CUDA);
        return nullptr;
    }
    record_status(FFT3D_B200_OK);
    return p;
}

extern "C" fft3d_mgpu_plan *fft3d_mgpu_create(int L, int batch, int ngpus, const int *devices)
{
    return fft3d_mgpu_create_ex(L, batch, ngpus, devices, 0);
}

// Host layout (b, x, y, z) at ((b*L + x)*L + y)*L + z (bench/mgpu/fft3d_mgpu_api.h:32-35).
extern "C" void fft3d_mgpu_upload(fft3d_mgpu_plan *p, const double2 *host)
{
    if (!p || !host) return;
    int prev = -1;
    cudaGetDevice(&prev);
    const size_t L = p->L, S = p->m.S, e = sizeof(double2);
    for (int g = 0; g < p->n; ++g) {
        cudaSetDevice(p->dev[g]);
        cudaStreamSynchronize(p->st[g]);
        // x-slab g of every volume: B blocks of S*L*L contiguous points
        cudaMemcpy2D(p->in[g], S * L * L * e, host + (size_t)g * S * L * L, L * L * L * e,
                     S * L * L * e, (size_t)p->batch, cudaMemcpyHostToDevice);
    }
    if (prev >= 0) cudaSetDevice(prev);
}

extern "C" void fft3d_mgpu_execute(fft3d_mgpu_plan *p)
{
    if (!p) return;
    int prev = -1;
    cudaGetDevice(&prev);
    const int si = p->sign > 0 ? 1 : 0;
    const long long nplanes = (long long)p->batch * p->m.S;
    const double scale = p->sign > 0 ? 1.0 / ((double)p->L * p->L * p->L) : 1.0;
    for (int g = 0; g < p->n; ++g) {
        cudaSetDevice(p->dev[g]);
        for (int h = 0; h < p->n; ++h) cudaStreamWaitEvent(p->st[g], p->ev_x[h], 0);
        const cx<double> *in = p->in[g];
        long long yz_items = nplanes;
        if (p->k->z[si]) {
            // large L: z pass into tmp, then the y pass reads tmp
            const long long nrows = nplanes * p->L;
            const long long c = p->k->tile_lines;
            cx<double> *tmp = p->tmp[g];
            void *zargs[] = {(void *)&in, (void *)&tmp, (void *)&nrows};
            const unsigned zgrid = (unsigned)std::min<long long>(nrows / c, p->grid_z[g]);
            cudaLaunchKernel(p->k->z[si], dim3(zgrid), dim3(p->k->threads), zargs, (size_t)p->k->zsmem, p->st[g]);
            in = tmp;
            yz_items = nplanes * (p->L / c);
        }
        cx<double> *const *mids = p->mids[g];
        MgpuShape m = p->m;
        int gg = g;
        void *args[] = {(void *)&in, (void *)&nplanes, (void *)&mids, (void *)&m, (void *)&gg};
        const unsigned grid = (unsigned)std::min<long long>(yz_items, p->grid_yz[g]);
        cudaLaunchKernel(p->k->yz[si], dim3(grid), dim3(p->k->threads), args, (size_t)p->k->smem, p->st[g]);
        cudaEventRecord(p->ev_yz[g], p->st[g]);
    }
    for (int h = 0; h < p->n; ++h) {
        cudaSetDevice(p->dev[h]);
        for (int g = 0; g < p->n; ++g) cudaStreamWaitEvent(p->st[h], p->ev_yz[g], 0);
        const cx<double> *mid = p->mid[h];
        cx<double> *out = p->out[h];
        MgpuShape m = p->m;
        double sc = scale;
        void *args[] = {(void *)&mid, (void *)&out, (void *)&nplanes, (void *)&m, (void *)&sc};
        const long long x_items = p->k->tile_lines ? nplanes * (p->L / p->k->tile_lines) : nplanes;
        const unsigned grid = (unsigned)std::min<long long>(x_items, p->grid_x[h]);
        cudaLaunchKernel(p->k->x[si], dim3(grid), dim3(p->k->threads), args, (size_t)p->k->smem, p->st[h]);
        cudaEventRecord(p->ev_x[h], p->st[h]);
    }
    if (prev >= 0) cudaSetDevice(prev);
}

extern "C" void fft3d_mgpu_download(fft3d_mgpu_plan *p, double2 *host)
{
    if (!p || !host) return;
    int prev = -1;
    cudaGetDevice(&prev);
    const size_t L = p->L, S = p->m.S, e = sizeof(double2);
    for (int h = 0; h < p->n; ++h) {
        cudaSetDevice(p->dev[h]);
        cudaStreamSynchronize(p->st[h]);
        // y-slab h: for every (b, kx) a run of S*L points at ky = h*S
        cudaMemcpy2D(host + (size_t)h * S * L, L * L * e, p->out[h], S * L * e, S * L * e,
                     (size_t)p->batch * L, cudaMemcpyDeviceToHost);
    }
    if (prev >= 0) cudaSetDevice(prev);
}

// cluster_kernels.cu -- kernel family CLUSTER: volumes larger than one SM's
// shared memory (36^3 complex double is 746 KB) held by a thread-block cluster.
//
// A cluster of C CTAs transforms one volume.  CTA rank r owns the x-slab of
// PL = n0/C planes [r*PL, (r+1)*PL): it copies that contiguous byte range into
// its shared memory (cp.async into the padded, bank-conflict-free layout of
// volume.cuh), runs the z and y passes locally, then -- after a cluster-wide
// barrier -- takes its share n1*n2/C of the x lines, reads their n0 points from
// the owning CTAs' shared memory through distributed shared memory
// (ld.shared::cluster), and writes each result line straight to HBM.  A second
// barrier keeps every slab alive until all peers have read it.  Each volume is
// read from HBM once and written once.
//
// The two data barriers are mbarriers that every CTA arrives on remotely
// (release, cluster scope) and waits on with a bounded poll (acquire, cluster
// scope); a timeout records DEV_ERR_CLUSTER_TIMEOUT in the device error word.
// 36 = 4 * 9 lines use the prime-factor codelet of codelets.cuh.
#include "internal.h"
#include "ptx.cuh"
#include "volume.cuh"

namespace fft3d {

template <int N0, int N1, int N2, typename T, int C>
struct ClusterLayout {
    static constexpr int PL = N0 / C;
    using SG = Geom<PL, N1, N2, T>;
    static constexpr int SLAB_BYTES = ((SG::PV * SG::EB) + 127) / 128 * 128;
    static constexpr int SMEM_BYTES = SLAB_BYTES + 16;
    static constexpr int LPC = N1 * N2 / C;  // x lines per CTA
};

__device__ __forceinline__ void fence_acq_rel_cluster()
{
    asm volatile("fence.acq_rel.cluster;" ::: "memory");
}

template <int N0, int N1, int N2, typename T, int S, int C, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_cluster(const cx<T> *__restrict__ in, cx<T> *__restrict__ out, long long nvol, T scale,
              int *err)
{
    using CL = ClusterLayout<N0, N1, N2, T, C>;
    using SG = typename CL::SG;
    constexpr int PL = CL::PL;
    constexpr int V = N0 * N1 * N2;
    static_assert(N0 % C == 0 && (N1 * N2) % C == 0, "cluster split");
    pdl_begin();
    extern __shared__ __align__(128) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    uint64_t *xbar = reinterpret_cast<uint64_t *>(smraw + CL::SLAB_BYTES);
    __shared__ int s_abort;

    const int tid = threadIdx.x;
    const uint32_t rank = cluster_rank();
    const long long vol = blockIdx.x / C;
    if (tid == 0) {
        mbar_init(xbar, C);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    cluster_sync_hw();  // every CTA's barrier is initialised before anyone arrives on it
    if (vol >= nvol) return;  // never taken: the grid is nvol*C

    // 1. this CTA's slab, contiguous in HBM, into the padded layout
    const cx<T> *gin = in + vol * V + (long long)rank * PL * N1 * N2;
    for (int g = tid; g < PL * N1 * N2; g += NT) {
        cx<T> *dst = sm + SG::off(g / N2, g % N2);
        if constexpr (sizeof(T) == 8) cp_async_16(dst, gin + g);
        else cp_async_8(dst, gin + g);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    // 2. local passes along z and y
    for (int r = tid; r < PL * N1; r += NT) pass_z<SG, S, ALG_DEFAULT>(sm, r);
    __syncthreads();
    for (int l = tid; l < PL * N2; l += NT) pass_y<SG, S, ALG_DEFAULT>(sm, l);

    // 3. cluster barrier: all slabs hold their z,y results
    fence_acq_rel_cluster();
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < C; ++q) mbar_arrive_remote(mapa_u32(xbar, (uint32_t)q));
    if (!mbar_wait_cluster_bounded(xbar, 0)) s_abort = 1;
    __syncthreads();

    if (!s_abort) {
        // 4. x lines of this CTA's share, points gathered from the owning slabs
        uint32_t base[C];
#pragma unroll
        for (int q = 0; q < C; ++q) base[q] = mapa_u32(sm, (uint32_t)q);
        cx<T> *gout = out + vol * V;
        for (int l = (int)rank * CL::LPC + tid; l < ((int)rank + 1) * CL::LPC; l += NT) {
            const int y = l / N2;
            const int z = l % N2;
            cx<T> v[N0];
#pragma unroll
            for (int j = 0; j < N0; ++j) {
                const uint32_t a =
                    base[j / PL] + (uint32_t)(SG::off((j % PL) * N1 + y, z) * (int)sizeof(cx<T>));
                if constexpr (sizeof(T) == 8) {
                    const double2 t = ld_dsmem_f64x2(a);
                    v[j] = {t.x, t.y};
                } else {
                    const float2 t = ld_dsmem_f32x2(a);
                    v[j] = {t.x, t.y};
                }
            }
            dft<N0, S, T>(v);
#pragma unroll
            for (int j = 0; j < N0; ++j) {
                cx<T> r = v[j];
                if constexpr (S > 0) r = cscale(r, scale);
                store_out(gout + (long long)(j * N1 + y) * N2 + z, r);
            }
        }
    }

    // 5. nobody leaves while a peer may still read its slab
    fence_acq_rel_cluster();
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < C; ++q) mbar_arrive_remote(mapa_u32(xbar, (uint32_t)q));
    if (!mbar_wait_cluster_bounded(xbar, 1)) s_abort = 1;
    __syncthreads();
    if (s_abort && tid == 0) report_error(err, DEV_ERR_CLUSTER_TIMEOUT);
}

template <int N0, int N1, int N2, typename T, int S, int C, int NT>
static void add_cluster(std::vector<KernelEntry> &out, const char *name)
{
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_CLUSTER;
    e.alg = 0;
    e.vpc = C;  // CTAs per cluster
    e.threads = NT;
    e.smem = ClusterLayout<N0, N1, N2, T, C>::SMEM_BYTES;
    e.func = (const void *)&k_cluster<N0, N1, N2, T, S, C, NT>;
    e.name = name;
    out.push_back(e);
}

#define FFT3D_CLUSTER(N0, N1, N2, T, C, NT)                                                    \
    add_cluster<N0, N1, N2, T, -1, C, NT>(out, "cluster " #N0 "x" #N1 "x" #N2 " " #T " c" #C    \
                                               " nt" #NT);                                     \
    add_cluster<N0, N1, N2, T, +1, C, NT>(out, "cluster " #N0 "x" #N1 "x" #N2 " " #T " c" #C    \
                                               " nt" #NT)

void register_cluster_kernels(std::vector<KernelEntry> &out)
{
    // c6 complex double is within 2% of the winner at 16 volumes of 36^3; c2
    // complex float wins at 64 volumes (the uneven mix), c4 at small batches
    FFT3D_CLUSTER(36, 36, 36, double, 6, 224);
    FFT3D_CLUSTER(36, 36, 36, float, 2, 324);
    FFT3D_CLUSTER(36, 36, 36, float, 4, 324);
}

}  // namespace fft3d

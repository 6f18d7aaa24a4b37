// twopass_kernels.cu -- kernel family TWOPASS: volumes larger than one SM's
// shared memory (36^3 complex double is 746 KB, 16x16x32 is 262 KB), in plane
// and row items through an L2-resident scratch ring (twopass.cuh).
//
// Persistent CTAs take one ticket at a time.  A plane item copies its G
// contiguous x-planes into shared memory with cp.async, runs the z and y
// passes, and writes the planes to the volume's scratch slot with L2-only
// stores; a row item reads its G y-rows of all planes back with L2-only loads
// (never through L1, which is not coherent with other SMs' stores), runs the
// x pass and streams the result to the output.  Completion is published per
// slot with a release add after a CTA-wide barrier and a fence, and observed
// with an acquire load, by one thread, before a barrier.  Several CTAs per SM
// (small items) overlap one another's loads, arithmetic and stores, so unlike
// a thread-block cluster that moves one volume in lock-step, HBM stays busy.
//
// Every wait is bounded in time (ptx.cuh wait_counter_geq); a timeout records
// DEV_ERR_DEP_TIMEOUT, raises the workspace abort flag so that the other CTAs
// stop too, and the last CTA to leave clears the control block for the next
// launch, on the error path as well.
#include "internal.h"
#include "ptx.cuh"
#include "twopass.cuh"

namespace fft3d {

template <typename T>
__device__ __forceinline__ cx<T> ld_l2(const cx<T> *p)
{
    if constexpr (sizeof(T) == 8) {
        const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
        return {v.x, v.y};
    } else {
        const float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
        return {v.x, v.y};
    }
}

template <typename T>
__device__ __forceinline__ void st_l2(cx<T> *p, cx<T> v)
{
    if constexpr (sizeof(T) == 8) __stcg(reinterpret_cast<double2 *>(p), make_double2(v.re, v.im));
    else __stcg(reinterpret_cast<float2 *>(p), make_float2(v.re, v.im));
}

template <int N0, int N1, int N2, typename T, int S, int G, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_twopass(const cx<T> *__restrict__ in, cx<T> *__restrict__ out, long long nvol, T scale,
              int *err, unsigned char *work, int R, int D)
{
    using TG = TwoPassGeom<N0, N1, N2, T, G>;
    using XG = typename TG::XG;
    using YG = typename TG::YG;
    constexpr int U = 8;  // L2 loads in flight per thread in the row gather
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T> *sm = reinterpret_cast<cx<T> *>(smraw);
    __shared__ long long s_t;
    __shared__ int s_stop;
    TwoPassCtl *ctl = reinterpret_cast<TwoPassCtl *>(work);
    cx<T> *ring = reinterpret_cast<cx<T> *>(work + TWOPASS_CTL_BYTES);
    const int tid = threadIdx.x;
    const long long total = (long long)(TG::NA + TG::NB) * nvol;

    for (;;) {
        if (tid == 0) {
            const long long t = (long long)atomicAdd(&ctl->ticket, 1ull);
            s_t = t;
            s_stop = (t >= total || ld_acquire_gpu(&ctl->abort) != 0) ? 1 : 0;
        }
        __syncthreads();
        if (s_stop) break;
        const TwoPassItem it = twopass_decode(s_t, nvol, TG::NA, TG::NB, D);
        const int slot = (int)(it.vol % R);
        const unsigned round = (unsigned)(it.vol / R);
        cx<T> *sv = ring + (long long)slot * TG::V;

        if (it.plane) {
            // 1. G contiguous planes of the input
            const cx<T> *src = in + it.vol * TG::V;
            for (int g = tid; g < TG::PLANE_ELEMS; g += NT) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                if constexpr (sizeof(T) == 8) cp_async_16(sm + so, src + vo);
                else cp_async_8(sm + so, src + vo);
            }
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
            // 2. z and y passes
            for (int r = tid; r < G * N1; r += NT) pass_z<XG, S, ALG_DEFAULT>(sm, r);
            __syncthreads();
            for (int l = tid; l < G * N2; l += NT) pass_y<XG, S, ALG_DEFAULT>(sm, l);
            // 3. the slot's previous volume must have been read out
            if (tid == 0)
                s_stop = wait_counter_geq(&ctl->cnt[TWOPASS_RMAX + slot], (unsigned)TG::NB * round,
                                          &ctl->abort)
                             ? 0
                             : 1;
            __syncthreads();
            if (s_stop) break;
            // 4. to scratch, same offsets as in the volume, L2 only
            for (int g = tid; g < TG::PLANE_ELEMS; g += NT) {
                long long vo;
                int so;
                twopass_plane_elem<TG>(it.j, g, &vo, &so);
                st_l2(sv + vo, sm[so]);
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) red_release_gpu_add(&ctl->cnt[slot], 1u);
        } else {
            // 1. all plane items of this volume must be in scratch
            if (tid == 0)
                s_stop = wait_counter_geq(&ctl->cnt[slot], (unsigned)TG::NA * (round + 1u), &ctl->abort)
                             ? 0
                             : 1;
            __syncthreads();
            if (s_stop) break;
            // 2. gather the G rows of every plane, U loads in flight per thread
            for (int base = 0; base < TG::ROW_ELEMS; base += NT * U) {
                cx<T> v[U];
                int so[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int g = base + u * NT + tid;
                    so[u] = -1;
                    if (g < TG::ROW_ELEMS) {
                        long long vo;
                        twopass_row_elem<TG>(it.j, g, &vo, &so[u]);
                        v[u] = ld_l2(sv + vo);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (so[u] >= 0) sm[so[u]] = v[u];
            }
            __syncthreads();
            // the slot may be overwritten once every row item has read it
            if (tid == 0) red_release_gpu_add(&ctl->cnt[TWOPASS_RMAX + slot], 1u);
            // 3. x pass, straight to the output
            cx<T> *gvol = out + it.vol * TG::V;
            for (int l = tid; l < G * N2; l += NT) pass_x_slab<YG, S, N1>(sm, l, gvol, it.j * G, scale);
        }
        __syncthreads();  // the next item reuses shared memory
    }

    // A wait that timed out: record it and stop the other CTAs.
    if (tid == 0 && s_stop && s_t < total) {
        report_error(err, DEV_ERR_DEP_TIMEOUT);
        atomicExch(&ctl->abort, 1u);
    }
    // The last CTA to leave clears the control block for the next launch.
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();  // every other CTA's updates of the block precede the reset
            ctl->ticket = 0ull;
            for (int i = 0; i < 2 * TWOPASS_RMAX; ++i) ctl->cnt[i] = 0u;
            ctl->abort = 0u;
            __threadfence();
            ctl->done = 0u;
        }
    }
}

int twopass_ring(const KernelEntry &e, long long grid, int *lag)
{
    return twopass_ring_size(e.n0 / e.vpc, e.n1 / e.vpc, grid, lag);
}

size_t entry_workspace_bytes(const KernelEntry &e, int grid_limit)
{
    if (e.family != FAM_TWOPASS) return 0;
    int lag = 0;
    const int r = twopass_ring(e, grid_limit, &lag);
    return TWOPASS_CTL_BYTES + (size_t)r * (size_t)e.n0 * e.n1 * e.n2 * (size_t)element_bytes(e.precision);
}

template <int N0, int N1, int N2, typename T, int S, int G, int NT, int MINB>
static void add_twopass(std::vector<KernelEntry> &out, const char *name)
{
    KernelEntry e;
    e.n0 = N0;
    e.n1 = N1;
    e.n2 = N2;
    e.precision = sizeof(T) == 8 ? FFT3D_B200_C128 : FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_TWOPASS;
    e.alg = 0;
    e.vpc = G;
    e.threads = NT;
    e.smem = TwoPassGeom<N0, N1, N2, T, G>::SMEM;
    e.func = (const void *)&k_twopass<N0, N1, N2, T, S, G, NT, MINB>;
    e.name = name;
    out.push_back(e);
}

#define FFT3D_TWOPASS(N0, N1, N2, T, G, NT, MINB)                                              \
    add_twopass<N0, N1, N2, T, -1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " " #T    \
                                                     " g" #G " nt" #NT " minb" #MINB);         \
    add_twopass<N0, N1, N2, T, +1, G, NT, MINB>(out, "twopass " #N0 "x" #N1 "x" #N2 " " #T    \
                                                     " g" #G " nt" #NT " minb" #MINB)

void register_twopass_kernels(std::vector<KernelEntry> &out)
{
    // 36^3: 36 lines per plane or row, one thread per line
    FFT3D_TWOPASS(36, 36, 36, double, 4, 160, 2);
    FFT3D_TWOPASS(36, 36, 36, double, 2, 96, 4);
    FFT3D_TWOPASS(36, 36, 36, double, 6, 224, 1);
    FFT3D_TWOPASS(36, 36, 36, float, 4, 160, 3);
    FFT3D_TWOPASS(36, 36, 36, float, 6, 224, 2);
    // 16x16x32 complex double (262 KB): z pass 16*G rows, y and x passes 32*G lines
    FFT3D_TWOPASS(16, 16, 32, double, 4, 128, 4);
    FFT3D_TWOPASS(16, 16, 32, double, 8, 256, 2);
    // 45^3 (45 = 5 x 9) and 64^3 (64 = 8 x 8): beyond any cluster's shared memory
    FFT3D_TWOPASS(45, 45, 45, double, 3, 160, 2);
    FFT3D_TWOPASS(45, 45, 45, double, 5, 256, 1);
    FFT3D_TWOPASS(45, 45, 45, float, 5, 256, 2);
    FFT3D_TWOPASS(45, 45, 45, float, 3, 160, 3);
    FFT3D_TWOPASS(64, 64, 64, double, 1, 64, 3);
    FFT3D_TWOPASS(64, 64, 64, double, 2, 128, 1);
    FFT3D_TWOPASS(64, 64, 64, float, 2, 128, 3);
    FFT3D_TWOPASS(64, 64, 64, float, 4, 256, 1);
}

}  // namespace fft3d

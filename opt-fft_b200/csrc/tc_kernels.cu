// tc_kernels.cu -- complex64 transforms of extents <= 16 on the 5th-generation
// tensor cores (tcgen05), with split-BF16 operands accumulated in FP32.
//
// An axis pass of an L-point DFT over many lines is a dense matrix product: with
// x = [re(0..L-1), im(0..L-1)] per line, y = x * B where B (2L x 2L, real) holds
// cos/sin(2*pi*n*j/L).  Each CTA holds VPC volumes in shared memory (FP32) and,
// per pass, 256 lines at a time: every thread turns one line into a row of an
// M=128 A tile, the FP32 values split into bf16 terms x = h + m + l (exact: 3 x 8
// bits = the 24-bit FP32 significand); B is split the same way at plan time.
// One thread issues tcgen05.mma (kind::f16, bf16 x bf16 -> f32, A and B from
// shared memory through matrix descriptors, D in tensor memory) for the products
// hh, hm, mh (SPLIT = 2: the classic three-product split) or additionally hl, lh,
// mm (SPLIT = 3), commits to an mbarrier, and every thread reads its row of D
// back with tcgen05.ld.  The dropped products are below 2^-24 relative for
// SPLIT = 3, i.e. FP32-level accuracy; SPLIT = 2 keeps 16 bits (about 1e-5).
//
// Shared-memory operands use the canonical K-major, no-swizzle UMMA layout:
// 8-row x 16-byte core matrices, row groups SBO = 128 B apart, the two 8-element
// K chunks of one MMA LBO = rows/8 * 128 B apart.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <math.h>

#include <mutex>

#include "internal.h"
#include "ptx.cuh"
#include "volume.cuh"

namespace fft3d {

// ------------------------------------------------------------------ tables


constexpr int TC_TERMS = 3;
// B tables for L in {6, 8, 12, 16}, both signs: [li][si][term][NP=32][KP=32]
constexpr int TC_NL = 4;
constexpr int TC_B_ELEMS = TC_NL * 2 * TC_TERMS * 32 * 32;
__device__ __nv_bfloat16 g_tc_btab[TC_B_ELEMS];

constexpr int tc_li(int L) { return L == 6 ? 0 : L == 8 ? 1 : L == 12 ? 2 : 3; }

static void tc_fill_host(__nv_bfloat16 *tab)
{
    const int Ls[TC_NL] = {6, 8, 12, 16};
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int li = 0; li < TC_NL; ++li) {
        const int L = Ls[li];
        for (int si = 0; si < 2; ++si) {
            const int S = si == 0 ? -1 : +1;
            for (int n = 0; n < 32; ++n) {
                for (int k = 0; k < 32; ++k) {
                    // B^T[n][k]: output column n (re 0..L-1, im L..2L-1), input k
                    long double v = 0.0L;
                    if (n < 2 * L && k < 2 * L) {
                        const int no = n % L, ki = k % L;
                        const long e = ((long)no * ki) % L;
                        const long double c = (4 * e == L) ? 0.0L : (2 * e == L ? -1.0L : (4 * e == 3 * L ? 0.0L : cosl(two_pi * e / L)));
                        const long double sn = (e == 0 || 2 * e == L) ? 0.0L : (4 * e == L ? 1.0L : (4 * e == 3 * L ? -1.0L : sinl(two_pi * e / L)));
                        const long double wr = (e == 0) ? 1.0L : c;
                        const long double wi = S * sn;
                        const bool out_im = n >= L, in_im = k >= L;
                        if (!out_im && !in_im) v = wr;
                        else if (!out_im && in_im) v = -wi;
                        else if (out_im && !in_im) v = wi;
                        else v = wr;
                    }
                    float w = (float)v;
                    for (int t = 0; t < TC_TERMS; ++t) {
                        const __nv_bfloat16 b = __float2bfloat16_rn(w);
                        tab[((((li * 2 + si) * TC_TERMS + t) * 32) + n) * 32 + k] = b;
                        w -= __bfloat162float(b);
                    }
                }
            }
        }
    }
}

int tc_tables_upload()
{
    static __nv_bfloat16 host[TC_B_ELEMS];
    static std::once_flag once;
    std::call_once(once, [] { tc_fill_host(host); });
    return cudaMemcpyToSymbol(g_tc_btab, host, sizeof(host)) == cudaSuccess ? FFT3D_B200_OK
                                                                           : FFT3D_B200_ERR_CUDA;
}

// ------------------------------------------------------------------ tcgen05 wrappers

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem desc] * B[smem desc]^T, bf16 x bf16 -> f32, one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate)
{
    const uint32_t z = 0;  // disable-output-lane mask: all lanes written
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 16 consecutive 32-bit columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Matrix descriptor, K-major, no swizzle (version 1, Blackwell).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // version
    // base offset 0, lbo mode 0, layout type 0 (no swizzle)
    return d;
}

// Instruction descriptor: bf16 x bf16 -> f32, both K-major, M x N.
constexpr uint32_t umma_idesc(int M, int N)
{
    return (1u << 4)                      // D format f32
           | (1u << 7)                    // A bf16
           | (1u << 10)                   // B bf16
           | ((uint32_t)(N >> 3) << 17)   // N
           | ((uint32_t)(M >> 4) << 24);  // M
}

// Byte offset of element (row, k) in a K-major no-swizzle tile with ROWS rows.
__device__ __forceinline__ int umma_off(int row, int k, int rows)
{
    return ((k >> 3) * (rows >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// ------------------------------------------------------------------ kernel

template <int L, int VPC, int SPLIT>
struct TcCfg {
    using G = Geom<L, L, L, float>;
    static constexpr int KP = 32;  // padded K (2L <= 32)
    static constexpr int NP = 32;  // padded N
    static constexpr int ROWS = 128;
    static constexpr int NTERM = SPLIT;
    static constexpr int NPROD = SPLIT == 2 ? 3 : 6;
    static constexpr int A_BYTES = ROWS * KP * 2;  // one term of one tile
    static constexpr int B_BYTES = NP * KP * 2;    // one term
    static constexpr int VOL_BYTES = ((VPC * G::PV * G::EB) + 1023) / 1024 * 1024;
    static constexpr int OFF_A = VOL_BYTES;
    static constexpr int OFF_B = OFF_A + 2 * NTERM * A_BYTES;
    static constexpr int OFF_BAR = OFF_B + NTERM * B_BYTES;
    // + 1 KB: the kernel rounds the dynamic shared-memory base up to 1024 bytes
    static constexpr int SMEM = OFF_BAR + 64 + 1024;
    static constexpr int LINES = VPC * L * L;
    static constexpr int ROUNDS = (LINES + 255) / 256;
};

template <int L, int S, int VPC, int SPLIT>
__global__ void __launch_bounds__(256, 1)
    k_tc(const cx<float> *__restrict__ in, cx<float> *__restrict__ out, long long nvol, float scale,
         int *err)
{
    pdl_begin();
    using C = TcCfg<L, VPC, SPLIT>;
    using G = typename C::G;
    // The dynamic segment follows the static one (s_abort) and starts only
    // 16-byte aligned (0x410 on B200), whatever alignment it is declared with;
    // a no-swizzle UMMA core matrix must start on a 128-byte boundary (16 bytes
    // off, the hardware reads its rows shifted), so the base is rounded up here.
    // Declared 16-byte aligned so that the compiler cannot fold the rounding away.
    extern __shared__ __align__(16) unsigned char smdyn[];
    unsigned char *smraw = smdyn + ((1024u - (smem_u32(smdyn) & 1023u)) & 1023u);
    cx<float> *vol = reinterpret_cast<cx<float> *>(smraw);
    unsigned char *sA = smraw + C::OFF_A;
    unsigned char *sB = smraw + C::OFF_B;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + C::OFF_BAR);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smraw + C::OFF_BAR + 8);
    __shared__ int s_abort;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;

    // set-up: tensor memory (64 columns: two 128 x 32 f32 accumulators), barrier, B
    if (warp == 0) {
        tmem_alloc(tmem_slot, 64);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
        s_abort = 0;
    }
    {
        const __nv_bfloat16 *bt = g_tc_btab + (size_t)((tc_li(L) * 2 + (S < 0 ? 0 : 1)) * TC_TERMS) * 32 * 32;
        for (int i = tid; i < C::NTERM * 32 * 32; i += 256) {
            const int t = i / 1024, n = (i / 32) % 32, k = i % 32;
            *reinterpret_cast<__nv_bfloat16 *>(sB + t * C::B_BYTES + umma_off(n, k, C::NP)) = bt[i];
        }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    constexpr uint32_t IDESC = umma_idesc(128, C::NP);
    uint32_t phase = 0;
    int pending = 0;

    const long long nitems = (nvol + VPC - 1) / VPC;
    for (long long item = blockIdx.x; item < nitems && !s_abort; item += gridDim.x) {
        const long long v0 = item * VPC;
        const int nv = (int)((nvol - v0) < VPC ? (nvol - v0) : VPC);
        const cx<float> *gin = in + v0 * G::V;
        cx<float> *gout = out + v0 * G::V;
        for (int g = tid; g < nv * G::V; g += 256) stage_in<G>(vol, gin, g);
        __syncthreads();
        for (int pass = 0; pass < 3 && !s_abort; ++pass) {
            for (int round = 0; round < C::ROUNDS; ++round) {
                if (s_abort) break;
                const int line = round * 256 + tid;
                const bool valid = line < nv * L * L;
                // gather the line (pass 0: z rows; 1: y lines; 2: x lines)
                float xr[L], xi[L];
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    xr[j] = 0.f;
                    xi[j] = 0.f;
                }
                int vv = 0, a = 0, b = 0;
                if (valid) {
                    if (pass == 0) {
#pragma unroll
                        for (int j = 0; j < L; ++j) {
                            const cx<float> p = vol[G::off(line, j)];
                            xr[j] = p.re;
                            xi[j] = p.im;
                        }
                    } else if (pass == 1) {
                        const int z = line % L, rb = (line / L) * L;
#pragma unroll
                        for (int j = 0; j < L; ++j) {
                            const cx<float> p = vol[G::off(rb + j, z)];
                            xr[j] = p.re;
                            xi[j] = p.im;
                        }
                    } else {
                        a = line % L;                  // z
                        b = (line / L) % L;            // y
                        vv = line / (L * L);           // volume
#pragma unroll
                        for (int j = 0; j < L; ++j) {
                            const cx<float> p = vol[G::off((vv * L + j) * L + b, a)];
                            xr[j] = p.re;
                            xi[j] = p.im;
                        }
                    }
                }
                // split into bf16 terms and write this thread's A row
                {
                    // 8 consecutive k of one row are 16 contiguous bytes of a core matrix
                    const int tile = tid >> 7, row = tid & 127;
#pragma unroll
                    for (int c = 0; c < C::KP / 8; ++c) {
                        // words[t][h]: bf16 terms t of k = c*8 + 2h (low half) and 2h + 1
                        uint32_t words[C::NTERM][4];
#pragma unroll
                        for (int t = 0; t < C::NTERM; ++t)
#pragma unroll
                            for (int h = 0; h < 4; ++h) words[t][h] = 0u;
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int k = c * 8 + q;
                            float w = k < L ? xr[k < L ? k : 0] : (k < 2 * L ? xi[k >= L && k < 2 * L ? k - L : 0] : 0.f);
#pragma unroll
                            for (int t = 0; t < C::NTERM; ++t) {
                                const __nv_bfloat16 b = __float2bfloat16_rn(w);
                                w -= __bfloat162float(b);
                                words[t][q >> 1] |= (uint32_t)__bfloat16_as_ushort(b) << (16 * (q & 1));
                            }
                        }
#pragma unroll
                        for (int t = 0; t < C::NTERM; ++t)
                            *reinterpret_cast<uint4 *>(sA + (tile * C::NTERM + t) * C::A_BYTES +
                                                       umma_off(row, c * 8, 128)) =
                                make_uint4(words[t][0], words[t][1], words[t][2], words[t][3]);
                    }
                }
                fence_proxy_async_smem();
                tc_fence_before();
                __syncthreads();
                if (tid == 0) {
                    tc_fence_after();
                    // products (a-term, b-term)
                    constexpr int PA[6] = {0, 0, 1, 0, 2, 1};
                    constexpr int PB[6] = {0, 1, 0, 2, 0, 1};
                    const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
#pragma unroll
                    for (int tile = 0; tile < 2; ++tile) {
#pragma unroll
                        for (int p = 0; p < C::NPROD; ++p) {
#pragma unroll
                            for (int s = 0; s < C::KP / 16; ++s) {
                                const uint32_t aaddr = aBase + (tile * C::NTERM + PA[p]) * C::A_BYTES +
                                                       s * 2 * (128 / 8) * 128;
                                const uint32_t baddr = bBase + PB[p] * C::B_BYTES + s * 2 * (C::NP / 8) * 128;
                                const uint64_t ad = umma_desc(aaddr, (128 / 8) * 128, 128);
                                const uint64_t bd = umma_desc(baddr, (C::NP / 8) * 128, 128);
                                umma_bf16(tmem + tile * C::NP, ad, bd, IDESC, (p | s) ? 1u : 0u);
                            }
                        }
                    }
                    umma_commit(bar);
                }
                if (!mbar_wait_bounded(bar, phase)) {
                    s_abort = 1;
                    pending = 1;  // the commit of this phase may still arrive
                } else {
                    phase ^= 1;
                }
                tc_fence_after();
                __syncwarp();  // tcgen05.ld is warp-collective (.sync.aligned)
                // this thread's row of D: tile = warp / 4, lanes 32 * (warp % 4) + lane
                float d[C::NP];
                {
                    const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) +
                                           (uint32_t)((warp >> 2) * C::NP);
                    tmem_ld16(taddr, d);
                    tmem_ld16(taddr + 16, d + 16);
                }
                if (valid && !s_abort) {
                    if (pass == 0) {
#pragma unroll
                        for (int n = 0; n < L; ++n) vol[G::off(line, n)] = {d[n], d[L + n]};
                    } else if (pass == 1) {
                        const int z = line % L, rb = (line / L) * L;
#pragma unroll
                        for (int n = 0; n < L; ++n) vol[G::off(rb + n, z)] = {d[n], d[L + n]};
                    } else {
#pragma unroll
                        for (int n = 0; n < L; ++n) {
                            cx<float> r = {d[n], d[L + n]};
                            if (S > 0) r = cscale(r, scale);
                            store_out(gout + (long long)vv * G::V + (n * L + b) * L + a, r);
                        }
                    }
                }
                tc_fence_before();
                __syncthreads();
            }
        }
    }
    if (s_abort) {
        if (tid == 0) report_error(err, DEV_ERR_LOAD_TIMEOUT);
        // bounded wait for MMAs still in flight before their tensor memory is freed
        if (pending) mbar_wait_bounded(bar, phase);
    }
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, 64);
}

template <int L, int S, int VPC, int SPLIT>
static void add_tc(std::vector<KernelEntry> &out, const char *name)
{
    KernelEntry e;
    e.n0 = e.n1 = e.n2 = L;
    e.precision = FFT3D_B200_C64;
    e.sign = S;
    e.family = FAM_STREAM;  // persistent launch: (in, out, nvol, scale, err)
    e.alg = 10 + SPLIT;
    e.vpc = VPC;
    e.threads = 256;
    e.smem = TcCfg<L, VPC, SPLIT>::SMEM;
    e.func = (const void *)&k_tc<L, S, VPC, SPLIT>;
    e.name = name;
    out.push_back(e);
}

#define FFT3D_TC(L, VPC, SPLIT)                                                                \
    add_tc<L, -1, VPC, SPLIT>(out, "tensor " #L "x" #L "x" #L " float split" #SPLIT " vpc" #VPC); \
    add_tc<L, +1, VPC, SPLIT>(out, "tensor " #L "x" #L "x" #L " float split" #SPLIT " vpc" #VPC)

void register_tc_kernels(std::vector<KernelEntry> &out)
{
    FFT3D_TC(16, 1, 3);
    FFT3D_TC(16, 1, 2);
    FFT3D_TC(8, 4, 3);
    FFT3D_TC(8, 4, 2);
    FFT3D_TC(12, 4, 3);
    FFT3D_TC(6, 7, 3);
}

}  // namespace fft3d

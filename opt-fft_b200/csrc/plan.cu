// plan.cu -- plans, the autotuner, host-pointer staging and every exported symbol.
//
// Exports the reference contract twice -- host pointers (bench/geom/fft3d_api.h:49-66)
// and device pointers (bench/gpu/fft3d_gpu_api.h:57-83) -- and the extension API
// of fft3d_b200.h.  All precomputation happens at plan creation
// (bench/geom/fft3d_api.h:30-32): tables, kernel choice by timing the compiled
// variants (the plan-time race of bench/geom/best/fft3d_best.c:131-193, done on
// the GPU over kernel variants), device buffers and pinned staging.  There is no
// CPU fallback: without a usable CUDA device every create fails.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/fft3d_api.h"
#include "../../include/fft3d_b200.h"
#include "../../include/fft3d_gpu_api.h"
#include "internal.h"

namespace fft3d {

static thread_local int t_last_status = FFT3D_B200_OK;

static int set_status(int s)
{
    t_last_status = s;
    return s;
}

int record_status(int s) { return set_status(s); }

int element_bytes(int precision) { return precision == FFT3D_B200_C64 ? 8 : 16; }

const std::vector<KernelEntry> &registry()
{
    static std::vector<KernelEntry> reg;
    static std::once_flag once;
    std::call_once(once, [] {
        register_stream_kernels(reg);
        register_direct_kernels(reg);
        register_tc_kernels(reg);
        register_kernels(reg);
        register_cluster_kernels(reg);
        register_twopass_kernels(reg);
    });
    return reg;
}

// Programmatic dependent launch for every kernel started here (each calls
// pdl_begin() before touching global memory): the CTAs of a launch are placed
// while the previous kernel of the stream drains, and start work the moment it
// completes.  FFT3D_B200_PDL=0 turns it off (plain stream order); the legacy
// default stream always gets plain order.
static bool pdl_enabled()
{
    static const bool on = [] {
        const char *v = std::getenv("FFT3D_B200_PDL");
        return !(v && v[0] == '0');
    }();
    return on;
}

static cudaError_t launch_ex(const KernelEntry &e, dim3 grid, void **args, cudaStream_t stream,
                             unsigned cluster /* CTAs per cluster, 0: none */)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(e.threads);
    cfg.dynamicSmemBytes = (size_t)e.smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[2];
    unsigned n = 0;
    if (cluster) {
        attr[n].id = cudaLaunchAttributeClusterDimension;
        attr[n].val.clusterDim.x = cluster;
        attr[n].val.clusterDim.y = 1;
        attr[n].val.clusterDim.z = 1;
        ++n;
    }
    if (pdl_enabled() && stream != nullptr && stream != cudaStreamLegacy) {
        attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n].val.programmaticStreamSerializationAllowed = 1;
        ++n;
    }
    cfg.attrs = attr;
    cfg.numAttrs = n;
    return cudaLaunchKernelExC(&cfg, e.func, args);
}

cudaError_t launch_entry(const KernelEntry &e, const void *in, void *out, long long nvol,
                         double scale, cudaStream_t stream, int grid_limit, int *err, void *work)
{
    if (nvol <= 0) return cudaSuccess;
    if (e.family == FAM_TWOPASS) {
        if (!work) return cudaErrorInvalidValue;
        const long long items = (long long)(e.n0 / e.vpc + e.n1 / e.vpc) * nvol;
        const long long grid = std::max(1LL, std::min(items, (long long)grid_limit));
        int lag = 0;
        int ring = twopass_ring(e, grid, &lag);
        unsigned char *w = (unsigned char *)work;
        if (e.precision == FFT3D_B200_C128) {
            double s = scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s,
                            (void *)&err, (void *)&w,  (void *)&ring, (void *)&lag};
            return launch_ex(e, dim3((unsigned)grid), args, stream, 0);
        } else {
            float s = (float)scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s,
                            (void *)&err, (void *)&w,  (void *)&ring, (void *)&lag};
            return launch_ex(e, dim3((unsigned)grid), args, stream, 0);
        }
    }
    if (e.family == FAM_STREAM) {
        const long long items = (nvol + e.vpc - 1) / e.vpc;
        const long long grid = std::max(1LL, std::min(items, (long long)grid_limit));
        if (e.precision == FFT3D_B200_C128) {
            double s = scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s, (void *)&err};
            return launch_ex(e, dim3((unsigned)grid), args, stream, 0);
        } else {
            float s = (float)scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s, (void *)&err};
            return launch_ex(e, dim3((unsigned)grid), args, stream, 0);
        }
    }
    if (e.family == FAM_VOLUME) {
        const long long grid = (nvol + e.vpc - 1) / e.vpc;
        if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        if (e.precision == FFT3D_B200_C128) {
            double s = scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s};
            return launch_ex(e, dim3((unsigned)grid), args, stream, 0);
        } else {
            float s = (float)scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s};
            return launch_ex(e, dim3((unsigned)grid), args, stream, 0);
        }
    }
    if (e.family == FAM_CLUSTER) {
        // one cluster of e.vpc CTAs per volume
        if (nvol * e.vpc > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        const dim3 grid((unsigned)(nvol * e.vpc));
        if (e.precision == FFT3D_B200_C128) {
            double s = scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s, (void *)&err};
            return launch_ex(e, grid, args, stream, (unsigned)e.vpc);
        } else {
            float s = (float)scale;
            void *args[] = {(void *)&in, (void *)&out, (void *)&nvol, (void *)&s, (void *)&err};
            return launch_ex(e, grid, args, stream, (unsigned)e.vpc);
        }
    }
    return cudaErrorInvalidValue;
}

// Per-device attribute setup of a kernel (dynamic shared memory above 48 KB) and
// its occupancy, memoised.
int entry_occupancy(const KernelEntry &e, int device)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> occ;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(e.func, device);
    auto it = occ.find(key);
    if (it != occ.end()) return it->second;
    int n = 0;
    if (cudaFuncSetAttribute(e.func, cudaFuncAttributeMaxDynamicSharedMemorySize, e.smem) ==
        cudaSuccess) {
        if (e.family == FAM_CLUSTER) {
            // clusters: the number of clusters that can be resident at once
            if (e.vpc > 8 &&
                cudaFuncSetAttribute(e.func, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                    cudaSuccess)
                cudaGetLastError();
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)e.vpc * 16);
            cfg.blockDim = dim3(e.threads);
            cfg.dynamicSmemBytes = (size_t)e.smem;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = e.vpc;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            if (cudaOccupancyMaxActiveClusters(&n, e.func, &cfg) != cudaSuccess) n = 0;
        } else if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, e.func, e.threads,
                                                                 (size_t)e.smem) != cudaSuccess) {
            n = 0;
        }
    }
    cudaGetLastError();
    occ[key] = n;
    return n;
}

static int prepare_entry(const KernelEntry &e, int device)
{
    return entry_occupancy(e, device) > 0 ? FFT3D_B200_OK : FFT3D_B200_ERR_UNSUPPORTED;
}

static std::vector<const KernelEntry *> candidates(int n0, int n1, int n2, int precision, int sign)
{
    std::vector<const KernelEntry *> c;
    for (const auto &e : registry())
        if (e.n0 == n0 && e.n1 == n1 && e.n2 == n2 && e.precision == precision && e.sign == sign)
            c.push_back(&e);
    return c;
}

// Process-wide memo of tuning results: (device, geometry, precision, sign, batch
// bucket) -> registry index of the winner.
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int, int, int, int>, const KernelEntry *> g_tuned;

static int batch_bucket(long long b)
{
    int k = 0;
    while (b > 1 && k < 62) { b >>= 1; ++k; }
    return k;
}

// Time every candidate on plan-owned scratch of min(batch, cap) volumes and
// return the fastest.  Candidates that fail to launch are skipped.
static const KernelEntry *tune(const std::vector<const KernelEntry *> &cands, int device,
                               long long batch, int precision, long long vol_elems, int num_sms,
                               int *err, std::string *log)
{
    if (cands.size() == 1) return cands[0];
    const size_t eb = (size_t)element_bytes(precision);
    long long cap = (long long)((size_t)512 << 20) / (long long)(vol_elems * eb);
    if (cap < 1) cap = 1;
    const long long nb = std::max(1LL, std::min(batch, cap));
    const size_t bytes = (size_t)nb * vol_elems * eb;
    // Rotate over enough buffer pairs that a launch never finds its input in L2:
    // the candidates are timed the way an HBM-bound batch runs.
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device);
    const int sets = (int)std::min<long long>(8, std::max<long long>(1, (3LL * l2) / (long long)(2 * bytes) + 1));
    std::vector<void *> bufs;
    for (int i = 0; i < 2 * sets; ++i) {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            break;
        }
        cudaMemset(p, 0x3f, bytes);  // finite, normal values in both precisions
        bufs.push_back(p);
    }
    if (bufs.size() < 2) {
        for (void *p : bufs) cudaFree(p);
        return cands[0];
    }
    const int nsets = (int)bufs.size() / 2;
    cudaStream_t s;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const KernelEntry *best = nullptr;
    float best_ms = 1e30f;
    for (const KernelEntry *k : cands) {
        const int occ = entry_occupancy(*k, device);
        if (occ <= 0) continue;
        const int glim = occ * num_sms;
        void *work = nullptr;
        const size_t wb = entry_workspace_bytes(*k, glim);
        if (wb && (cudaMalloc(&work, wb) != cudaSuccess ||
                   cudaMemset(work, 0, TWOPASS_CTL_BYTES) != cudaSuccess)) {
            cudaGetLastError();
            if (work) cudaFree(work);
            continue;
        }
        bool ok = true;
        for (int w = 0; w < 2 && ok; ++w)
            ok = launch_entry(*k, bufs[0], bufs[1], nb, 1.0, s, glim, err, work) == cudaSuccess;
        if (!ok || cudaStreamSynchronize(s) != cudaSuccess) {
            cudaGetLastError();
            if (work) cudaFree(work);
            continue;
        }
        float ms_min = 1e30f;
        const int reps = 2 * nsets;
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0, s);
            for (int it = 0; it < reps; ++it) {
                const int j = it % nsets;
                launch_entry(*k, bufs[2 * j], bufs[2 * j + 1], nb, 1.0, s, glim, err, work);
            }
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_min = std::min(ms_min, ms / (float)reps);
        }
        if (work) {
            cudaStreamSynchronize(s);
            cudaFree(work);
        }
        if (log) {
            char buf[256];
            snprintf(buf, sizeof buf, "%s: %.3f us; ", k->name, ms_min * 1e3f);
            *log += buf;
        }
        if (ms_min < best_ms) {
            best_ms = ms_min;
            best = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    for (void *p : bufs) cudaFree(p);
    return best ? best : cands[0];
}

const KernelEntry *tuned_entry(int device, int n0, int n1, int n2, int precision, int sign,
                               long long batch, bool workspace_ok)
{
    std::vector<const KernelEntry *> cands;
    for (const KernelEntry *k : candidates(n0, n1, n2, precision, sign))
        if (workspace_ok || k->family != FAM_TWOPASS) cands.push_back(k);
    if (cands.empty()) return nullptr;
    // a memo of its own, per candidate set
    static std::map<std::tuple<int, int, int, int, int, int, int, bool>, const KernelEntry *> memo;
    auto key = std::make_tuple(device, n0, n1, n2, precision, sign, batch_bucket(batch), workspace_ok);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const KernelEntry *k =
        getenv("FFT3D_B200_NO_TUNE")
            ? cands[0]
            : tune(cands, device, batch, precision, (long long)n0 * n1 * n2, sms, nullptr, nullptr);
    memo[key] = k;
    return k;
}

}  // namespace fft3d

using namespace fft3d;

struct fft3d_b200_plan {
    fft3d_b200_desc desc;
    int device;
    int num_sms;
    long long vol_elems;
    size_t bytes;  // whole batch, one buffer
    double scale;
    const KernelEntry *kernel;
    int grid_limit;          // persistent families: CTAs per SM x SMs
    int *d_err = nullptr;    // device error word (bounded-wait timeouts)
    // kernel workspace (TWOPASS scratch ring): [0] for device-pointer executes,
    // [1] for the second stream of host-pointer executes; 0 bytes for other families
    size_t work_bytes = 0;
    void *work[2] = {nullptr, nullptr};
    std::string describe;
    // host-pointer execution
    void *d_in = nullptr, *d_out = nullptr;
    void *pin[2] = {nullptr, nullptr};
    size_t pin_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t xs[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

static int validate_desc(const fft3d_b200_desc *d)
{
    if (!d) return FFT3D_B200_ERR_INVALID;
    if (d->n0 < 1 || d->n1 < 1 || d->n2 < 1 || d->batch < 0) return FFT3D_B200_ERR_INVALID;
    if (d->direction != FFT3D_B200_FORWARD && d->direction != FFT3D_B200_BACKWARD)
        return FFT3D_B200_ERR_INVALID;
    if (d->precision != FFT3D_B200_C128 && d->precision != FFT3D_B200_C64)
        return FFT3D_B200_ERR_INVALID;
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_supports(int n0, int n1, int n2, int precision)
{
    if (n0 < 1 || n1 < 1 || n2 < 1) return 0;
    return candidates(n0, n1, n2, precision, -1).empty() ? 0 : 1;
}

extern "C" int fft3d_b200_variants(int n0, int n1, int n2, int precision, int direction,
                                   const char **names, int max)
{
    auto c = candidates(n0, n1, n2, precision, direction);
    for (int i = 0; i < (int)c.size() && i < max && names; ++i) names[i] = c[i]->name;
    return (int)c.size();
}

// ------------------------------------------------------------------ wisdom
//
// The plan-time race (bench/geom/best/fft3d_best.c:148-193) generalised to a
// per-host cache (bench/gen/PANEL_BRIEF.md:12-20): the tuner's choices are
// written as text, one per line,
//     <device name>|sm<major>.<minor>|<SMs> TAB <n0 n1 n2 precision sign bucket> TAB <variant>
// and read back into the memo for every visible device of the same type, so a
// later process skips the timing.  Lines for device types not present here are
// kept and written back unchanged.  The memo mutex (g_tune_mu) guards all of it.

namespace fft3d {

static std::vector<std::string> g_wisdom_foreign;
static bool g_wisdom_autoloaded = false;

static std::string device_tag(int device)
{
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, device) != cudaSuccess) {
        cudaGetLastError();
        return std::string();
    }
    char buf[400];
    snprintf(buf, sizeof buf, "%s|sm%d.%d|%d", pr.name, pr.major, pr.minor, pr.multiProcessorCount);
    for (char *c = buf; *c; ++c)
        if (*c == '\t' || *c == '\n') *c = ' ';
    return buf;
}

// Write the memo (and the kept foreign lines) to `path` via a temporary file.
static int wisdom_write(const char *path)
{
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = fopen(tmp.c_str(), "w");
    if (!f) return FFT3D_B200_ERR_INVALID;
    fprintf(f, "fft3d_b200 wisdom 1\n");
    int n = 0;
    std::map<int, std::string> tags;
    for (const auto &kv : g_tuned) {
        int dev, n0, n1, n2, prec, sign, bucket;
        std::tie(dev, n0, n1, n2, prec, sign, bucket) = kv.first;
        if (!tags.count(dev)) tags[dev] = device_tag(dev);
        if (tags[dev].empty() || !kv.second) continue;
        fprintf(f, "%s\t%d %d %d %d %d %d\t%s\n", tags[dev].c_str(), n0, n1, n2, prec, sign, bucket,
                kv.second->name);
        ++n;
    }
    for (const auto &line : g_wisdom_foreign) fprintf(f, "%s\n", line.c_str());
    const bool ok = fclose(f) == 0;
    if (!ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return FFT3D_B200_ERR_INVALID;
    }
    return n;
}

// Merge the entries of `path` into the memo; returns entries taken or an error.
static int wisdom_read(const char *path)
{
    FILE *f = fopen(path, "r");
    if (!f) return FFT3D_B200_ERR_INVALID;
    char line[1024];
    if (!fgets(line, sizeof line, f) || strncmp(line, "fft3d_b200 wisdom 1", 19) != 0) {
        fclose(f);
        return FFT3D_B200_ERR_INVALID;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
        cudaGetLastError();
        ndev = 0;
    }
    std::vector<std::string> tags(ndev);
    for (int d = 0; d < ndev; ++d) tags[d] = device_tag(d);
    int taken = 0;
    while (fgets(line, sizeof line, f)) {
        std::string s(line);
        while (!s.empty() && (s.back() == '\n' || s.back() == '\r')) s.pop_back();
        const size_t t1 = s.find('\t'), t2 = t1 == std::string::npos ? t1 : s.find('\t', t1 + 1);
        if (t2 == std::string::npos) continue;  // malformed: ignored
        const std::string tag = s.substr(0, t1), name = s.substr(t2 + 1);
        int n0, n1, n2, prec, sign, bucket;
        if (sscanf(s.c_str() + t1 + 1, "%d %d %d %d %d %d", &n0, &n1, &n2, &prec, &sign, &bucket) != 6)
            continue;
        const KernelEntry *e = nullptr;
        for (const auto &r : registry())
            if (name == r.name && r.n0 == n0 && r.n1 == n1 && r.n2 == n2 && r.precision == prec &&
                r.sign == sign)
                e = &r;
        bool matched = false;
        for (int d = 0; d < ndev; ++d) {
            if (tags[d].empty() || tags[d] != tag) continue;
            matched = true;
            if (!e) continue;  // a variant this build does not have
            g_tuned[std::make_tuple(d, n0, n1, n2, prec, sign, bucket)] = e;
            ++taken;
        }
        if (!matched && std::find(g_wisdom_foreign.begin(), g_wisdom_foreign.end(), s) ==
                            g_wisdom_foreign.end())
            g_wisdom_foreign.push_back(s);
    }
    fclose(f);
    return taken;
}

// FFT3D_B200_WISDOM=<path>: read once, at the first plan creation that tunes.
static void wisdom_autoload()
{
    if (g_wisdom_autoloaded) return;
    g_wisdom_autoloaded = true;
    if (const char *w = getenv("FFT3D_B200_WISDOM")) wisdom_read(w);
}

}  // namespace fft3d

extern "C" int fft3d_b200_wisdom_export(const char *path)
{
    if (!path) return fft3d::set_status(FFT3D_B200_ERR_INVALID);
    std::lock_guard<std::mutex> lk(fft3d::g_tune_mu);
    const int n = fft3d::wisdom_write(path);
    fft3d::set_status(n < 0 ? n : FFT3D_B200_OK);
    return n;
}

extern "C" int fft3d_b200_wisdom_import(const char *path)
{
    if (!path) return fft3d::set_status(FFT3D_B200_ERR_INVALID);
    std::lock_guard<std::mutex> lk(fft3d::g_tune_mu);
    const int n = fft3d::wisdom_read(path);
    fft3d::set_status(n < 0 ? n : FFT3D_B200_OK);
    return n;
}

extern "C" void fft3d_b200_wisdom_forget(void)
{
    std::lock_guard<std::mutex> lk(fft3d::g_tune_mu);
    fft3d::g_tuned.clear();
    fft3d::g_wisdom_foreign.clear();
}

// Allocate workspace `i` of a plan whose kernel needs one; its control block
// starts zeroed (each launch leaves it zeroed again).
static int ensure_work(fft3d_b200_plan *p, int i)
{
    if (!p->work_bytes || p->work[i]) return FFT3D_B200_OK;
    if (cudaMalloc(&p->work[i], p->work_bytes) != cudaSuccess ||
        cudaMemset(p->work[i], 0, TWOPASS_CTL_BYTES) != cudaSuccess) {
        cudaGetLastError();
        if (p->work[i]) cudaFree(p->work[i]);
        p->work[i] = nullptr;
        return FFT3D_B200_ERR_NOMEM;
    }
    return FFT3D_B200_OK;
}

static int plan_create_impl(const fft3d_b200_desc *desc, const char *variant,
                            fft3d_b200_plan **out)
{
    if (!out) return set_status(FFT3D_B200_ERR_INVALID);
    *out = nullptr;
    int st = validate_desc(desc);
    if (st) return set_status(st);
    auto cands = candidates(desc->n0, desc->n1, desc->n2, desc->precision, desc->direction);
    if (cands.empty()) return set_status(FFT3D_B200_ERR_UNSUPPORTED);
    const KernelEntry *forced = nullptr;
    if (variant) {
        for (const KernelEntry *c : cands)
            if (strcmp(c->name, variant) == 0) forced = c;
        if (!forced) return set_status(FFT3D_B200_ERR_UNSUPPORTED);
    }

    int device = desc->device;
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) {
            cudaGetLastError();
            return set_status(FFT3D_B200_ERR_CUDA);
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device >= ndev) {
        cudaGetLastError();
        return set_status(FFT3D_B200_ERR_CUDA);
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return set_status(FFT3D_B200_ERR_CUDA);
    st = ensure_device_tables(device);
    if (st) {
        if (prev >= 0) cudaSetDevice(prev);
        return set_status(st);
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);

    fft3d_b200_plan *p = new fft3d_b200_plan();
    p->desc = *desc;
    p->device = device;
    p->num_sms = sms;
    p->vol_elems = (long long)desc->n0 * desc->n1 * desc->n2;
    p->bytes = (size_t)desc->batch * (size_t)p->vol_elems * (size_t)element_bytes(desc->precision);
    p->scale = desc->direction == FFT3D_B200_BACKWARD ? 1.0 / (double)p->vol_elems : 1.0;
    if (cudaMalloc(&p->d_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(p->d_err, 0, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        delete p;
        if (prev >= 0) cudaSetDevice(prev);
        return set_status(FFT3D_B200_ERR_NOMEM);
    }

    const bool no_tune = (desc->flags & FFT3D_B200_FLAG_NO_TUNE) || getenv("FFT3D_B200_NO_TUNE");
    const KernelEntry *k = forced;
    if (!k) {
        auto key = std::make_tuple(device, desc->n0, desc->n1, desc->n2, desc->precision,
                                   desc->direction, batch_bucket(desc->batch));
        std::lock_guard<std::mutex> lk(g_tune_mu);
        wisdom_autoload();
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            k = it->second;
        } else if (!no_tune && desc->batch > 0) {
            std::string log;
            k = tune(cands, device, desc->batch, desc->precision, p->vol_elems, sms, p->d_err,
                     &log);
            g_tuned[key] = k;
            if (getenv("FFT3D_B200_TUNE_LOG")) fprintf(stderr, "fft3d_b200 tune: %s\n", log.c_str());
            if (const char *w = getenv("FFT3D_B200_WISDOM")) wisdom_write(w);
        }
    }
    if (!k) k = cands[0];
    if (prepare_entry(*k, device) != FFT3D_B200_OK) {
        cudaFree(p->d_err);
        delete p;
        if (prev >= 0) cudaSetDevice(prev);
        return set_status(FFT3D_B200_ERR_UNSUPPORTED);
    }
    p->kernel = k;
    p->grid_limit = entry_occupancy(*k, device) * sms;
    p->describe = k->name;
    p->work_bytes = entry_workspace_bytes(*k, p->grid_limit);
    if (p->work_bytes && ensure_work(p, 0) != FFT3D_B200_OK) {
        cudaFree(p->d_err);
        delete p;
        if (prev >= 0) cudaSetDevice(prev);
        return set_status(FFT3D_B200_ERR_NOMEM);
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    *out = p;
    return set_status(FFT3D_B200_OK);
}

extern "C" int fft3d_b200_plan_create(const fft3d_b200_desc *desc, fft3d_b200_plan **out)
{
    return plan_create_impl(desc, nullptr, out);
}

extern "C" int fft3d_b200_plan_create_variant(const fft3d_b200_desc *desc, const char *variant,
                                              fft3d_b200_plan **out)
{
    if (!variant) return set_status(FFT3D_B200_ERR_INVALID);
    return plan_create_impl(desc, variant, out);
}

static void free_staging(fft3d_b200_plan *p)
{
    if (p->d_in) cudaFree(p->d_in);
    if (p->d_out) cudaFree(p->d_out);
    for (int i = 0; i < 2; ++i) {
        if (p->pin[i]) cudaFreeHost(p->pin[i]);
        if (p->xs[i]) cudaStreamDestroy(p->xs[i]);
        if (p->ev[i]) cudaEventDestroy(p->ev[i]);
        p->pin[i] = nullptr;
        p->xs[i] = nullptr;
        p->ev[i] = nullptr;
    }
    if (p->stream) cudaStreamDestroy(p->stream);
    p->d_in = p->d_out = nullptr;
    p->stream = nullptr;
}

// Status of the device error word; a recorded error is reported once and cleared.
static int read_device_error(fft3d_b200_plan *p)
{
    int v = 0;
    if (cudaMemcpy(&v, p->d_err, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    if (v == 0) return FFT3D_B200_OK;
    cudaMemset(p->d_err, 0, sizeof(int));
    return FFT3D_B200_ERR_TIMEOUT;
}

extern "C" int fft3d_b200_plan_check(fft3d_b200_plan *p)
{
    if (!p) return set_status(FFT3D_B200_ERR_INVALID);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p->device) cudaSetDevice(p->device);
    int st = FFT3D_B200_OK;
    if (cudaDeviceSynchronize() != cudaSuccess) st = FFT3D_B200_ERR_CUDA;
    if (st == FFT3D_B200_OK) st = read_device_error(p);
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
    return set_status(st);
}

// Test hook: start the next device-pointer execute of a TWOPASS plan at the
// first row item's ticket.  The plane items of volume 0 are then never handed
// out, so the row items that depend on them -- and, through the abort flag,
// every other CTA -- give up after their bounded wait: the launch ends by
// itself, fft3d_b200_plan_check reports FFT3D_B200_ERR_TIMEOUT, and the last
// CTA leaves the control block cleared for the following execute.
extern "C" int fft3d_b200_debug_stall_next_execute(fft3d_b200_plan *p)
{
    if (!p) return set_status(FFT3D_B200_ERR_INVALID);
    if (p->kernel->family != FAM_TWOPASS || !p->work[0] || p->desc.batch < 1)
        return set_status(FFT3D_B200_ERR_UNSUPPORTED);
    const KernelEntry &e = *p->kernel;
    const long long na = e.n0 / e.vpc, nb = e.n1 / e.vpc;
    const long long grid = std::max(1LL, std::min((na + nb) * p->desc.batch, (long long)p->grid_limit));
    int lag = 0;
    twopass_ring(e, grid, &lag);
    const long long nvol = p->desc.batch;
    const unsigned long long first_row = nvol <= lag ? (unsigned long long)(na * nvol)
                                                     : (unsigned long long)(na * lag + na);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p->device) cudaSetDevice(p->device);
    const cudaError_t ce = cudaMemcpy(p->work[0], &first_row, sizeof first_row, cudaMemcpyHostToDevice);
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
    return set_status(ce == cudaSuccess ? FFT3D_B200_OK : FFT3D_B200_ERR_CUDA);
}

extern "C" void fft3d_b200_plan_destroy(fft3d_b200_plan *p)
{
    if (!p) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    cudaDeviceSynchronize();
    free_staging(p);
    if (p->d_err) cudaFree(p->d_err);
    for (void *w : p->work)
        if (w) cudaFree(w);
    if (prev >= 0) cudaSetDevice(prev);
    delete p;
}

static bool ranges_overlap(const void *a, const void *b, size_t n)
{
    const char *x = (const char *)a, *y = (const char *)b;
    return x < y + n && y < x + n;
}

extern "C" int fft3d_b200_execute(fft3d_b200_plan *p, const void *d_in, void *d_out, void *stream)
{
    if (!p) return set_status(FFT3D_B200_ERR_INVALID);
    if (p->desc.batch == 0) return set_status(FFT3D_B200_OK);
    if (!d_in || !d_out) return set_status(FFT3D_B200_ERR_INVALID);
    const uintptr_t al = (uintptr_t)element_bytes(p->desc.precision);
    if (((uintptr_t)d_in % al) || ((uintptr_t)d_out % al)) return set_status(FFT3D_B200_ERR_ALIGN);
    if (ranges_overlap(d_in, d_out, p->bytes)) return set_status(FFT3D_B200_ERR_OVERLAP);
    cudaError_t e = launch_entry(*p->kernel, d_in, d_out, p->desc.batch, p->scale,
                                 (cudaStream_t)stream, p->grid_limit, p->d_err, p->work[0]);
    if (e != cudaSuccess) return set_status(FFT3D_B200_ERR_CUDA);
    return set_status(FFT3D_B200_OK);
}

// ------------------------------------------------------------------ host-pointer execution

static int ensure_staging(fft3d_b200_plan *p)
{
    if (p->d_in) return FFT3D_B200_OK;
    const size_t eb = (size_t)element_bytes(p->desc.precision);
    const size_t vb = (size_t)p->vol_elems * eb;
    if (cudaMalloc(&p->d_in, p->bytes) != cudaSuccess || cudaMalloc(&p->d_out, p->bytes) != cudaSuccess) {
        cudaGetLastError();
        free_staging(p);
        return FFT3D_B200_ERR_NOMEM;
    }
    // the largest chunk: about 1/8 of the batch (4..64 MB, whole volumes), or
    // FFT3D_B200_HOST_CHUNK_MB; run_host_chain ramps the first and last chunks
    size_t target = std::min<size_t>((size_t)64 << 20, std::max<size_t>((size_t)4 << 20, p->bytes / 8));
    if (const char *e = getenv("FFT3D_B200_HOST_CHUNK_MB")) {
        const long mb = strtol(e, nullptr, 10);
        if (mb >= 1 && mb <= 4096) target = (size_t)mb << 20;
    }
    size_t chunk = std::max(vb, (target + vb - 1) / vb * vb);
    chunk = std::min(chunk, p->bytes);
    p->pin_bytes = chunk;
    for (int i = 0; i < 2; ++i) {
        if (cudaHostAlloc(&p->pin[i], 2 * chunk, cudaHostAllocDefault) != cudaSuccess ||
            cudaStreamCreateWithFlags(&p->xs[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&p->ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            free_staging(p);
            return FFT3D_B200_ERR_NOMEM;
        }
    }
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        free_staging(p);
        return FFT3D_B200_ERR_NOMEM;
    }
    return FFT3D_B200_OK;
}

static bool is_pinned(const void *ptr)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static void par_memcpy(void *dst, const void *src, size_t n)
{
    const size_t kMin = (size_t)4 << 20;
    unsigned nt = std::thread::hardware_concurrency();
    if (nt > 8) nt = 8;
    if (n < kMin || nt < 2) {
        memcpy(dst, src, n);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        const size_t o = (size_t)t * per;
        if (o >= n) break;
        const size_t len = std::min(per, n - o);
        th.emplace_back([=] { memcpy((char *)dst + o, (const char *)src + o, len); });
    }
    for (auto &x : th) x.join();
}

// Run `nplans` transforms on device copies of the batch, chunk by chunk, between
// one upload and one download.  Chunks alternate over two streams so the copy
// engines, the kernels and (for pageable buffers) the host copies overlap.
// Chunk sizes (whole volumes) of a host-pointer execute: full chunks of
// `full` volumes in the middle, ramped 1/8, 1/4, 1/2 of that at both ends.
// Only the first chunk's upload and the last chunk's download run without
// traffic in the other direction; small end chunks keep those short (about
// 2.5 MB instead of 20 MB for the 161 MB of a 2048 x 17^3 round trip).
static std::vector<long long> host_chunks(long long nvol, long long full)
{
    std::vector<long long> head, mid, tail;
    long long left = nvol;
    for (int r = 3; r >= 1 && left > 0; --r) {
        const long long n = std::max(1LL, full >> r);
        head.push_back(std::min(left, n));
        left -= head.back();
        if (left > 0) {
            tail.push_back(std::min(left, n));
            left -= tail.back();
        }
    }
    while (left > 0) {
        mid.push_back(std::min(left, full));
        left -= mid.back();
    }
    std::vector<long long> out(head);
    out.insert(out.end(), mid.begin(), mid.end());
    out.insert(out.end(), tail.rbegin(), tail.rend());
    return out;
}

static int run_host_chain(fft3d_b200_plan *const *plans, int nplans, const void *h_in, void *h_out)
{
    fft3d_b200_plan *p = plans[0];
    int st = ensure_staging(p);
    if (st) return st;
    // staged chunks alternate over two streams: a second workspace for the second one
    for (int i = 0; i < nplans; ++i)
        if ((st = ensure_work(plans[i], 1)) != FFT3D_B200_OK) return st;
    const size_t eb = (size_t)element_bytes(p->desc.precision);
    const size_t vb = (size_t)p->vol_elems * eb;
    const bool pinned = is_pinned(h_in) && is_pinned(h_out);
    const size_t chunk = p->pin_bytes;  // the largest chunk: staging slot size
    const std::vector<long long> sizes = host_chunks(p->desc.batch, (long long)(chunk / vb));
    const size_t nchunks = sizes.size();
    std::vector<size_t> off(nchunks + 1, 0);
    for (size_t c = 0; c < nchunks; ++c) off[c + 1] = off[c] + (size_t)sizes[c] * vb;
    const char *src = (const char *)h_in;
    char *dst = (char *)h_out;
    cudaError_t err = cudaSuccess;
    auto chunk_len = [&](size_t c) { return off[c + 1] - off[c]; };
    // the kernels of one chunk; returns the device buffer holding the result
    auto transform = [&](char *din, char *dout, long long nv, cudaStream_t s, int slot, char **res) {
        char *a = din, *b = dout;
        for (int i = 0; i < nplans; ++i) {
            if (launch_entry(*plans[i]->kernel, a, b, nv, plans[i]->scale, s, plans[i]->grid_limit,
                             plans[i]->d_err, plans[i]->work[slot]) != cudaSuccess)
                return false;
            std::swap(a, b);
        }
        *res = a;
        return true;
    };
    if (pinned) {
        // page-locked buffers: uploads, transforms and downloads on streams of
        // their own, each chunk's steps ordered by events, so no upload waits
        // for an earlier download
        cudaStream_t up = p->xs[0], down = p->xs[1], comp = p->stream;
        // Copy boundaries on 64 KB: DMA from or to offsets that are only
        // 16-byte aligned runs markedly slower.  Upload c ends at the boundary
        // at or after chunk c's last volume (it may carry the head of chunk
        // c+1), download c at the boundary at or before it (only finished
        // results), so each chunk still waits for one upload and one transform.
        const size_t total = off[nchunks];
        const size_t A = (size_t)64 << 10;
        auto up_end = [&](size_t c) { return c + 1 == nchunks ? total : std::min(total, (off[c + 1] + A - 1) / A * A); };
        auto down_end = [&](size_t c) { return c + 1 == nchunks ? total : off[c + 1] / A * A; };
        const char *res_base = (nplans & 1) ? (const char *)p->d_out : (const char *)p->d_in;
        size_t ua = 0, da = 0;
        for (size_t c = 0; c < nchunks; ++c) {
            char *din = (char *)p->d_in + off[c];
            char *dout = (char *)p->d_out + off[c];
            char *res = nullptr;
            const size_t ub = std::max(ua, up_end(c)), db = std::max(da, down_end(c));
            if ((ub > ua && cudaMemcpyAsync((char *)p->d_in + ua, src + ua, ub - ua, cudaMemcpyHostToDevice, up) != cudaSuccess) ||
                cudaEventRecord(p->ev[0], up) != cudaSuccess || cudaStreamWaitEvent(comp, p->ev[0], 0) != cudaSuccess ||
                !transform(din, dout, sizes[c], comp, 0, &res) || cudaEventRecord(p->ev[1], comp) != cudaSuccess ||
                cudaStreamWaitEvent(down, p->ev[1], 0) != cudaSuccess ||
                (db > da && cudaMemcpyAsync(dst + da, res_base + da, db - da, cudaMemcpyDeviceToHost, down) != cudaSuccess))
                return FFT3D_B200_ERR_CUDA;
            ua = ub;
            da = db;
        }
        if (cudaStreamSynchronize(down) != cudaSuccess || cudaStreamSynchronize(comp) != cudaSuccess ||
            cudaStreamSynchronize(up) != cudaSuccess)
            return FFT3D_B200_ERR_CUDA;
    } else {
        // pageable buffers: through the plan's page-locked staging, two slots
        for (size_t c = 0; c < nchunks; ++c) {
            const int slot = (int)(c & 1);
            cudaStream_t s = p->xs[slot];
            const size_t len = chunk_len(c);
            char *din = (char *)p->d_in + off[c];
            char *dout = (char *)p->d_out + off[c];
            char *stage_in = (char *)p->pin[slot];
            char *stage_out = stage_in + chunk;
            // the slot's previous chunk must be downloaded and copied out first
            if (c >= 2) {
                if (cudaEventSynchronize(p->ev[slot]) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
                par_memcpy(dst + off[c - 2], stage_out, chunk_len(c - 2));
            }
            par_memcpy(stage_in, src + off[c], len);
            char *res = nullptr;
            if (cudaMemcpyAsync(din, stage_in, len, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                !transform(din, dout, sizes[c], s, slot, &res) ||
                cudaMemcpyAsync(stage_out, res, len, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaEventRecord(p->ev[slot], s) != cudaSuccess)
                return FFT3D_B200_ERR_CUDA;
        }
        for (size_t c = (nchunks >= 2 ? nchunks - 2 : 0); c < nchunks; ++c) {
            const int slot = (int)(c & 1);
            if (cudaEventSynchronize(p->ev[slot]) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
            par_memcpy(dst + off[c], (char *)p->pin[slot] + chunk, chunk_len(c));
        }
        for (int i = 0; i < 2; ++i)
            if (cudaStreamSynchronize(p->xs[i]) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    }
    for (int i = 0; i < nplans; ++i) {
        const int st = read_device_error(plans[i]);
        if (st) return st;
    }
    return FFT3D_B200_OK;
}

extern "C" int fft3d_b200_execute_host_chain(fft3d_b200_plan *const *plans, int nplans,
                                             const void *h_in, void *h_out)
{
    if (!plans || nplans < 1 || !plans[0]) return set_status(FFT3D_B200_ERR_INVALID);
    const fft3d_b200_plan *p0 = plans[0];
    for (int i = 1; i < nplans; ++i) {
        const fft3d_b200_plan *q = plans[i];
        if (!q || q->desc.n0 != p0->desc.n0 || q->desc.n1 != p0->desc.n1 ||
            q->desc.n2 != p0->desc.n2 || q->desc.precision != p0->desc.precision ||
            q->desc.batch != p0->desc.batch || q->device != p0->device)
            return set_status(FFT3D_B200_ERR_INVALID);
    }
    if (p0->desc.batch == 0) return set_status(FFT3D_B200_OK);
    if (!h_in || !h_out) return set_status(FFT3D_B200_ERR_INVALID);
    if (ranges_overlap(h_in, h_out, p0->bytes)) return set_status(FFT3D_B200_ERR_OVERLAP);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p0->device) cudaSetDevice(p0->device);
    int st = run_host_chain(plans, nplans, h_in, h_out);
    if (prev >= 0 && prev != p0->device) cudaSetDevice(prev);
    return set_status(st);
}

extern "C" int fft3d_b200_execute_host(fft3d_b200_plan *p, const void *h_in, void *h_out)
{
    fft3d_b200_plan *const one[1] = {p};
    return fft3d_b200_execute_host_chain(one, 1, h_in, h_out);
}

extern "C" const char *fft3d_b200_plan_describe(const fft3d_b200_plan *p)
{
    return p ? p->describe.c_str() : "";
}

extern "C" int fft3d_b200_plan_launches(const fft3d_b200_plan *p) { return p ? 1 : 0; }

extern "C" int fft3d_b200_last_status(void) { return t_last_status; }

extern "C" const char *fft3d_b200_status_string(int s)
{
    switch (s) {
    case FFT3D_B200_OK: return "ok";
    case FFT3D_B200_ERR_INVALID: return "invalid argument";
    case FFT3D_B200_ERR_UNSUPPORTED: return "unsupported geometry or precision";
    case FFT3D_B200_ERR_ALIGN: return "buffer not aligned to its element size";
    case FFT3D_B200_ERR_CUDA: return "CUDA runtime error";
    case FFT3D_B200_ERR_NOMEM: return "out of memory";
    case FFT3D_B200_ERR_TIMEOUT: return "bounded device wait timed out";
    case FFT3D_B200_ERR_BUDGET: return "request exceeds the admission budget";
    case FFT3D_B200_ERR_OVERLAP: return "input and output overlap";
    case FFT3D_B200_ERR_BUSY: return "queue full";
    case FFT3D_B200_ERR_PEER: return "listed devices cannot access each other's memory";
    default: return "unknown status";
    }
}

// ------------------------------------------------------------------ reference contract, host pointers

struct fft3d_plan {
    fft3d_b200_plan *p;
};

static const char kName[] = "b200_fft3d";
static const char kDesc[] =
    "B200 sm_100a: volumes staged once in CTA shared memory (clusters + DSMEM beyond it), "
    "register codelets (PFA/CT/Rader-17), coalesced streaming stores";

extern "C" const char *fft3d_name(void) { return kName; }
extern "C" const char *fft3d_description(void) { return kDesc; }
extern "C" int fft3d_supports(int L) { return fft3d_b200_supports(L, L, L, FFT3D_B200_C128); }

extern "C" fft3d_plan *fft3d_create(int L, int batch)
{
    if (L < 1 || batch < 1) {
        set_status(FFT3D_B200_ERR_INVALID);
        return nullptr;
    }
    fft3d_b200_desc d = {L, L, L, batch, FFT3D_B200_FORWARD, FFT3D_B200_C128, 0u, -1};
    fft3d_b200_plan *p = nullptr;
    if (fft3d_b200_plan_create(&d, &p) != FFT3D_B200_OK) return nullptr;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    const int st = ensure_staging(p);  // all allocation happens in create
    if (prev >= 0) cudaSetDevice(prev);
    if (st) {
        fft3d_b200_plan_destroy(p);
        set_status(st);
        return nullptr;
    }
    fft3d_plan *h = new fft3d_plan{p};
    return h;
}

extern "C" void fft3d_execute(fft3d_plan *plan, const FFT3D_COMPLEX *in, FFT3D_COMPLEX *out)
{
    if (!plan) {
        set_status(FFT3D_B200_ERR_INVALID);
        return;
    }
    const int st = fft3d_b200_execute_host(plan->p, in, out);
    if (st != FFT3D_B200_OK)
        fprintf(stderr, "fft3d_execute: %s\n", fft3d_b200_status_string(st));
}

extern "C" void fft3d_destroy(fft3d_plan *plan)
{
    if (!plan) return;
    fft3d_b200_plan_destroy(plan->p);
    delete plan;
}

// ------------------------------------------------------------------ reference contract, device pointers

struct fft3d_gpu_plan {
    fft3d_b200_plan *p;
};

extern "C" const char *fft3d_gpu_name(void) { return kName; }
extern "C" const char *fft3d_gpu_description(void) { return kDesc; }
extern "C" int fft3d_gpu_supports(int L) { return fft3d_b200_supports(L, L, L, FFT3D_B200_C128); }

extern "C" fft3d_gpu_plan *fft3d_gpu_create(int L, int batch)
{
    if (L < 1 || batch < 1) {
        set_status(FFT3D_B200_ERR_INVALID);
        return nullptr;
    }
    fft3d_b200_desc d = {L, L, L, batch, FFT3D_B200_FORWARD, FFT3D_B200_C128, 0u, -1};
    fft3d_b200_plan *p = nullptr;
    if (fft3d_b200_plan_create(&d, &p) != FFT3D_B200_OK) return nullptr;
    return new fft3d_gpu_plan{p};
}

// Enqueued on the legacy default stream, which orders it after the caller's
// cudaMemcpy/cudaMemset on that stream, as the reference driver relies on
// (bench/gpu/driver.cu:230-253).
extern "C" void fft3d_gpu_execute(fft3d_gpu_plan *plan, const double2 *in, double2 *out)
{
    if (!plan) {
        set_status(FFT3D_B200_ERR_INVALID);
        return;
    }
    fft3d_b200_execute(plan->p, in, out, (void *)cudaStreamLegacy);
}

extern "C" void fft3d_gpu_destroy(fft3d_gpu_plan *plan)
{
    if (!plan) return;
    fft3d_b200_plan_destroy(plan->p);
    delete plan;
}

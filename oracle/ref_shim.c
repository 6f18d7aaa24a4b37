/* ref_shim.c -- persistent-thread driver around the reference's CPU code for
 * this path: its best C kernels, its textbook exemplar and FFTW 3.3.10 built
 * from its vendored source tree.
 *
 * BASELINE / TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libfft3d_best.so
 * next to the reference's own sources, and called only by bench.py (the CPU
 * baseline legs and the --impl reference arm) and tests/.
 *
 * The transforms are the reference's:
 *   REF_BEST      fft3d_best_create / _execute / _destroy
 *                 (bench/geom/best/fft3d_best.h:35-60), one plan per thread slice,
 *                 as the reference's multicore phase runs one batch slice per core;
 *   REF_TEXTBOOK  bench/geom/impl_11/baseline_matrix.c (compiled with its six
 *                 symbols renamed tb_*), one plan per thread slice;
 *   REF_FFTW      fftw_plan_many_dft over each thread's slice, the call of
 *                 bench/geom/sota/fftw3.c:43-48 with its planner flags;
 *   REF_FFTW_THREADS  one fftw_plan_many_dft over the whole batch planned with
 *                 fftw_plan_with_nthreads(nthreads), as bench/mt/sota/fftw3.c:37-48
 *                 does with its fixed 32 threads;
 *   REF_MT        one of the reference's multicore kernels (bench/mt/impl_4/L*.c,
 *                 the six symbols of bench/mt/fft3d_api.h, built one shared object
 *                 each and opened by ref_open_mt): one plan over the whole batch,
 *                 its own OpenMP threads, their count set as the reference's
 *                 harness fixes OMP_NUM_THREADS (bench/mt/fft3d_api.h "MULTICORE").
 * This file adds only the thread pool (workers created once, released by a
 * barrier for every run, so a timed run pays no thread creation), the slicing,
 * and the inverse half of a round trip: FFTW_BACKWARD plans and a 1/V scale for
 * FFTW; for the forward-only reference kernels, conjugation,
 * ifft(X) = conj(fft(conj(X))) / V.
 */
#include <complex.h>
#include <dlfcn.h>
#include <fftw3.h>
#include <omp.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "fft3d_best.h"

typedef double _Complex cplx;
typedef float _Complex cplxf;

/* The kernels of bench/geom/best/kernels, linked with their six symbols renamed
   per tag (oracle/Makefile KERNELS).  fft3d_best_create races a geometry's
   candidates in every call; with one plan per thread slice that race would run
   once per slice, so the first slice races and the others create the winner. */
#define BEST_TAGS(X) X(k6) X(k6b) X(k8) X(k8b) X(k13) X(k13b) X(k17) X(k17b) X(k23) X(k23b) \
    X(k36) X(k36b) X(k36c) X(k45) X(k45b) X(k64) X(k64b)
#define BEST_DECL(t)                                  \
    const char *t##_name(void);                       \
    void *t##_create(int L, int batch);               \
    void t##_execute(void *p, const cplx *in, cplx *out); \
    void t##_destroy(void *p);
BEST_TAGS(BEST_DECL)
struct best_kernel {
    const char *(*name)(void);
    void *(*create)(int, int);
    void (*execute)(void *, const cplx *, cplx *);
    void (*destroy)(void *);
};
#define BEST_ROW(t) {t##_name, t##_create, t##_execute, t##_destroy},
static const struct best_kernel BEST_KERNELS[] = {BEST_TAGS(BEST_ROW)};
#define NBEST ((int)(sizeof BEST_KERNELS / sizeof BEST_KERNELS[0]))

/* bench/geom/impl_11/baseline_matrix.c, renamed at compile time */
typedef struct fft3d_plan tb_plan;
tb_plan *tb_create(int L, int batch);
void tb_execute(tb_plan *p, const cplx *in, cplx *out);
void tb_destroy(tb_plan *p);

enum { REF_BEST = 0, REF_TEXTBOOK = 1, REF_FFTW = 2, REF_FFTW_THREADS = 3, REF_MT = 4 };

/* a bench/mt kernel opened by ref_open_mt */
struct mt_kernel {
    const char *(*name)(void);
    int (*supports)(int);
    void *(*create)(int, int);
    void (*execute)(void *, const cplx *, cplx *);
    void (*destroy)(void *);
};
#define MAXT 512

struct slice {
    long b0, nb;
    void *plan;                 /* best / textbook plan */
    const struct best_kernel *direct;  /* best: kernel created without the race */
    fftw_plan pf, pb;           /* FFTW slice plans, complex double */
    fftwf_plan pff, pbf;        /* complex float */
    void *tmp;
};

typedef struct ref_ctx {
    int backend, n0, n1, n2, precision, nthreads, roundtrip, effort;
    long batch, vol;
    struct slice s[MAXT];
    fftw_plan pf, pb;           /* REF_FFTW_THREADS, complex double */
    fftwf_plan pff, pbf;        /* complex float */
    void *tmp;
    const void *in;
    void *out;
    void (*job)(struct ref_ctx *, int);
    pthread_t tid[MAXT];
    struct worker_arg {
        struct ref_ctx *c;
        int t;
    } args[MAXT];
    pthread_barrier_t start, done;
    int quit;
    double plan_seconds;
    char name[160];
    struct mt_kernel mt;        /* REF_MT */
    void *mt_plan;
    int omp_threads;
} ref_ctx;

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

static unsigned effort_flag(int e)
{
    return e == 2 ? FFTW_PATIENT : e == 1 ? FFTW_MEASURE : FFTW_ESTIMATE;
}

static const char *effort_name(int e)
{
    return e == 2 ? "patient" : e == 1 ? "measure" : "estimate";
}

static size_t elem_bytes(const ref_ctx *c) { return c->precision ? sizeof(cplxf) : sizeof(cplx); }

/* ---------------------------------------------------------------- per-slice work */

static void scale_range(ref_ctx *c, void *buf, long first, long count)
{
    const double inv = 1.0 / (double)c->vol;
    if (c->precision) {
        cplxf *p = (cplxf *)buf + first;
        const float f = (float)inv;
        for (long i = 0; i < count; ++i) p[i] *= f;
    } else {
        cplx *p = (cplx *)buf + first;
        for (long i = 0; i < count; ++i) p[i] *= inv;
    }
}

static void forward_kernel(ref_ctx *c, struct slice *s, const cplx *in, cplx *out)
{
    if (s->direct) s->direct->execute(s->plan, in, out);
    else if (c->backend == REF_BEST) fft3d_best_execute((fft3d_best_plan *)s->plan, in, out);
    else tb_execute((tb_plan *)s->plan, in, out);
}

static void job_slice(ref_ctx *c, int t)
{
    struct slice *s = &c->s[t];
    if (s->nb <= 0) return;
    const long off = s->b0 * c->vol;
    const long n = s->nb * c->vol;
    if (c->backend == REF_FFTW) {
        if (c->precision) {
            const cplxf *in = (const cplxf *)c->in + off;
            cplxf *out = (cplxf *)c->out + off;
            if (!c->roundtrip) {
                fftwf_execute_dft(s->pff, (fftwf_complex *)in, (fftwf_complex *)out);
            } else {
                fftwf_execute_dft(s->pff, (fftwf_complex *)in, (fftwf_complex *)s->tmp);
                fftwf_execute_dft(s->pbf, (fftwf_complex *)s->tmp, (fftwf_complex *)out);
                scale_range(c, out, 0, n);
            }
        } else {
            const cplx *in = (const cplx *)c->in + off;
            cplx *out = (cplx *)c->out + off;
            if (!c->roundtrip) {
                fftw_execute_dft(s->pf, (fftw_complex *)in, (fftw_complex *)out);
            } else {
                fftw_execute_dft(s->pf, (fftw_complex *)in, (fftw_complex *)s->tmp);
                fftw_execute_dft(s->pb, (fftw_complex *)s->tmp, (fftw_complex *)out);
                scale_range(c, out, 0, n);
            }
        }
        return;
    }
    const cplx *in = (const cplx *)c->in + off;
    cplx *out = (cplx *)c->out + off;
    forward_kernel(c, s, in, out);
    if (c->roundtrip) {
        cplx *tmp = (cplx *)s->tmp;
        const double inv = 1.0 / (double)c->vol;
        for (long i = 0; i < n; ++i) out[i] = conj(out[i]);
        forward_kernel(c, s, out, tmp);
        for (long i = 0; i < n; ++i) out[i] = conj(tmp[i]) * inv;
    }
}

static void job_scale(ref_ctx *c, int t)
{
    const long total = c->batch * c->vol;
    const long per = (total + c->nthreads - 1) / c->nthreads;
    const long first = (long)t * per;
    if (first >= total) return;
    scale_range(c, c->out, first, first + per > total ? total - first : per);
}

/* ---------------------------------------------------------------- thread pool */

static void *worker(void *p)
{
    struct worker_arg *a = p;
    ref_ctx *c = a->c;
    for (;;) {
        pthread_barrier_wait(&c->start);
        if (c->quit) break;
        c->job(c, a->t);
        pthread_barrier_wait(&c->done);
    }
    return NULL;
}

static void pool_run(ref_ctx *c, void (*job)(ref_ctx *, int))
{
    c->job = job;
    if (c->nthreads > 1) pthread_barrier_wait(&c->start);
    job(c, 0);
    if (c->nthreads > 1) pthread_barrier_wait(&c->done);
}

static int pool_start(ref_ctx *c)
{
    if (c->nthreads <= 1) return 0;
    pthread_barrier_init(&c->start, NULL, (unsigned)c->nthreads);
    pthread_barrier_init(&c->done, NULL, (unsigned)c->nthreads);
    for (int t = 1; t < c->nthreads; ++t) {
        struct worker_arg *a = &c->args[t];
        a->c = c;
        a->t = t;
        if (pthread_create(&c->tid[t], NULL, worker, a)) return -1;
    }
    return 0;
}

/* ---------------------------------------------------------------- create / run */

static int plan_slice_fftw(ref_ctx *c, struct slice *s)
{
    const int n[3] = {c->n0, c->n1, c->n2};
    const int dist = (int)c->vol;
    const int hm = (int)s->nb;
    const unsigned fl = effort_flag(c->effort);
    const size_t bytes = (size_t)s->nb * c->vol * elem_bytes(c);
    /* plan on scratch of the same (SIMD) alignment as the callers' buffers, then
       execute on them with the new-array interface, as the reference does */
    if (c->precision) {
        fftwf_complex *a = fftwf_alloc_complex((size_t)s->nb * c->vol);
        fftwf_complex *b = fftwf_alloc_complex((size_t)s->nb * c->vol);
        s->pff = fftwf_plan_many_dft(3, n, hm, a, NULL, 1, dist, b, NULL, 1, dist, FFTW_FORWARD, fl);
        if (c->roundtrip)
            s->pbf = fftwf_plan_many_dft(3, n, hm, b, NULL, 1, dist, a, NULL, 1, dist, FFTW_BACKWARD, fl);
        fftwf_free(a);
        fftwf_free(b);
        if (!s->pff || (c->roundtrip && !s->pbf)) return -1;
    } else {
        fftw_complex *a = fftw_alloc_complex((size_t)s->nb * c->vol);
        fftw_complex *b = fftw_alloc_complex((size_t)s->nb * c->vol);
        s->pf = fftw_plan_many_dft(3, n, hm, a, NULL, 1, dist, b, NULL, 1, dist, FFTW_FORWARD, fl);
        if (c->roundtrip)
            s->pb = fftw_plan_many_dft(3, n, hm, b, NULL, 1, dist, a, NULL, 1, dist, FFTW_BACKWARD, fl);
        fftw_free(a);
        fftw_free(b);
        if (!s->pf || (c->roundtrip && !s->pb)) return -1;
    }
    if (c->roundtrip && posix_memalign(&s->tmp, 64, bytes)) return -1;
    return 0;
}

static int threads_ready;

ref_ctx *ref_open(int backend, int n0, int n1, int n2, long batch, int precision, int nthreads,
                  int roundtrip, int effort)
{
    if (n0 < 1 || n1 < 1 || n2 < 1 || batch < 1 || nthreads < 1) return NULL;
    if (backend < REF_BEST || backend > REF_FFTW_THREADS) return NULL;
    if (backend <= REF_TEXTBOOK && (n0 != n1 || n1 != n2 || precision)) return NULL;
    if (backend == REF_BEST && !fft3d_best_supports(n0)) return NULL;
    if (nthreads > MAXT) nthreads = MAXT;
    ref_ctx *c = calloc(1, sizeof *c);
    if (!c) return NULL;
    c->backend = backend;
    c->n0 = n0;
    c->n1 = n1;
    c->n2 = n2;
    c->precision = precision;
    c->roundtrip = roundtrip;
    c->effort = effort;
    c->batch = batch;
    c->vol = (long)n0 * n1 * n2;
    const double t0 = now_s();
    if (backend == REF_FFTW_THREADS) {
        c->nthreads = nthreads;
        if (!threads_ready) {
            if (!fftw_init_threads() || !fftwf_init_threads()) goto fail;
            threads_ready = 1;
        }
        fftw_plan_with_nthreads(nthreads);
        fftwf_plan_with_nthreads(nthreads);
        struct slice whole;
        memset(&whole, 0, sizeof whole);
        whole.nb = batch;
        if (plan_slice_fftw(c, &whole)) goto fail;
        c->pf = whole.pf;
        c->pb = whole.pb;
        c->pff = whole.pff;
        c->pbf = whole.pbf;
        c->tmp = whole.tmp;
        fftw_plan_with_nthreads(1);
        fftwf_plan_with_nthreads(1);
    } else {
        if (backend == REF_FFTW && threads_ready) {
            fftw_plan_with_nthreads(1);
            fftwf_plan_with_nthreads(1);
        }
        /* slices start on 64-byte boundaries of the callers' buffers
           (bench/geom/fft3d_api.h:19), so every slice is a multiple of g volumes */
        long g = 1;
        while ((g * c->vol * (long)elem_bytes(c)) % 64) ++g;
        const long units = (batch + g - 1) / g;
        if (nthreads > units) nthreads = (int)units;
        c->nthreads = nthreads;
        const long per = units / nthreads, extra = units % nthreads;
        long b0 = 0;
        for (int t = 0; t < nthreads; ++t) {
            struct slice *s = &c->s[t];
            long nb = (per + (t < extra ? 1 : 0)) * g;
            if (b0 + nb > batch) nb = batch - b0;
            s->b0 = b0;
            s->nb = nb;
            b0 += nb;
            if (nb <= 0) continue;
            if (backend == REF_FFTW) {
                if (plan_slice_fftw(c, s)) goto fail;
                continue;
            }
            if (backend == REF_BEST && t > 0) {
                /* the kernel slice 0's race chose */
                const char *won = fft3d_best_selected_name((fft3d_best_plan *)c->s[0].plan);
                for (int k = 0; k < NBEST && !s->direct; ++k)
                    if (!strcmp(BEST_KERNELS[k].name(), won)) s->direct = &BEST_KERNELS[k];
                if (!s->direct) goto fail;
                s->plan = s->direct->create(n0, (int)nb);
            } else {
                s->plan = backend == REF_BEST ? (void *)fft3d_best_create(n0, (int)nb)
                                              : (void *)tb_create(n0, (int)nb);
            }
            if (!s->plan) goto fail;
            if (roundtrip && posix_memalign(&s->tmp, 64, (size_t)nb * c->vol * sizeof(cplx))) goto fail;
        }
    }
    c->plan_seconds = now_s() - t0;
    if (backend == REF_BEST)
        snprintf(c->name, sizeof c->name, "bench/geom/best %s", fft3d_best_selected_name(c->s[0].plan));
    else if (backend == REF_TEXTBOOK)
        snprintf(c->name, sizeof c->name, "bench/geom/impl_11/baseline_matrix (textbook, O(L^4))");
    else
        snprintf(c->name, sizeof c->name, "FFTW 3.3.10 plan_many_dft %s%s, %s", precision ? "fftwf " : "",
                 effort_name(effort),
                 backend == REF_FFTW ? "one plan per thread slice" : "fftw_plan_with_nthreads");
    if (pool_start(c)) {
        /* workers already started wait on this context's barrier: it is left
           allocated (a leak on this error path only) rather than freed under them */
        return NULL;
    }
    return c;
fail:
    free(c);  /* plans leak on this error path only; the baseline then reports it */
    return NULL;
}

/* the earlier best-C entry point */
ref_ctx *ref_create(int L, long batch, int nthreads, int roundtrip)
{
    return ref_open(REF_BEST, L, L, L, batch, 0, nthreads, roundtrip, 0);
}

/* A bench/mt/impl_4 kernel from its shared object, with `nthreads` OpenMP
 * threads (complex128 cubes), one plan over the whole batch.  The kernels are
 * forward-only and tuned for whole large batches (their per-call overhead makes
 * any chunked inverse unfair to them), so a "round trip" here is charged as two
 * forward transforms of the batch, in -> tmp -> out: the cost of a round trip
 * whose inverse ran as fast as the forward, with no conjugation or scaling;
 * out is then FFT(FFT(in)) = V times the index reversal of in.  The object
 * stays loaded for the life of the process. */
ref_ctx *ref_open_mt(const char *path, int L, long batch, int nthreads, int roundtrip)
{
    if (!path || L < 1 || batch < 1 || batch > 0x7fffffffL || nthreads < 1) return NULL;
    void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return NULL;
    ref_ctx *c = calloc(1, sizeof *c);
    if (!c) return NULL;
    c->mt.name = (const char *(*)(void))dlsym(h, "fft3d_name");
    c->mt.supports = (int (*)(int))dlsym(h, "fft3d_supports");
    c->mt.create = (void *(*)(int, int))dlsym(h, "fft3d_create");
    c->mt.execute = (void (*)(void *, const cplx *, cplx *))dlsym(h, "fft3d_execute");
    c->mt.destroy = (void (*)(void *))dlsym(h, "fft3d_destroy");
    if (!c->mt.name || !c->mt.supports || !c->mt.create || !c->mt.execute || !c->mt.destroy ||
        !c->mt.supports(L))
        goto fail;
    c->backend = REF_MT;
    c->n0 = c->n1 = c->n2 = L;
    c->roundtrip = roundtrip;
    c->batch = batch;
    c->vol = (long)L * L * L;
    c->nthreads = 1;  /* no pool: the kernel runs its own threads */
    c->omp_threads = nthreads;
    omp_set_num_threads(nthreads);
    const double t0 = now_s();
    c->mt_plan = c->mt.create(L, (int)batch);
    if (!c->mt_plan) goto fail;
    if (roundtrip && posix_memalign(&c->tmp, 64, (size_t)batch * c->vol * sizeof(cplx))) goto fail;
    c->plan_seconds = now_s() - t0;
    snprintf(c->name, sizeof c->name, "bench/mt/impl_4 %s (OpenMP, %d threads)", c->mt.name(), nthreads);
    return c;
fail:
    free(c);
    return NULL;
}

int ref_run(ref_ctx *c, const void *in, void *out)
{
    if (!c) return -1;
    c->in = in;
    c->out = out;
    if (c->backend == REF_MT) {
        omp_set_num_threads(c->omp_threads);
        if (!c->roundtrip) {
            c->mt.execute(c->mt_plan, (const cplx *)in, (cplx *)out);
        } else {
            c->mt.execute(c->mt_plan, (const cplx *)in, (cplx *)c->tmp);
            c->mt.execute(c->mt_plan, (const cplx *)c->tmp, (cplx *)out);
        }
        return 0;
    }
    if (c->backend != REF_FFTW_THREADS) {
        pool_run(c, job_slice);
        return 0;
    }
    if (c->precision) {
        if (!c->roundtrip) {
            fftwf_execute_dft(c->pff, (fftwf_complex *)in, (fftwf_complex *)out);
            return 0;
        }
        fftwf_execute_dft(c->pff, (fftwf_complex *)in, (fftwf_complex *)c->tmp);
        fftwf_execute_dft(c->pbf, (fftwf_complex *)c->tmp, (fftwf_complex *)out);
    } else {
        if (!c->roundtrip) {
            fftw_execute_dft(c->pf, (fftw_complex *)in, (fftw_complex *)out);
            return 0;
        }
        fftw_execute_dft(c->pf, (fftw_complex *)in, (fftw_complex *)c->tmp);
        fftw_execute_dft(c->pb, (fftw_complex *)c->tmp, (fftw_complex *)out);
    }
    pool_run(c, job_scale);
    return 0;
}

const char *ref_kernel_name(ref_ctx *c) { return c ? c->name : ""; }
int ref_threads(ref_ctx *c) { return c ? (c->backend == REF_MT ? c->omp_threads : c->nthreads) : 0; }
double ref_plan_seconds(ref_ctx *c) { return c ? c->plan_seconds : 0.0; }

void ref_destroy(ref_ctx *c)
{
    if (!c) return;
    if (c->backend == REF_MT) {
        if (c->mt_plan) c->mt.destroy(c->mt_plan);
        free(c->tmp);
        free(c);
        return;
    }
    if (c->nthreads > 1) {
        c->quit = 1;
        pthread_barrier_wait(&c->start);
        for (int t = 1; t < c->nthreads; ++t) pthread_join(c->tid[t], NULL);
        pthread_barrier_destroy(&c->start);
        pthread_barrier_destroy(&c->done);
    }
    for (int t = 0; t < MAXT; ++t) {
        struct slice *s = &c->s[t];
        if (s->plan && s->direct) s->direct->destroy(s->plan);
        else if (s->plan && c->backend == REF_BEST) fft3d_best_destroy((fft3d_best_plan *)s->plan);
        if (s->plan && c->backend == REF_TEXTBOOK) tb_destroy((tb_plan *)s->plan);
        if (s->pf) fftw_destroy_plan(s->pf);
        if (s->pb) fftw_destroy_plan(s->pb);
        if (s->pff) fftwf_destroy_plan(s->pff);
        if (s->pbf) fftwf_destroy_plan(s->pbf);
        free(s->tmp);
    }
    if (c->pf) fftw_destroy_plan(c->pf);
    if (c->pb) fftw_destroy_plan(c->pb);
    if (c->pff) fftwf_destroy_plan(c->pff);
    if (c->pbf) fftwf_destroy_plan(c->pbf);
    free(c->tmp);
    free(c);
}

/* ref_shim.c -- multithreaded driver around the reference's best C library.
 *
 * BASELINE / TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libfft3d_best.so
 * next to the reference's own bench/geom/best sources, and called only by
 * bench.py (the CPU baseline and the --impl reference arm) and tests/.
 *
 * The transforms are the reference's (fft3d_best_create / _execute / _destroy,
 * bench/geom/best/fft3d_best.h:35-60).  This file only splits a batch into one
 * contiguous slice per host thread (each thread owns a plan for its slice, as
 * the reference's multicore phase runs one batch slice per core) and, for a round
 * trip, builds the inverse from the forward-only library by conjugation:
 * ifft(X) = conj(fft(conj(X))) / V.
 */
#include <complex.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "fft3d_best.h"

typedef double _Complex cplx;

struct slice {
    int L;
    long b0, nb;
    int roundtrip;
    fft3d_best_plan *plan;
    cplx *tmp;
    const cplx *in;
    cplx *out;
};

typedef struct ref_ctx {
    int L, nthreads, roundtrip;
    long batch;
    struct slice *s;
} ref_ctx;

ref_ctx *ref_create(int L, long batch, int nthreads, int roundtrip)
{
    if (!fft3d_best_supports(L) || batch < 1 || nthreads < 1) return NULL;
    if (nthreads > batch) nthreads = (int)batch;
    ref_ctx *c = calloc(1, sizeof *c);
    c->L = L;
    c->batch = batch;
    c->nthreads = nthreads;
    c->roundtrip = roundtrip;
    c->s = calloc((size_t)nthreads, sizeof *c->s);
    const long vol = (long)L * L * L;
    /* the reference kernels want 64-byte aligned buffers (bench/geom/fft3d_api.h:19),
       so every slice starts at a multiple of g volumes */
    long g = 1;
    while ((g * vol * (long)sizeof(cplx)) % 64) ++g;
    const long units = (batch + g - 1) / g;
    if (nthreads > units) nthreads = (int)units;
    c->nthreads = nthreads;
    long per = units / nthreads, extra = units % nthreads, b0 = 0;
    for (int t = 0; t < nthreads; ++t) {
        long nb = (per + (t < extra ? 1 : 0)) * g;
        if (b0 + nb > batch) nb = batch - b0;
        c->s[t].L = L;
        c->s[t].b0 = b0;
        c->s[t].nb = nb;
        c->s[t].roundtrip = roundtrip;
        c->s[t].plan = fft3d_best_create(L, (int)nb);
        if (roundtrip && posix_memalign((void **)&c->s[t].tmp, 64, (size_t)nb * vol * sizeof(cplx)))
            c->s[t].tmp = NULL;
        b0 += nb;
    }
    return c;
}

static void *run_slice(void *arg)
{
    struct slice *s = arg;
    const long vol = (long)s->L * s->L * s->L;
    const cplx *in = s->in + s->b0 * vol;
    cplx *out = s->out + s->b0 * vol;
    fft3d_best_execute(s->plan, in, out);
    if (s->roundtrip) {
        const long n = s->nb * vol;
        const double inv = 1.0 / (double)vol;
        for (long i = 0; i < n; ++i) out[i] = conj(out[i]);
        fft3d_best_execute(s->plan, out, s->tmp);
        for (long i = 0; i < n; ++i) out[i] = conj(s->tmp[i]) * inv;
    }
    return NULL;
}

int ref_run(ref_ctx *c, const void *in, void *out)
{
    if (!c) return -1;
    pthread_t tid[512];
    int n = c->nthreads > 512 ? 512 : c->nthreads;
    for (int t = 0; t < n; ++t) {
        c->s[t].in = in;
        c->s[t].out = out;
    }
    for (int t = 1; t < n; ++t) pthread_create(&tid[t], NULL, run_slice, &c->s[t]);
    run_slice(&c->s[0]);
    for (int t = 1; t < n; ++t) pthread_join(tid[t], NULL);
    return 0;
}

const char *ref_kernel_name(ref_ctx *c)
{
    return c && c->s[0].plan ? fft3d_best_selected_name(c->s[0].plan) : "";
}

void ref_destroy(ref_ctx *c)
{
    if (!c) return;
    for (int t = 0; t < c->nthreads; ++t) {
        if (c->s[t].plan) fft3d_best_destroy(c->s[t].plan);
        free(c->s[t].tmp);
    }
    free(c->s);
    free(c);
}

/* fft3d_oracle.c -- CPU restatement of the reference's textbook 3D FFT.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product is
 * compared against; it is imported only by tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg.  The product library never links or calls it.
 *
 * It restates, in plain C99 on double _Complex, the algorithm of the
 * reference's from-scratch Python oracle (python/fft3d.py):
 *
 *   - twiddle table exp(sign*2*pi*i*j/n), exponent reduced mod n   (fft3d.py:139-148)
 *   - direct O(n^2) DFT for primes <= DIRECT_MAX_PRIME = 11          (fft3d.py:79, :153-163)
 *   - mixed-radix decimation-in-time Cooley-Tukey, radix = smallest
 *     prime factor                                                   (fft3d.py:166-188)
 *   - Rader for primes > 11: permutation by a primitive root, cyclic
 *     correlation of length p-1 evaluated by the convolution theorem (fft3d.py:191-245)
 *   - primitive root / factorisation helpers                         (fft3d.py:86-133)
 *   - row-column n-D transform over the last three axes, batch
 *     slowest, forward unnormalised, inverse scaled by 1/V           (fft3d.py:349-423)
 *
 * Layout: element (b, i0, i1, i2) of an n0 x n1 x n2 batch lives at
 * ((b*n0 + i0)*n1 + i1)*n2 + i2, interleaved complex (bench/geom/fft3d_api.h:14-18).
 *
 * Parity of this restatement is pinned by tests/test_oracle.py against golden
 * vectors that tests/golden/make_golden.py produced by running the reference's
 * own python/fft3d.py and python/slow_dft.py.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

#define ORACLE_DIRECT_MAX_PRIME 11 /* fft3d.py:79 */

/* ------------------------------------------------------------ number theory */

/* fft3d.py:102-111 */
static int smallest_prime_factor(int n)
{
    if (n % 2 == 0) return 2;
    for (int d = 3; d * d <= n; d += 2)
        if (n % d == 0) return d;
    return n;
}

/* fft3d.py:114-116 */
static int is_prime(int n) { return n >= 2 && smallest_prime_factor(n) == n; }

static long powmod(long b, long e, long m)
{
    long r = 1 % m;
    b %= m;
    while (e > 0) {
        if (e & 1) r = (r * b) % m;
        b = (b * b) % m;
        e >>= 1;
    }
    return r;
}

/* Smallest primitive root of the prime p (fft3d.py:119-133): g has order p-1 iff
 * g^((p-1)/q) != 1 for every prime q dividing p-1. */
int oracle_primitive_root(int p)
{
    if (!is_prime(p)) return -1;
    if (p == 2) return 1;
    int qs[32], nq = 0, m = p - 1;
    for (int d = 2; d * d <= m; ++d) {
        if (m % d == 0) {
            qs[nq++] = d;
            while (m % d == 0) m /= d;
        }
    }
    if (m > 1) qs[nq++] = m;
    for (int g = 2; g < p; ++g) {
        int ok = 1;
        for (int i = 0; i < nq && ok; ++i)
            if (powmod(g, (p - 1) / qs[i], p) == 1) ok = 0;
        if (ok) return g;
    }
    return -1;
}

/* ------------------------------------------------------------ twiddles */

/* W[j] = exp(sign*2*pi*i*j/n); callers index it with exponents reduced mod n
 * (fft3d.py:139-148). */
static void twiddle_table(int n, int sign, cplx *w)
{
    for (int j = 0; j < n; ++j) {
        double a = (double)sign * 2.0 * M_PI * (double)j / (double)n;
        w[j] = cos(a) + I * sin(a);
    }
}

/* ------------------------------------------------------------ 1D routes */

static void fft_auto(const cplx *x, cplx *out, int n, int sign);

/* The definition, O(n^2) (fft3d.py:153-163). */
static void dft_direct(const cplx *x, cplx *out, int n, int sign)
{
    cplx *w = malloc((size_t)n * sizeof *w);
    twiddle_table(n, sign, w);
    for (int k = 0; k < n; ++k) {
        cplx acc = 0.0;
        for (int j = 0; j < n; ++j) acc += x[j] * w[((long)j * k) % n];
        out[k] = acc;
    }
    free(w);
}

/* Decimation in time with r = smallest prime factor (fft3d.py:166-188):
 * X[k] = sum_a W_n^{ak} Y_a[k mod m], Y_a = length-m transform of x[a::r]. */
static void fft_mixed_radix(const cplx *x, cplx *out, int n, int sign)
{
    int r = smallest_prime_factor(n);
    int m = n / r;
    cplx *sub = malloc((size_t)n * sizeof *sub); /* sub[a*m + t] */
    cplx *tmp = malloc((size_t)m * sizeof *tmp);
    for (int a = 0; a < r; ++a) {
        for (int t = 0; t < m; ++t) tmp[t] = x[a + r * t];
        fft_auto(tmp, sub + (size_t)a * m, m, sign);
    }
    cplx *w = malloc((size_t)n * sizeof *w);
    twiddle_table(n, sign, w);
    for (int k = 0; k < n; ++k) {
        cplx acc = 0.0;
        for (int a = 0; a < r; ++a) acc += w[((long)a * k) % n] * sub[(size_t)a * m + (k % m)];
        out[k] = acc;
    }
    free(w);
    free(tmp);
    free(sub);
}

/* Cyclic convolution by the convolution theorem (fft3d.py:191-201). */
static void cyclic_convolution(const cplx *u, const cplx *v, cplx *out, int m)
{
    cplx *fu = malloc((size_t)m * sizeof *fu);
    cplx *fv = malloc((size_t)m * sizeof *fv);
    fft_auto(u, fu, m, -1);
    fft_auto(v, fv, m, -1);
    for (int i = 0; i < m; ++i) fu[i] *= fv[i];
    fft_auto(fu, out, m, +1);
    for (int i = 0; i < m; ++i) out[i] /= (double)m;
    free(fu);
    free(fv);
}

/* Rader (fft3d.py:204-245): for prime p with primitive root g,
 * X[g^-s] = x[0] + sum_q x[g^q] W^{g^(q-s)}, a length p-1 cyclic correlation. */
static void fft_rader(const cplx *x, cplx *out, int p, int sign)
{
    if (p == 2) { dft_direct(x, out, p, sign); return; }
    int m = p - 1;
    int g = oracle_primitive_root(p);
    int *powers = malloc((size_t)m * sizeof *powers);
    long value = 1;
    for (int q = 0; q < m; ++q) { powers[q] = (int)value; value = (value * g) % p; }
    cplx *w = malloc((size_t)p * sizeof *w);
    twiddle_table(p, sign, w);
    cplx *a = malloc((size_t)m * sizeof *a);
    cplx *b = malloc((size_t)m * sizeof *b);
    cplx *brev = malloc((size_t)m * sizeof *brev);
    cplx *c = malloc((size_t)m * sizeof *c);
    for (int q = 0; q < m; ++q) { a[q] = x[powers[q]]; b[q] = w[powers[q]]; }
    for (int t = 0; t < m; ++t) brev[t] = b[((-t) % m + m) % m];
    cyclic_convolution(a, brev, c, m);
    cplx s = 0.0;
    for (int j = 0; j < p; ++j) s += x[j];
    out[0] = s;
    for (int q = 0; q < m; ++q) {
        long k = powmod(g, (long)((m - q) % m), p); /* g^-q mod p */
        out[k] = x[0] + c[q];
    }
    free(c); free(brev); free(b); free(a); free(w); free(powers);
}

/* Route by length (fft3d.py:286-295). */
static void fft_auto(const cplx *x, cplx *out, int n, int sign)
{
    if (n == 1) { out[0] = x[0]; return; }
    if (!is_prime(n)) { fft_mixed_radix(x, out, n, sign); return; }
    if (n <= ORACLE_DIRECT_MAX_PRIME) { dft_direct(x, out, n, sign); return; }
    fft_rader(x, out, n, sign);
}

/* ------------------------------------------------------------ public entry points */

/* 1D transform of n interleaved complex values (fft3d.py:300-334, auto route).
 * Returns 0, or -1 for an invalid argument. */
int oracle_fft1d(int n, int sign, const double *in, double *out)
{
    if (n < 1 || (sign != -1 && sign != 1) || !in || !out) return -1;
    fft_auto((const cplx *)in, (cplx *)out, n, sign);
    return 0;
}

struct job {
    int n[3];
    long b0, b1;
    int sign;
    double scale;
    const cplx *in;
    cplx *out;
};

/* Row-column over axes 0, 1, 2 of each volume in [b0, b1) (fft3d.py:349-399). */
static void *run_volumes(void *arg)
{
    struct job *jb = arg;
    const int n0 = jb->n[0], n1 = jb->n[1], n2 = jb->n[2];
    const size_t vol = (size_t)n0 * n1 * n2;
    int nmax = n0 > n1 ? n0 : n1;
    if (n2 > nmax) nmax = n2;
    cplx *line = malloc((size_t)nmax * sizeof *line);
    cplx *res = malloc((size_t)nmax * sizeof *res);
    for (long b = jb->b0; b < jb->b1; ++b) {
        cplx *v = jb->out + (size_t)b * vol;
        memcpy(v, jb->in + (size_t)b * vol, vol * sizeof *v);
        for (int axis = 0; axis < 3; ++axis) {
            const int n = jb->n[axis];
            const size_t stride = axis == 0 ? (size_t)n1 * n2 : (axis == 1 ? (size_t)n2 : 1);
            /* the two other axes enumerate the lines */
            const int oa = axis == 0 ? n1 : n0;
            const int ob = axis == 2 ? n1 : n2;
            for (int i = 0; i < oa; ++i) {
                for (int j = 0; j < ob; ++j) {
                    size_t base;
                    if (axis == 0) base = (size_t)i * n2 + j;
                    else if (axis == 1) base = (size_t)i * n1 * n2 + j;
                    else base = ((size_t)i * n1 + j) * n2;
                    for (int t = 0; t < n; ++t) line[t] = v[base + t * stride];
                    fft_auto(line, res, n, jb->sign);
                    for (int t = 0; t < n; ++t) v[base + t * stride] = res[t];
                }
            }
        }
        if (jb->scale != 1.0)
            for (size_t e = 0; e < vol; ++e) v[e] *= jb->scale;
    }
    free(res);
    free(line);
    return NULL;
}

static int run_batch(int n0, int n1, int n2, long batch, int sign, double scale,
                     const double *in, double *out, int nthreads)
{
    if (n0 < 1 || n1 < 1 || n2 < 1 || batch < 0 || !in || !out) return -1;
    if (sign != -1 && sign != 1) return -1;
    if (batch == 0) return 0;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > batch) nthreads = (int)batch;
    if (nthreads > 256) nthreads = 256;
    struct job jobs[256];
    pthread_t tid[256];
    long per = batch / nthreads, extra = batch % nthreads, start = 0;
    for (int t = 0; t < nthreads; ++t) {
        long cnt = per + (t < extra ? 1 : 0);
        jobs[t] = (struct job){{n0, n1, n2}, start, start + cnt, sign, scale,
                               (const cplx *)in, (cplx *)out};
        start += cnt;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&tid[t], NULL, run_volumes, &jobs[t]);
    run_volumes(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(tid[t], NULL);
    return 0;
}

/* Unnormalised transform with exponent sign `sign` (-1 forward, +1 backward) of a
 * batch of n0 x n1 x n2 volumes (fft3d.py:360-399 with axes (-3,-2,-1)). */
int oracle_fft3d(int n0, int n1, int n2, long batch, int sign, const double *in,
                 double *out, int nthreads)
{
    return run_batch(n0, n1, n2, batch, sign, 1.0, in, out, nthreads);
}

/* Inverse with the 1/(n0*n1*n2) normalisation (fft3d.py:402-407, :418-423). */
int oracle_ifft3d(int n0, int n1, int n2, long batch, const double *in, double *out,
                  int nthreads)
{
    return run_batch(n0, n1, n2, batch, +1, 1.0 / ((double)n0 * n1 * n2), in, out, nthreads);
}

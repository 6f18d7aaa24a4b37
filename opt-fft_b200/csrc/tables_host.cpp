// tables_host.cpp -- plan-time twiddle and Rader-kernel tables (host side).
//
// fft3d_create() does all table work (bench/geom/fft3d_api.h:30-32): the
// cos/sin(2*pi*e/N) table for every extent N <= 64 with the exponent reduced mod N
// (python/fft3d.py:139-148), and the Rader-17 kernel spectrum
// K = FFT16(brev)/16 with brev[t] = W17^{3^-t} (python/fft3d.py:229-238), and the
// residues of the cosine kernel c[m] = cos(2*pi*3^m/17) that dft17_crt multiplies
// by (mod x-1 and x+1 scaled 1/8, mod x^2+1 scaled 1/4, mod x^4+1 scaled 1/2), are
// evaluated in x87 extended precision, rounded once to double and to float, and
// copied by tables.cu to __constant__ memory of each device the first time a plan
// is created on it.
#include <math.h>
#include <mutex>

#include "codelets.cuh"

double2 h_tw_d[fft3d::TW_ENTRIES];
float2 h_tw_f[fft3d::TW_ENTRIES];
double2 h_rader17_d[fft3d::RADER17_ENTRIES];
float2 h_rader17_f[fft3d::RADER17_ENTRIES];
double h_crt17_d[fft3d::CRT17_ENTRIES];
float h_crt17_f[fft3d::CRT17_ENTRIES];
double2 h_twbig_d[fft3d::TWBIG_ENTRIES];
float2 h_twbig_f[fft3d::TWBIG_ENTRIES];

namespace fft3d {

static const long double kTwoPi = 6.283185307179586476925286766559005768L;

// cos/sin(2*pi*e/n) with the values that are exact in binary produced exactly.
static void exact_cis(long e, long n, long double *c, long double *s)
{
    e %= n;
    if (e < 0) e += n;
    if (e == 0) { *c = 1.0L; *s = 0.0L; return; }
    if (4 * e == n) { *c = 0.0L; *s = 1.0L; return; }
    if (2 * e == n) { *c = -1.0L; *s = 0.0L; return; }
    if (4 * e == 3 * n) { *c = 0.0L; *s = -1.0L; return; }
    const long double a = kTwoPi * (long double)e / (long double)n;
    *c = cosl(a);
    *s = sinl(a);
}

static std::once_flag g_host_once;

static void fill_host_tables()
{
    for (int n = 1; n <= TW_MAXN; ++n) {
        for (int e = 0; e < n; ++e) {
            long double c, s;
            exact_cis(e, n, &c, &s);
            h_tw_d[tw_off(n) + e] = make_double2((double)c, (double)s);
            h_tw_f[tw_off(n) + e] = make_float2((float)c, (float)s);
        }
    }
    for (int n : {96, 128, 192, 256, 83, 97}) {
        for (int e = 0; e < n; ++e) {
            long double c, s;
            exact_cis(e, n, &c, &s);
            h_twbig_d[twbig_off(n) + e] = make_double2((double)c, (double)s);
            h_twbig_f[twbig_off(n) + e] = make_float2((float)c, (float)s);
        }
    }
    // Rader-17 kernel spectra for both exponent signs.
    int pw[16];
    pw[0] = 1;
    for (int q = 1; q < 16; ++q) pw[q] = (pw[q - 1] * 3) % 17;
    for (int si = 0; si < 2; ++si) {
        const int sign = si == 0 ? -1 : +1;
        long double br[16], bi[16];
        for (int t = 0; t < 16; ++t) {
            long double c, s;
            exact_cis(pw[(16 - t) % 16], 17, &c, &s);  // W17^{g^-t}
            br[t] = c;
            bi[t] = sign * s;
        }
        for (int k = 0; k < 16; ++k) {
            long double re = 0.0L, im = 0.0L;
            for (int t = 0; t < 16; ++t) {
                long double c, s;
                exact_cis((long)t * k, 16, &c, &s);  // exp(-2*pi*i*t*k/16) = c - i s
                re += br[t] * c + bi[t] * s;
                im += bi[t] * c - br[t] * s;
            }
            re /= 16.0L;
            im /= 16.0L;
            h_rader17_d[si * 16 + k] = make_double2((double)re, (double)im);
            h_rader17_f[si * 16 + k] = make_float2((float)re, (float)im);
        }
    }
    // CRT-17 cosine-kernel residues
    long double c[8];
    for (int m = 0; m < 8; ++m) {
        long double s;
        exact_cis(pw[m], 17, &c[m], &s);
    }
    long double P[4], Q[4];
    for (int i = 0; i < 4; ++i) {
        P[i] = c[i] + c[i + 4];  // mod x^4 - 1
        Q[i] = c[i] - c[i + 4];  // mod x^4 + 1
    }
    const long double P10 = P[0] + P[2], P11 = P[1] + P[3];  // mod x^2 - 1
    const long double res[8] = {(P10 + P11) / 8.0L, (P10 - P11) / 8.0L,      // mod x - 1, x + 1
                                (P[0] - P[2]) / 4.0L, (P[1] - P[3]) / 4.0L,  // mod x^2 + 1
                                Q[0] / 2.0L, Q[1] / 2.0L, Q[2] / 2.0L, Q[3] / 2.0L};
    for (int i = 0; i < 8; ++i) {
        h_crt17_d[i] = (double)res[i];
        h_crt17_f[i] = (float)res[i];
    }
}

void ensure_host_tables() { std::call_once(g_host_once, fill_host_tables); }

}  // namespace fft3d

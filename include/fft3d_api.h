/* fft3d_api.h -- host-pointer C ABI of the batched 3D complex FFT.
 *
 * Exactly the six entry points of the reference contract
 * bench/geom/fft3d_api.h:49-66 (wdetmold/opt-fft), so the reference's CPU timing
 * driver (bench/geom/driver.c) links libfft3d_b200.so as one more backend:
 *
 *   out[b][k0][k1][k2] = sum_j in[b][j0][j1][j2] exp(-2*pi*i (k0 j0 + k1 j1 + k2 j2) / L)
 *
 * forward, unnormalised, complex double, cube L^3, batch slowest; element
 * (b, x, y, z) at ((b*L + x)*L + y)*L + z; out-of-place, `in` not modified.
 * fft3d_create does all precomputation (tables, kernel choice, device buffers,
 * pinned staging); fft3d_execute copies the batch to the GPU, transforms it and
 * copies it back before returning, and is repeatable bit for bit.
 * Anisotropic extents, the inverse, complex64 and status returns are in
 * fft3d_b200.h.
 */
#ifndef FFT3D_API_H
#define FFT3D_API_H

#ifdef __cplusplus
extern "C" {
typedef struct fft3d_c128 { double re, im; } fft3d_c128; /* layout of C99 double _Complex */
#define FFT3D_COMPLEX fft3d_c128
#else
#include <complex.h>
#define FFT3D_COMPLEX double _Complex
#endif

typedef struct fft3d_plan fft3d_plan;

/* Results key: "b200_fft3d".  bench/geom/fft3d_api.h:51-52 */
const char *fft3d_name(void);

/* One-line technique description.  bench/geom/fft3d_api.h:54-55 */
const char *fft3d_description(void);

/* Nonzero when a cube of side L is supported.  bench/geom/fft3d_api.h:57-58 */
int fft3d_supports(int L);

/* All setup; NULL when L is unsupported or setup failed (the reason is in
 * fft3d_b200_last_status()).  bench/geom/fft3d_api.h:60-61 */
fft3d_plan *fft3d_create(int L, int batch);

/* Forward transform of the whole batch, host pointers, synchronous.
 * bench/geom/fft3d_api.h:63-64 */
void fft3d_execute(fft3d_plan *plan, const FFT3D_COMPLEX *in, FFT3D_COMPLEX *out);

/* bench/geom/fft3d_api.h:66 */
void fft3d_destroy(fft3d_plan *plan);

#ifdef __cplusplus
}
#endif

#endif /* FFT3D_API_H */

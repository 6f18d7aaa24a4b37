/* fft3d_gpu_api.h -- device-pointer C ABI of the batched 3D complex FFT.
 *
 * The six entry points of the reference's single-GPU contract
 * bench/gpu/fft3d_gpu_api.h:57-83 (wdetmold/opt-fft), so its GPU timing driver
 * (bench/gpu/driver.cu) links libfft3d_b200.so unchanged.  Same mathematics and
 * layout as fft3d_api.h; `in` and `out` are distinct cudaMalloc'd buffers of
 * double2 {re, im}.  Execute is asynchronous: it enqueues on the plan's stream,
 * which synchronises with the legacy default stream, and returns; the caller
 * synchronises (bench/gpu/fft3d_gpu_api.h:75-77).  A kernel fault is reported by
 * cudaGetLastError() as the contract requires (bench/gpu/fft3d_gpu_api.h:46-50),
 * and the status of the call by fft3d_b200_last_status().
 */
#ifndef FFT3D_GPU_API_H
#define FFT3D_GPU_API_H

#include <vector_types.h> /* double2 */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fft3d_gpu_plan fft3d_gpu_plan;

/* bench/gpu/fft3d_gpu_api.h:63-64 */
const char *fft3d_gpu_name(void);

/* bench/gpu/fft3d_gpu_api.h:66-67 */
const char *fft3d_gpu_description(void);

/* bench/gpu/fft3d_gpu_api.h:69-70 */
int fft3d_gpu_supports(int L);

/* bench/gpu/fft3d_gpu_api.h:72-73 */
fft3d_gpu_plan *fft3d_gpu_create(int L, int batch);

/* bench/gpu/fft3d_gpu_api.h:75-77 */
void fft3d_gpu_execute(fft3d_gpu_plan *plan, const double2 *in, double2 *out);

/* bench/gpu/fft3d_gpu_api.h:79 */
void fft3d_gpu_destroy(fft3d_gpu_plan *plan);

#ifdef __cplusplus
}
#endif

#endif /* FFT3D_GPU_API_H */

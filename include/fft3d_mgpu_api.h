/* fft3d_mgpu_api.h -- multi-GPU C ABI of the 3D complex FFT (one process, n GPUs).
 *
 * The eight entry points of the reference's multi-GPU contract
 * bench/mgpu/fft3d_mgpu_api.h:70-95 (wdetmold/opt-fft), so its driver
 * (bench/mgpu/driver.cu) links libfft3d_b200.so unchanged: forward, unnormalised
 * complex-double DFT of a batch of L^3 cubes distributed over `ngpus` GPUs of
 * one node.  Host layout of upload() and download(): element (b, x, y, z) at
 * ((b*L + x)*L + y)*L + z, interleaved double2 {re, im}.
 *
 * Decomposition: GPU g holds x-slab g (planes [g*L/n, (g+1)*L/n)) of every
 * volume; its kernel transforms z and y and stores each point into the GPU that
 * owns the point's y range (peer stores: the all-to-all is fused into the
 * kernel), then each GPU transforms x over its y-slab.  execute() is
 * asynchronous and idempotent (it reads the uploaded input and writes the plan's
 * output buffers); download() waits for it.  Supported: L in {36, 45, 64, 96,
 * 128, 192, 256} with L divisible by ngpus, ngpus <= 16; the same device may
 * appear more than once.  For L >= 96 (lines spread over 8 or 16 lanes, planes
 * larger than shared memory) the z pass runs first into a per-GPU buffer and the
 * exchange is fused into the y pass instead.
 */
#ifndef FFT3D_MGPU_API_H
#define FFT3D_MGPU_API_H

#include <vector_types.h> /* double2 */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fft3d_mgpu_plan fft3d_mgpu_plan;

/* bench/mgpu/fft3d_mgpu_api.h:72-73 */
const char *fft3d_mgpu_name(void);

/* bench/mgpu/fft3d_mgpu_api.h:75-76 */
const char *fft3d_mgpu_description(void);

/* bench/mgpu/fft3d_mgpu_api.h:78-79: nonzero if a cube of side L can be split
 * over exactly `ngpus` GPUs. */
int fft3d_mgpu_supports(int L, int ngpus);

/* bench/mgpu/fft3d_mgpu_api.h:81-83: all setup (buffers, streams, events, peer
 * access, tables).  `devices` lists the CUDA ordinals, length ngpus.  NULL if
 * unsupported or if a device, an allocation or peer access fails; the reason is
 * then fft3d_b200_last_status() (fft3d_b200.h): FFT3D_B200_ERR_PEER when two
 * distinct listed devices cannot access each other's memory (checked for every
 * pair before anything is allocated), FFT3D_B200_ERR_INVALID for an ordinal
 * that is not a visible device. */
fft3d_mgpu_plan *fft3d_mgpu_create(int L, int batch, int ngpus, const int *devices);

/* Extension, no counterpart in the reference: `inverse` nonzero builds the
 * inverse transform (sign +1, scaled by 1/L^3); fft3d_mgpu_create is
 * fft3d_mgpu_create_ex(..., 0). */
fft3d_mgpu_plan *fft3d_mgpu_create_ex(int L, int batch, int ngpus, const int *devices, int inverse);

/* bench/mgpu/fft3d_mgpu_api.h:85-86: distribute the host batch (synchronous). */
void fft3d_mgpu_upload(fft3d_mgpu_plan *plan, const double2 *host);

/* bench/mgpu/fft3d_mgpu_api.h:88-90: transform the uploaded input into the
 * plan's output buffers (asynchronous, idempotent). */
void fft3d_mgpu_execute(fft3d_mgpu_plan *plan);

/* bench/mgpu/fft3d_mgpu_api.h:92-93: gather the result in canonical order. */
void fft3d_mgpu_download(fft3d_mgpu_plan *plan, double2 *host);

/* bench/mgpu/fft3d_mgpu_api.h:95 */
void fft3d_mgpu_destroy(fft3d_mgpu_plan *plan);

#ifdef __cplusplus
}
#endif

#endif /* FFT3D_MGPU_API_H */

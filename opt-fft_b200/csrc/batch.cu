// batch.cu -- descriptor-list batches of uneven geometry (persistent launch).
#include "../../include/fft3d_b200.h"
#include "internal.h"

struct fft3d_b200_batch {
    int dummy;
};

extern "C" int fft3d_b200_batch_create(const fft3d_b200_segment *segs, int nseg, unsigned flags,
                                       int device, fft3d_b200_batch **out)
{
    (void)segs; (void)nseg; (void)flags; (void)device;
    if (out) *out = nullptr;
    return FFT3D_B200_ERR_UNSUPPORTED;
}

extern "C" int fft3d_b200_batch_execute(fft3d_b200_batch *b, void *stream)
{
    (void)b; (void)stream;
    return FFT3D_B200_ERR_UNSUPPORTED;
}

extern "C" void fft3d_b200_batch_destroy(fft3d_b200_batch *b) { delete b; }

extern "C" const char *fft3d_b200_batch_describe(const fft3d_b200_batch *b)
{
    (void)b;
    return "";
}

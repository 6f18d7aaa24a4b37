// mgpu.cuh -- data layout of the multi-GPU slab decomposition (host and device).
//
// One L^3 volume batch over n GPUs (bench/mgpu/fft3d_mgpu_api.h), n | L, S = L/n:
//   input on GPU g   [B][S][L][L]  x-slab g: planes x in [g*S, (g+1)*S), as uploaded
//   middle on GPU h  [B][L][S][L]  y-slab h: rows y in [h*S, (h+1)*S) of every plane
//   output on GPU h  [B][L][S][L]  y-slab h of the transform (kx, ky in slab h, kz)
// GPU g transforms the z and y lines of its planes and stores every point (x, y, z)
// straight into the middle buffer of GPU y / S (peer stores over NVLink): the
// all-to-all is the epilogue of that kernel.  GPU h then transforms the x lines of
// its y-slab.  download() gathers the y-slabs into canonical C order.
#pragma once

#include "volume.cuh"

namespace fft3d {

struct MgpuShape {
    int L, n, S;  // cube side, GPUs, slab thickness L / n
};

// Destination of point (x_local, y, z) of plane p = b*S + x_local of GPU g:
// sets *h (owner GPU) and returns the element offset in h's middle buffer.
FFT_HD long long mgpu_mid_offset(const MgpuShape &m, int g, long long p, int y, int z, int *h)
{
    const long long b = p / m.S;
    const int xl = (int)(p % m.S);
    const int x = g * m.S + xl;
    *h = y / m.S;
    const int yl = y % m.S;
    return ((b * m.L + x) * m.S + yl) * (long long)m.L + z;
}

// Offset of point (x, yl, z) of volume b in a y-slab buffer (middle or output).
FFT_HD long long mgpu_yslab_offset(const MgpuShape &m, long long b, int x, int yl, int z)
{
    return ((b * m.L + x) * m.S + yl) * (long long)m.L + z;
}

}  // namespace fft3d

// tables.cu -- device copies of the plan-time tables (see tables_host.cpp).
#include <mutex>

#include "codelets.cuh"
#include "internal.h"

__constant__ double2 c_tw_d[fft3d::TW_ENTRIES];
__constant__ float2 c_tw_f[fft3d::TW_ENTRIES];
__constant__ double2 c_rader17_d[fft3d::RADER17_ENTRIES];
__constant__ float2 c_rader17_f[fft3d::RADER17_ENTRIES];
__constant__ double c_crt17_d[fft3d::CRT17_ENTRIES];
__constant__ float c_crt17_f[fft3d::CRT17_ENTRIES];
__device__ double2 g_twbig_d[fft3d::TWBIG_ENTRIES];
__device__ float2 g_twbig_f[fft3d::TWBIG_ENTRIES];

namespace fft3d {

static std::mutex g_dev_mu;
static bool g_dev_done[64];

int ensure_device_tables(int device)
{
    ensure_host_tables();
    std::lock_guard<std::mutex> lk(g_dev_mu);
    if (device < 0 || device >= 64) return FFT3D_B200_ERR_CUDA;
    if (g_dev_done[device]) return FFT3D_B200_OK;
    if (cudaMemcpyToSymbol(c_tw_d, h_tw_d, sizeof(h_tw_d)) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    if (cudaMemcpyToSymbol(c_tw_f, h_tw_f, sizeof(h_tw_f)) != cudaSuccess) return FFT3D_B200_ERR_CUDA;
    if (cudaMemcpyToSymbol(c_rader17_d, h_rader17_d, sizeof(h_rader17_d)) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    if (cudaMemcpyToSymbol(c_rader17_f, h_rader17_f, sizeof(h_rader17_f)) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    if (cudaMemcpyToSymbol(c_crt17_d, h_crt17_d, sizeof(h_crt17_d)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_crt17_f, h_crt17_f, sizeof(h_crt17_f)) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    if (cudaMemcpyToSymbol(g_twbig_d, h_twbig_d, sizeof(h_twbig_d)) != cudaSuccess ||
        cudaMemcpyToSymbol(g_twbig_f, h_twbig_f, sizeof(h_twbig_f)) != cudaSuccess)
        return FFT3D_B200_ERR_CUDA;
    if (tc_tables_upload() != FFT3D_B200_OK) return FFT3D_B200_ERR_CUDA;
    g_dev_done[device] = true;
    return FFT3D_B200_OK;
}

}  // namespace fft3d

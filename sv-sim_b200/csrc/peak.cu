// Live measurement of the FP64 tensor-core rate (mma.sync m8n8k4 f64), the bound of the
// pair engine's blocks.  Each warp runs 8 independent accumulator chains in registers, so
// the loop is limited by the FP64 MMA pipe alone; the result is reported next to the pair
// kernel's achieved rate.
#include <string>

#include "svb_internal.h"

namespace svb {
namespace {

__global__ void __launch_bounds__(256) k_dmma_peak(double* __restrict__ out, int iters, double x, double y)
{
    double c[8][2];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        c[i][0] = threadIdx.x * 1e-3 + i;
        c[i][1] = i;
    }
    const double a = x + threadIdx.x * 1e-6, b = y;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(c[i][0]), "+d"(c[i][1])
                         : "d"(a), "d"(b));
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += c[i][0] + c[i][1];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace svb

using namespace svb;

extern "C" svb_status svb_fp64_mma_peak(int device, double* tflops)
{
    if (!tflops) { set_error("svb_fp64_mma_peak: tflops is NULL"); return SVB_ERR_INVALID; }
    *tflops = 0.0;
    int sms = 0;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int grid = sms * 4, iters = 8192;
    double* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&out, (size_t)grid * 256 * sizeof(double));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0.f;
    if (e == cudaSuccess) {
        k_dmma_peak<<<grid, 256>>>(out, 64, 0.999, 1e-3);            // warm-up
        cudaEventRecord(e0);
        k_dmma_peak<<<grid, 256>>>(out, iters, 0.999, 1e-3);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0.f) {
        set_error(std::string("svb_fp64_mma_peak: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return SVB_ERR_CUDA;
    }
    // 8 x 8 x 4 multiply-adds per warp MMA, 8 MMAs per iteration, 8 warps per CTA
    const double flops = 2.0 * 256.0 * 8.0 * iters * (double)grid * 8.0;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return SVB_OK;
}

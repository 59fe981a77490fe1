// Live measurements reported beside the kernels they bound (no reference counterpart):
//  * the FP64 tensor-core rate (mma.sync m8n8k4 f64), the bound of the pair engine's
//    blocks.  Each warp runs 8 independent accumulator chains in registers, so the loop is
//    limited by the FP64 MMA pipe alone;
//  * the L2 copy bandwidth, the bound of states that fit in L2 (n <= 22 FP64): a copy
//    between two 16 MiB buffers, read with ld.global.cg (L2, not L1) and repeated inside
//    one launch.
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

constexpr size_t L2_PROBE_ELEMS = (16u << 20) / sizeof(double2);    // 16 MiB per buffer

__global__ void __launch_bounds__(256) k_l2_copy(const double2* __restrict__ a, double2* __restrict__ b,
                                                 size_t count, int reps)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; r++) {
        const double2* src = (r & 1) ? b : a;
        double2* dst = (r & 1) ? const_cast<double2*>(a) : b;
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
            dst[i] = __ldcg(src + i);
        __syncthreads();
    }
}

}  // namespace
}  // namespace svb

using namespace svb;

extern "C" svb_status svb_l2_copy_peak(int device, double* gbs)
{
    if (!gbs) { set_error("svb_l2_copy_peak: gbs is NULL"); return SVB_ERR_INVALID; }
    *gbs = 0.0;
    int sms = 0;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double2* buf = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&buf, 2 * L2_PROBE_ELEMS * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemset(buf, 0, 2 * L2_PROBE_ELEMS * sizeof(double2));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const int reps = 64;
    float best = 0.f;
    if (e == cudaSuccess) {
        const int grid = sms * 8;
        k_l2_copy<<<grid, 256>>>(buf, buf + L2_PROBE_ELEMS, L2_PROBE_ELEMS, 4);   // warm-up
        for (int trial = 0; trial < 3 && e == cudaSuccess; trial++) {
            float ms = 0.f;
            cudaEventRecord(e0);
            k_l2_copy<<<grid, 256>>>(buf, buf + L2_PROBE_ELEMS, L2_PROBE_ELEMS, reps);
            cudaEventRecord(e1);
            e = cudaEventSynchronize(e1);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && ms > 0.f && (best == 0.f || ms < best)) best = ms;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    if (e != cudaSuccess || best <= 0.f) {
        set_error(std::string("svb_l2_copy_peak: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return SVB_ERR_CUDA;
    }
    // each repetition reads and writes one 16 MiB buffer
    *gbs = 2.0 * (double)(L2_PROBE_ELEMS * sizeof(double2)) * reps / (best * 1e-3) / 1e9;
    return SVB_OK;
}

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

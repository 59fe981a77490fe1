// Self-test of the bounded device waits (svb_selftest_waits): every wait of the
// persistent kernels on another warp, the tensor core or another block has a time limit
// after which it records an error and returns, so a lost arrival ends in an error status
// on the host rather than a hung GPU.  Here each kind of wait is made to run out on
// purpose — an mbarrier that nothing arrives at, a grid barrier whose count is never
// reached — and the host checks that it gave up, reported it, and left the context usable.
#include <string>

#include "svb_internal.h"
#include "tc_common.cuh"

namespace svb {
namespace {

// one thread waits (bounded, as the fused kernels' completion waits) on an mbarrier that
// expects one arrival which never comes
__global__ void k_mbarrier_probe(int* flag)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) *flag = mbar_wait(&bar, 0) ? 0 : 1;
}

}  // namespace

cudaError_t launch_mbarrier_probe(int* flag, cudaStream_t s)
{
    k_mbarrier_probe<<<1, 32, 0, s>>>(flag);
    return cudaGetLastError();
}

}  // namespace svb

using namespace svb;

extern "C" svb_status svb_selftest_waits(int device, int* mbar_timed_out, int* grid_timed_out)
{
    if (!mbar_timed_out || !grid_timed_out) {
        set_error("svb_selftest_waits: NULL output");
        return SVB_ERR_INVALID;
    }
    *mbar_timed_out = 0;
    *grid_timed_out = 0;
    cudaError_t e = cudaSetDevice(device);
    unsigned* words = nullptr;                 // [0] mbarrier flag (int), [1..2] grid barrier
    if (e == cudaSuccess) e = cudaMalloc(&words, 4 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(words, 0, 4 * sizeof(unsigned));
    if (e == cudaSuccess) e = launch_mbarrier_probe(reinterpret_cast<int*>(words), 0);
    if (e == cudaSuccess) e = launch_grid_barrier_probe(words + 1, 0);
    unsigned host[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(host, words, sizeof(host), cudaMemcpyDeviceToHost);
    cudaFree(words);
    if (e != cudaSuccess) {
        set_error(std::string("svb_selftest_waits: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return SVB_ERR_CUDA;
    }
    *mbar_timed_out = host[0] == 1u ? 1 : 0;
    *grid_timed_out = host[2] != 0u ? 1 : 0;   // bar[1] of the probe's barrier words
    return SVB_OK;
}

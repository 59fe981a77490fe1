// Pair engine kernel: FP64 two-qubit blocks on the FP64 tensor cores (mma.sync m16n8k8),
// one launch per pass (pairs.cpp).  Persistent CTAs of 256 threads each take tiles of
// 4,096 amplitudes; the per-tile machinery is in pairs_core.cuh.
#include "pairs_core.cuh"

namespace svb {
namespace {

__global__ void __launch_bounds__(PR_THREADS, 2)
k_pairs(double2* __restrict__ sv, const PairPass* __restrict__ passes, const PairOp* __restrict__ ops,
        const DevStage* __restrict__ layouts, const double2* __restrict__ gates, int pass_index,
        uint64_t tiles)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    __shared__ PairPass sP;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(passes + pass_index);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sP);
        for (int w = tid; w < (int)(sizeof(PairPass) / 4); w += PR_THREADS) dst[w] = src[w];
        __syncthreads();
    }
    const PairPass& P = sP;
    const PairStaged S = pair_stage(smem_raw, P, ops, layouts, gates, tid);
    PairGOffs gin, gout;
    pair_goffs(S.lay[0], P.local_q, tid, gin);
    pair_goffs(S.lay[S.n_lay - 1], P.local_q, tid, gout);
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x)
        pair_tile(sv, sm, P, S, gin, gout, tile, tid, lane);
}

}  // namespace

cudaError_t launch_pair_pass(void* state, int n, int pass_index, const DevPairBuffers& b, cudaStream_t s)
{
    static int max_ctas[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = (sizeof(double2) << PR_TILE_BITS) + b.stage_bytes;
    if (smem > PR_SMEM_CAP) return cudaErrorInvalidValue;
    if (dev < 64 && max_ctas[dev] == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PR_SMEM_CAP);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs, PR_THREADS, PR_SMEM_CAP);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        max_ctas[dev] = (per_sm > 0 ? per_sm : 1) * sms;
    }
    if (n < PR_TILE_BITS) return cudaErrorInvalidValue;
    const uint64_t tiles = 1ull << (n - PR_TILE_BITS);
    uint64_t grid = tiles;
    if (dev < 64 && grid > (uint64_t)max_ctas[dev]) grid = (uint64_t)max_ctas[dev];
    k_pairs<<<(unsigned)grid, PR_THREADS, smem, s>>>(static_cast<double2*>(state), b.passes, b.ops, b.layouts,
                                                     reinterpret_cast<const double2*>(b.gates), pass_index, tiles);
    return cudaGetLastError();
}

}  // namespace svb

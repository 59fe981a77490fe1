// Fused tensor-core engine: tcgen05 MMAs on an FP32 state tile in shared memory.
//
// One persistent CTA per SM (8 warps, two per TMEM lane quadrant) walks the tiles of a
// pass; the next tile is loaded into registers while the current one is in the tensor
// core.
// For a tile of 4096 amplitudes (12 local qubits) and a fused block on k target qubits,
// the tile is viewed as X[n][kk]: rows n = the 2^(12-k) values of the other local
// qubits, kk = 2a + re/im for the 2^k target values a.  The block's real-form gate
// G[m'][kk] (2^(k+1) square) is applied as
//        D[n][m'] = sum_kk X[n][kk] G[m'][kk]
// with tcgen05.mma.kind::tf32 (M = 128 rows per MMA, N = 2^(k+1), K = 8 per
// instruction) accumulating in TMEM, in three products X_hi G_hi + X_hi G_lo + X_lo G_hi
// (split TF32: hi = x rounded to TF32, lo = x - hi rounded to TF32), so the result keeps ~FP32
// accuracy.  Both operands sit in shared memory in the canonical K-major, no-swizzle
// layout (8-row x 16-byte core matrices).  Each thread then reads its D row (one row n,
// all 2^k amplitudes) with tcgen05.ld and scatters it, split again into hi/lo, into the
// operand layout of the next block — or, after the last block, into a plain staging
// copy of the tile that is written back to HBM.
//
// Every wait on the MMA-completion mbarrier is bounded; on timeout the kernel records
// an error, releases its tensor memory and returns.
#include <cstdint>

#include "svb_internal.h"

namespace svb {
namespace {

constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// canonical K-major, no-swizzle shared-memory descriptor
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;                 // descriptor version (sm_100)
    return d;                               // base offset 0, LBO mode 0, no swizzle
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc_tf32(uint32_t n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate),
          "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ float tf32_rna(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// 8 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v)
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

template <int K>
struct FusedSmem {
    static constexpr uint32_t x_bytes = 4096u * 2u * 4u;                  // one plane: 32 KiB
    static constexpr uint32_t n_real = 1u << (K + 1);
    static constexpr uint32_t gate_bytes = 2u * n_real * n_real * 4u;     // hi + lo planes
    static constexpr uint32_t max_blocks = (uint32_t)fused_max_blocks(K);
    static constexpr uint32_t x_hi = 0;
    static constexpr uint32_t x_lo = x_hi + x_bytes;
    static constexpr uint32_t gates = x_lo + x_bytes;
    static constexpr uint32_t blocks = gates + max_blocks * gate_bytes;
    static constexpr uint32_t pass = blocks + max_blocks * sizeof(FusedBlock);
    static constexpr uint32_t misc = pass + sizeof(FusedPass);
    static constexpr uint32_t total = misc + 64;
    static constexpr int ctas_per_sm = total <= 113u * 1024u ? 2 : 1;
    static_assert(gates % 16 == 0 && blocks % 16 == 0 && pass % 16 == 0 && misc % 16 == 0, "align");
};

// Writes amplitude (re, im) at word offset w of the state operand (re and im are adjacent
// K values, 8-byte aligned), split into a TF32 hi plane and a TF32 lo plane.  Both
// parts are rounded to nearest explicitly: the MMA reads only the upper 19 bits of each
// FP32 word, and a remainder left in full FP32 would lose its low bits by truncation,
// i.e. always towards zero, which shrinks the norm a little at every block.
__device__ __forceinline__ void put_operand(float* xh, float* xl, uint32_t w, float re, float im)
{
    const float hr = tf32_rna(re), hi = tf32_rna(im);
    *reinterpret_cast<float2*>(xh + w) = make_float2(hr, hi);
    *reinterpret_cast<float2*>(xl + w) = make_float2(tf32_rna(re - hr), tf32_rna(im - hi));
}

template <int K>
__global__ void __launch_bounds__(FT_THREADS, FusedSmem<K>::ctas_per_sm)
k_fused(float2* __restrict__ sv, const FusedPass* __restrict__ passes,
        const FusedBlock* __restrict__ blocks, const float* __restrict__ gates, int pass_index,
        uint64_t tiles, int* __restrict__ err)
{
    constexpr int N = 1 << (K + 1);                 // real gate dimension = MMA N = K extent
    constexpr int ROWS = 1 << (FT_TILE_BITS - K);   // rows of the state operand
    constexpr int MBLK = ROWS / 128;                // M = 128 blocks
    constexpr int KSTEPS = N / 8;                   // tf32 MMA K = 8
    constexpr int HALF = N / 2;                     // TMEM columns read per thread and M block
    constexpr uint32_t GATE_WORDS = 2u * N * N;     // hi + lo planes
    constexpr uint32_t IDESC = umma_idesc_tf32(N);
    constexpr int PAIRS = 4096 / 2 / FT_THREADS;    // float4 (2 amplitudes) per thread
    static_assert(MBLK * N <= (int)kTmemCols, "TMEM columns");

    extern __shared__ __align__(128) unsigned char sm[];
    using L = FusedSmem<K>;
    float* xh = reinterpret_cast<float*>(sm + L::x_hi);
    float* xl = reinterpret_cast<float*>(sm + L::x_lo);
    float* sg = reinterpret_cast<float*>(sm + L::gates);
    FusedBlock* sb = reinterpret_cast<FusedBlock*>(sm + L::blocks);
    FusedPass* sp = reinterpret_cast<FusedPass*>(sm + L::pass);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::misc);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::misc + 16);

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int quad = warp & 3;          // TMEM lane quadrant of this warp
    const int half = warp >> 2;         // which half of the D columns it reads

    // -- stage the pass, its blocks and their gate operands in shared memory
    {
        const FusedPass& gp = passes[pass_index];
        const uint4* src = reinterpret_cast<const uint4*>(&gp);
        uint4* dst = reinterpret_cast<uint4*>(sp);
        for (int w = tid; w < (int)(sizeof(FusedPass) / 16); w += FT_THREADS) dst[w] = src[w];
    }
    __syncthreads();
    const int nb = sp->n_blocks;
    {
        const uint4* src = reinterpret_cast<const uint4*>(blocks + sp->block_begin);
        uint4* dst = reinterpret_cast<uint4*>(sb);
        for (int w = tid; w < nb * (int)(sizeof(FusedBlock) / 16); w += FT_THREADS) dst[w] = src[w];
    }
    __syncthreads();
    for (int b = 0; b < nb; b++) {
        const uint4* src = reinterpret_cast<const uint4*>(gates + sb[b].gate_word);
        uint4* dst = reinterpret_cast<uint4*>(sg + b * GATE_WORDS);
        for (int w = tid; w < (int)(GATE_WORDS / 4); w += FT_THREADS) dst[w] = src[w];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"(kTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t x_hi_a = smem_u32(xh), x_lo_a = smem_u32(xl), g_a = smem_u32(sg);
    const FusedPass& P = *sp;
    uint32_t parity = 0;
    bool ok = true;

    auto tile_base = [&](uint64_t tile) {
        uint64_t base = 0;
        for (int j = 0; j < P.n_nonlocal; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];
        return base;
    };
    // thread t owns the amplitude pairs at local indices 2 (t + 256 j), j < PAIRS; the
    // lowest local qubit is global qubit 0, so each pair is 16 contiguous bytes.  Their
    // global offsets and their places in block 0's operand are fixed for the pass.
    uint64_t gof[PAIRS];
    uint32_t w0[PAIRS][2];
#pragma unroll
    for (int j = 0; j < PAIRS; j++) {
        const uint32_t l = 2u * ((uint32_t)tid + (uint32_t)FT_THREADS * (uint32_t)j);
        gof[j] = P.g_lo[l & 63u] + P.g_hi[l >> 6];
        w0[j][0] = sb[0].off_lo[l & 63u] + sb[0].off_hi[l >> 6];
        w0[j][1] = sb[0].off_lo[(l + 1) & 63u] + sb[0].off_hi[(l + 1) >> 6];
    }
    float4 cur[PAIRS];
    uint64_t base = tile_base(blockIdx.x);
    if (blockIdx.x < tiles) {
#pragma unroll
        for (int j = 0; j < PAIRS; j++) cur[j] = *reinterpret_cast<const float4*>(sv + base + gof[j]);
    }

    for (uint64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        // block 0 operand from the registers
#pragma unroll
        for (int j = 0; j < PAIRS; j++) {
            put_operand(xh, xl, w0[j][0], cur[j].x, cur[j].y);
            put_operand(xh, xl, w0[j][1], cur[j].z, cur[j].w);
        }
        // prefetch the next tile while this one is in the tensor core
        const uint64_t next = tile + gridDim.x;
        const uint64_t nbase = next < tiles ? tile_base(next) : 0;
        if (next < tiles) {
#pragma unroll
            for (int j = 0; j < PAIRS; j++) cur[j] = *reinterpret_cast<const float4*>(sv + nbase + gof[j]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();

        for (int b = 0; b < nb && ok; b++) {
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t gh = g_a + (uint32_t)b * GATE_WORDS * 4u;
                const uint32_t gl = gh + (uint32_t)N * N * 4u;
#pragma unroll
                for (int mb = 0; mb < MBLK; mb++) {
                    const uint32_t d = tmem + (uint32_t)(mb * N);
                    const uint32_t aoff = (uint32_t)mb * 16u * 128u;
#pragma unroll
                    for (int s = 0; s < KSTEPS; s++) {
                        const uint32_t ka = (uint32_t)s * 2u * (ROWS * 16u);
                        const uint32_t kb = (uint32_t)s * 2u * (N * 16u);
                        const uint64_t dah = umma_desc(x_hi_a + aoff + ka, ROWS * 16u, 128u);
                        const uint64_t dal = umma_desc(x_lo_a + aoff + ka, ROWS * 16u, 128u);
                        const uint64_t dbh = umma_desc(gh + kb, N * 16u, 128u);
                        const uint64_t dbl = umma_desc(gl + kb, N * 16u, 128u);
                        mma_tf32(d, dah, dbh, IDESC, s > 0 ? 1u : 0u);
                        mma_tf32(d, dah, dbl, IDESC, 1u);
                        mma_tf32(d, dal, dbh, IDESC, 1u);
                    }
                }
                mma_commit(bar);
            }
            const bool got = mbar_wait(bar, parity);
            parity ^= 1u;
            ok = __syncthreads_and(got ? 1 : 0) != 0;
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // this warp's D rows n = 32 quad + lane + 128 mb, columns of its half
            const FusedBlock& B = sb[b];
            const bool last = (b == nb - 1);
            float dv[MBLK][HALF];
#pragma unroll
            for (int mb = 0; mb < MBLK; mb++) {
                const uint32_t ta = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(mb * N + half * HALF);
                if constexpr (HALF >= 16) {
#pragma unroll
                    for (int c = 0; c < HALF; c += 16) tmem_ld16(ta + (uint32_t)c, &dv[mb][c]);
                } else {
                    tmem_ld8(ta, &dv[mb][0]);
                }
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();   // every row is read before the operand planes are overwritten
            float2* stage = reinterpret_cast<float2*>(xh);     // plain tile copy after the last block
#pragma unroll
            for (int mb = 0; mb < MBLK; mb++) {
                const uint32_t n = (uint32_t)(quad * 32 + (tid & 31) + 128 * mb);
                const uint32_t wn = B.nxt_nlo[n & 31u] + B.nxt_nhi[n >> 5];
#pragma unroll
                for (int a2 = 0; a2 < HALF / 2; a2++) {
                    const int a = half * (HALF / 2) + a2;
                    const uint32_t w = wn + B.nxt_a[a];
                    const float re = dv[mb][2 * a2], im = dv[mb][2 * a2 + 1];
                    if (last) stage[w] = make_float2(re, im);
                    else put_operand(xh, xl, w, re, im);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        }
        if (!ok) break;
        // store the tile
        const float4* stage4 = reinterpret_cast<const float4*>(xh);
#pragma unroll
        for (int j = 0; j < PAIRS; j++)
            *reinterpret_cast<float4*>(sv + base + gof[j]) = stage4[tid + FT_THREADS * j];
        base = nbase;
        __syncthreads();
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        mbar_wait(bar, parity ^ 1u);     // bounded: let an MMA still in flight finish
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(kTmemCols) : "memory");
}

template <int K>
cudaError_t launch_k(void* state, int n, int pass_index, const DevFusedBuffers& b, cudaStream_t s)
{
    static int ctas[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return cudaErrorInvalidDevice;
    if (ctas[dev] == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_fused<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)FusedSmem<K>::total);
        if (e != cudaSuccess) return e;
        int sms = 0, per_sm = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<K>, FT_THREADS,
                                                          FusedSmem<K>::total);
        if (e != cudaSuccess) return e;
        ctas[dev] = sms * (per_sm > 0 ? per_sm : 1);
    }
    const uint64_t tiles = 1ull << (n - FT_TILE_BITS);
    const uint64_t grid = tiles < (uint64_t)ctas[dev] ? tiles : (uint64_t)ctas[dev];
    k_fused<K><<<(unsigned)grid, FT_THREADS, FusedSmem<K>::total, s>>>(
        static_cast<float2*>(state), b.passes, b.blocks, b.gates, pass_index, tiles, b.err);
    return cudaGetLastError();
}

// FP64 sum of |a|^2 per block (grid-stride, fixed order within a block)
__global__ void __launch_bounds__(256) k_norm_partial(const float4* __restrict__ sv, uint64_t pairs,
                                                      double* __restrict__ partial)
{
    __shared__ double red[8];
    double acc = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pairs;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 v = sv[i];
        acc += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; w++) s += red[w];
        partial[blockIdx.x] = s;
    }
}

// a <- a / sqrt(sum |a|^2); every block forms the same total from the partials in the
// same order, so the scale is identical everywhere
__global__ void __launch_bounds__(256) k_renorm(float4* __restrict__ sv, uint64_t pairs,
                                                const double* __restrict__ partial, int np)
{
    __shared__ float scale;
    if (threadIdx.x < 32) {
        double s = 0.0;
        for (int i = threadIdx.x; i < np; i += 32) s += partial[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) scale = s > 0.0 ? (float)(1.0 / sqrt(s)) : 1.0f;
    }
    __syncthreads();
    const float f = scale;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pairs;
         i += (uint64_t)gridDim.x * blockDim.x) {
        float4 v = sv[i];
        v.x *= f; v.y *= f; v.z *= f; v.w *= f;
        sv[i] = v;
    }
}

}  // namespace

// The tensor cores accumulate the FP32 sums of an MMA with truncation (round towards
// zero), so every fused block takes a fraction of an ulp off each amplitude's magnitude
// and the norm of an FP32 fused run decays slowly (about 1e-7 per gate).  The decay is
// nearly uniform over the amplitudes, so one FP64 renormalisation after the run removes
// it: two reads and one write of the state.
cudaError_t launch_fused_renorm(void* state, int n, const DevFusedBuffers& b, cudaStream_t s)
{
    if (n < FT_TILE_BITS || !b.norm_partial) return cudaErrorInvalidValue;
    const uint64_t pairs = 1ull << (n - 1);
    float4* sv = static_cast<float4*>(state);
    k_norm_partial<<<REDUCE_BLOCKS, 256, 0, s>>>(sv, pairs, b.norm_partial);
    k_renorm<<<REDUCE_BLOCKS * 2, 256, 0, s>>>(sv, pairs, b.norm_partial, REDUCE_BLOCKS);
    return cudaGetLastError();
}

cudaError_t launch_fused_pass(void* state, int n, int k, int pass_index, int n_blocks,
                              int gate_words_per_block, const DevFusedBuffers& b, cudaStream_t s)
{
    (void)n_blocks;
    (void)gate_words_per_block;
    if (n < FT_TILE_BITS) return cudaErrorInvalidValue;
    switch (k) {
    case 3: return launch_k<3>(state, n, pass_index, b, s);
    case 4: return launch_k<4>(state, n, pass_index, b, s);
    case 5: return launch_k<5>(state, n, pass_index, b, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace svb

// Fused tensor-core engine at fusion width 6: one 6-qubit block per pass (fuse.cpp,
// plan_fused6), FP32 states, split TF32 on tcgen05.
//
// The block is applied in the transposed form
//        D^T[m'][n] = sum_kk G[m'][kk] X[n][kk]
// with G the block's real form (128 x 128: m' = 2a' + re/im of the output, kk = 2a +
// re/im of the input) and X the tile viewed as 64 rows n (the row qubits) of 128 reals
// (the 6 target qubits).  M = 128 is the full width of one tcgen05.mma, so the 6-qubit
// block runs at the tensor core's full rate with N = 64 rows per instruction:
//  * A = G_hi and G_lo (rounded to nearest TF32 on the host from FP64) sit in tensor
//    memory for the whole launch (columns 0..255), written once by the data warps;
//  * B = the tile in shared memory in the canonical K-major layout (no swizzle).  A tile
//    arrives by 8-byte cp.async straight into its place in the hi plane (the MMA reads an
//    FP32 value truncated to TF32, so the loaded values are X_hi as they are), and each
//    thread then writes the exact remainder, rounded to nearest TF32, into the lo plane;
//  * D^T += G_hi X_hi, += G_lo X_hi, += G_hi X_lo: 3 x 16 MMAs (K = 8 each) accumulate in
//    one FP32 accumulator of 64 columns.
// Three tiles are in flight (three slots of hi + lo planes, 192 KiB; three accumulators,
// columns 256..447): while the tensor core runs one tile the data warps prepare the next
// and write out the previous one.  The output goes from tensor memory straight to global
// memory: a thread holds one component of one output amplitude for 16 rows; neighbouring
// lanes (re, im) swap halves so that each writes whole amplitudes, two adjacent ones per
// 16-byte store when row bit 0 is qubit 0.
//
// No thread reads shared memory written by another thread (each prepares the lo terms of
// the amplitudes it copied itself), so the data warps need no barrier among themselves:
// the mbarriers of the loads, of the prepared operands and of the MMAs order everything.
// Every wait is bounded (tc_common.cuh); a wait that gives up raises an abort flag that
// ends the other waits, and the kernel then records an error, waits (bounded) for the
// copies and MMAs it counted as in flight, frees its tensor memory and returns.
#include <cstdint>

#include "svb_internal.h"
#include "tc_common.cuh"

namespace svb {
namespace {

constexpr int F6_DATA_WARPS = 16;
constexpr int F6_THREADS = 32 * (F6_DATA_WARPS + 1);
constexpr int F6_EPI = 32 * F6_DATA_WARPS;                    // 512 data threads
constexpr int F6_PER_THREAD = (1 << F6_TILE_BITS) / F6_EPI;   // 8 amplitudes
constexpr uint32_t F6_PLANE_BYTES = (1u << F6_TILE_BITS) * 8u;  // 32 KiB: 64 rows x 128 TF32
constexpr uint32_t F6_SLOT_BYTES = 2u * F6_PLANE_BYTES;         // hi + lo
constexpr uint32_t F6_TMEM_COLS = 512;
constexpr uint32_t F6_G_HI_COL = 0, F6_G_LO_COL = F6_N, F6_D_COL = 2 * F6_N;
constexpr uint32_t F6_LBO = F6_ROWS * 16u;    // between the two 16-byte K columns of a K step
constexpr uint32_t F6_SBO = 128u;             // between groups of 8 rows
constexpr uint32_t F6_KSTEPS = F6_N / 8;      // tf32 MMA: K = 8
constexpr uint32_t F6_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(F6_ROWS >> 3) << 17) |
                              ((128u >> 4) << 24);
static_assert(F6_D_COL + F6_SLOTS * F6_ROWS <= F6_TMEM_COLS, "tensor memory columns");

struct F6Smem {
    static constexpr uint32_t planes = 0;                                  // slot s: hi, lo
    static constexpr uint32_t tbase = planes + F6_SLOTS * F6_SLOT_BYTES;   // tile index -> base, 3 x 256
    static constexpr uint32_t misc = tbase + 3u * 256u * 8u;               // mbarriers, flags, counters
    static constexpr uint32_t total = misc + 256;
    static_assert(total <= 227u * 1024u, "shared memory of one CTA");
    // a second CTA on the SM would wait for the 512 tensor-memory columns this one holds
    static_assert(total > 114u * 1024u, "one CTA per SM");
};

__global__ void __launch_bounds__(F6_THREADS, 1)
k_fused6(float2* __restrict__ sv, const Fused6Pass* __restrict__ passes, const float* __restrict__ gates,
         int pass_index, uint64_t tiles, int* __restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* tb = reinterpret_cast<uint64_t*>(sm + F6Smem::tbase);
    uint64_t* bar_load = reinterpret_cast<uint64_t*>(sm + F6Smem::misc);   // per slot: tile landed
    uint64_t* bar_ready = bar_load + F6_SLOTS;                              // per slot: lo plane written
    uint64_t* bar_mma = bar_ready + F6_SLOTS;                               // per slot: MMAs done
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + F6Smem::misc + 72);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + F6Smem::misc + 76);
    // [0,3) MMA commits, [3,6) MMA completions consumed, [6,9) loads issued, [9,12) consumed
    uint32_t* counts = reinterpret_cast<uint32_t*>(sm + F6Smem::misc + 80);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool mma_warp = warp == F6_DATA_WARPS;
    const Fused6Pass& P = passes[pass_index];
    const int nn = P.n_nonlocal;
    const bool plan_ok = nn >= 0 && nn <= 24;
    const uint64_t my_tiles = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    // tile index bits 8t..8t+7 -> their share of the tile's global base
    for (int i = tid; plan_ok && i < 3 * 256; i += F6_THREADS) {
        const int t = i >> 8;
        uint64_t base = 0;
        for (int b = 0; b < 8; b++) {
            const int q = 8 * t + b;
            if (q < nn && ((i >> b) & 1)) base |= 1ull << P.nonlocal_q[q];
        }
        tb[i] = base;
    }
    if (tid == 0) {
        for (int s = 0; s < F6_SLOTS; s++) {
            mbar_init(bar_load + s, F6_EPI);
            mbar_init(bar_ready + s, F6_DATA_WARPS);
            mbar_init(bar_mma + s, 1);
        }
        *abort_flag = 0;
        for (int i = 0; i < 12; i++) counts[i] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"(F6_TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int quad = warp & 3, part = warp >> 2;                  // data warps: TMEM lane quadrant
    const uint32_t lane_base = (uint32_t)(quad * 32) << 16;

    // the block's G_hi and G_lo into tensor memory: lane m' = 32 quad + lane, columns
    // 32 part .. 32 part + 31 of each plane
    if (!mma_warp && plan_ok) {
        const uint32_t m = (uint32_t)(quad * 32 + lane);
        const float4* gh = reinterpret_cast<const float4*>(gates + P.gate_word + (size_t)m * F6_N + part * 32);
        const float4* gl = gh + (F6_N * F6_N) / 4;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float a[16], b[16];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float4 x = gh[4 * h + i], y = gl[4 * h + i];
                a[4 * i] = x.x; a[4 * i + 1] = x.y; a[4 * i + 2] = x.z; a[4 * i + 3] = x.w;
                b[4 * i] = y.x; b[4 * i + 1] = y.y; b[4 * i + 2] = y.z; b[4 * i + 3] = y.w;
            }
            tmem_st16(tmem + lane_base + F6_G_HI_COL + (uint32_t)(part * 32 + 16 * h), a);
            tmem_st16(tmem + lane_base + F6_G_LO_COL + (uint32_t)(part * 32 + 16 * h), b);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool run = plan_ok && my_tiles > 0;

    auto tile_base = [&](uint64_t j) {
        const uint64_t t = blockIdx.x + j * gridDim.x;
        return tb[t & 255u] | tb[256 + ((t >> 8) & 255u)] | tb[512 + ((t >> 16) & 255u)];
    };

    if (mma_warp) {
        // ---- one lane issues each tile's 48 MMAs once its lo plane is written
        if (lane == 0 && run) {
            const uint32_t planes = smem_u32(sm + F6Smem::planes);
            for (uint64_t j = 0; j < my_tiles; j++) {
                const int s = (int)(j % F6_SLOTS);
                if (!mbar_wait_abort(bar_ready + s, (uint32_t)((j / F6_SLOTS) & 1u), abort_flag)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + F6_D_COL + (uint32_t)(F6_ROWS * s);
                const uint32_t hi = planes + (uint32_t)s * F6_SLOT_BYTES, lo = hi + F6_PLANE_BYTES;
#pragma unroll
                for (int p3 = 0; p3 < 3; p3++) {
                    // G_hi X_hi, G_lo X_hi, G_hi X_lo
                    const uint32_t a = tmem + (p3 == 1 ? F6_G_LO_COL : F6_G_HI_COL);
                    const uint32_t b = p3 == 2 ? lo : hi;
#pragma unroll
                    for (uint32_t k8 = 0; k8 < F6_KSTEPS; k8++)
                        mma_tf32_ts(d, a + 8u * k8, umma_desc(b + k8 * 2u * F6_LBO, F6_LBO, F6_SBO), F6_IDESC,
                                    (p3 > 0 || k8 > 0) ? 1u : 0u);
                }
                mma_commit(bar_mma + s);
                counts[s]++;
            }
        }
    } else if (run) {
        // ---- the data warps: amplitudes x = tid + 512 i of each tile
        float2* planes = reinterpret_cast<float2*>(sm + F6Smem::planes);
        uint64_t goff[F6_PER_THREAD];
        uint32_t soff[F6_PER_THREAD];
        {
            const uint64_t g = P.g_lo[tid & 63];
            const uint32_t w = P.s_lo[tid & 63];
#pragma unroll
            for (int i = 0; i < F6_PER_THREAD; i++) {
                goff[i] = g | P.g_hi[(tid >> 6) + 8 * i];
                soff[i] = w + P.s_hi[(tid >> 6) + 8 * i];
            }
        }
        // output: this lane holds component (lane & 1) of amplitude a' = (32 quad + lane) / 2
        // for rows 16 part + j; after the swap with its neighbour an even lane writes rows
        // 16 part + j and an odd lane rows 16 part + 8 + j (j < 8), as whole amplitudes
        const bool odd = lane & 1;
        const uint64_t otgt = P.o_tgt[(quad * 32 + lane) >> 1];
        uint64_t orow[8];
#pragma unroll
        for (int j = 0; j < 8; j++) orow[j] = P.o_row[16 * part + (odd ? 8 : 0) + j] | otgt;
        const bool paired = P.rows_paired != 0;

        auto issue_load = [&](uint64_t j) {
            const int s = (int)(j % F6_SLOTS);
            const float2* src = sv + tile_base(j);
            float2* dst = planes + (size_t)s * (F6_SLOT_BYTES / 8);
#pragma unroll
            for (int i = 0; i < F6_PER_THREAD; i++) cp_async8(dst + soff[i], src + goff[i]);
            cp_async_arrive(bar_load + s);
            if (tid == 0) counts[6 + s]++;
        };
        // the lo plane of tile j from its hi plane, then this warp's arrival
        auto prepare = [&](uint64_t j) -> bool {
            const int s = (int)(j % F6_SLOTS);
            const bool got = __all_sync(0xffffffffu,
                                        mbar_wait_abort(bar_load + s, (uint32_t)((j / F6_SLOTS) & 1u), abort_flag));
            if (!got) return false;
            if (tid == 0) counts[9 + s]++;
            float2* hi = planes + (size_t)s * (F6_SLOT_BYTES / 8);
            float2* lo = hi + F6_PLANE_BYTES / 8;
#pragma unroll
            for (int i = 0; i < F6_PER_THREAD; i++) {
                const float2 x = hi[soff[i]];
                float h, l0, l1;
                split_tf32(x.x, h, l0);
                split_tf32(x.y, h, l1);
                lo[soff[i]] = make_float2(l0, l1);
            }
            // this thread's copies (landed) and stores, before the tensor core reads them
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_ready + s);
            return true;
        };
        // tile j out of its accumulator into the state
        auto output = [&](uint64_t j) -> bool {
            const int s = (int)(j % F6_SLOTS);
            const bool got = __all_sync(0xffffffffu,
                                        mbar_wait_abort(bar_mma + s, (uint32_t)((j / F6_SLOTS) & 1u), abort_flag));
            if (!got) return false;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float v[16];
            tmem_ld16(tmem + lane_base + F6_D_COL + (uint32_t)(F6_ROWS * s + 16 * part), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            if (tid == 0) counts[3 + s]++;
            float w[8];
#pragma unroll
            for (int i = 0; i < 8; i++) w[i] = __shfl_xor_sync(0xffffffffu, odd ? v[i] : v[8 + i], 1);
            float2* dst = sv + tile_base(j);
            if (paired) {
#pragma unroll
                for (int i = 0; i < 8; i += 2) {
                    const float4 q = odd ? make_float4(w[i], v[8 + i], w[i + 1], v[9 + i])
                                         : make_float4(v[i], w[i], v[i + 1], w[i + 1]);
                    *reinterpret_cast<float4*>(dst + orow[i]) = q;
                }
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) dst[orow[i]] = odd ? make_float2(w[i], v[8 + i]) : make_float2(v[i], w[i]);
            }
            return true;
        };

        bool ok = true;
        for (uint64_t j = 0; j < (uint64_t)F6_SLOTS && j < my_tiles; j++) issue_load(j);
        for (uint64_t j = 0; ok && j < my_tiles; j++) {
            ok = prepare(j);
            if (ok && j >= 1) {
                ok = output(j - 1);
                // slot (j - 1) % 3: its MMAs are done (this thread waited), so its planes
                // take tile j + 2
                if (ok && j + 2 < my_tiles) issue_load(j + 2);
            }
        }
        if (ok) ok = output(my_tiles - 1);
        if (!ok) *abort_flag = 1;
    }

    __syncthreads();
    if (!plan_ok && tid == 0) atomicExch(err, 1);
    if (*abort_flag && tid == 0) {
        atomicExch(err, 1);
        // let what is still in flight land before the memory goes away (bounded waits)
        for (int s = 0; s < F6_SLOTS; s++) {
            for (uint32_t c = counts[3 + s]; c < counts[s]; c++) mbar_wait(bar_mma + s, c & 1u);
            for (uint32_t c = counts[9 + s]; c < counts[6 + s]; c++) mbar_wait(bar_load + s, c & 1u);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(F6_TMEM_COLS) : "memory");
}

}  // namespace

cudaError_t launch_fused6_pass(void* state, int n, int pass_index, const DevFusedBuffers& b, cudaStream_t s)
{
    static int ctas[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return cudaErrorInvalidDevice;
    if (n < F6_TILE_BITS || !b.passes6 || !b.gates || !b.err) return cudaErrorInvalidValue;
    if (ctas[dev] == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_fused6, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)F6Smem::total);
        if (e != cudaSuccess) return e;
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        ctas[dev] = sms;                 // one CTA per SM (all of its tensor memory)
    }
    const uint64_t tiles = 1ull << (n - F6_TILE_BITS);
    const uint64_t grid = tiles < (uint64_t)ctas[dev] ? tiles : (uint64_t)ctas[dev];
    k_fused6<<<(unsigned)grid, F6_THREADS, F6Smem::total, s>>>(static_cast<float2*>(state), b.passes6, b.gates,
                                                                pass_index, tiles, b.err);
    return cudaGetLastError();
}

}  // namespace svb

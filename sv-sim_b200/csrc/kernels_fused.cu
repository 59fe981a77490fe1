// Fused tensor-core engine: tcgen05 MMAs on FP32 state tiles held in tensor memory.
//
// A pass applies its fused blocks to every tile of 4096 amplitudes (12 local qubits).
// For a block on k target qubits the tile is viewed as X[n][kk]: rows n = the 2^(12-k)
// values of the other local qubits, kk = 2a + re/im for the 2^k target values a.  The
// block's real-form gate G[m'][kk] (N = 2^(k+1) square) is applied as
//        D[n][m'] = sum_kk X[n][kk] G[m'][kk]
// with tcgen05.mma.kind::tf32 (M = 128 rows per MMA, K = 8 per instruction) in three
// products X_hi G_hi + X_hi G_lo + X_lo G_hi (split TF32: hi = x as the MMA reads it,
// i.e. truncated to TF32, lo = the remainder rounded to nearest TF32; the gate's halves
// are split on the host from FP64), so the result keeps ~FP32 accuracy.  The gate operand
// holds G_hi in rows 0..N-1 and G_lo in rows N..2N-1, so per K step one MMA of width 2N
// forms [X_hi G_hi | X_hi G_lo] and one of width N adds X_lo G_hi to the first half.
//
// One persistent CTA per SM: 16 warps (four per TMEM lane quadrant) move the data and one
// warp issues the MMAs.
//  * The state operand (hi and lo planes) lives in tensor memory as the MMA's A operand;
//    only the gate operand (B, canonical K-major layout, no swizzle) is read from shared
//    memory.  With both operands in shared memory the MMAs of a narrow block read more
//    bytes per cycle than shared memory delivers.
//  * After a block each thread reads its D rows (tcgen05.ld), adds the two halves, writes
//    them into a transpose buffer in the next block's row order (fused_slot), reads back its rows of the next block, splits
//    them into hi/lo and stores them into tensor memory (tcgen05.st).  Each warp then
//    arrives on the slot's "operands ready" mbarrier, on which the MMA warp waits.
//  * Two tiles are in flight, in two TMEM slots of 256 columns (A hi, A lo: 64 each; D:
//    128): while the threads turn one tile's D into the next operand, the tensor core
//    runs the other tile's MMAs.
//  * Tiles arrive by 16-byte cp.async (the 3 lowest qubits are always local: 64-byte
//    runs) into prefetch buffers some tiles ahead, each thread's copies completing on
//    the buffer's mbarrier, and leave by 16-byte stores from the transpose buffer used
//    as an output stage.  The layouts of both (per-run XOR swizzles the planner picks)
//    and of the transpose buffer keep every 8- and 16-byte shared-memory access of the
//    kernel free of bank conflicts wherever the pass's bit layout allows.
// Every mbarrier wait is bounded and gives up early when another warp has given up; the
// kernel then records an error, waits (bounded) for its MMAs and copies in flight,
// releases its tensor memory and returns.
#include <cstdint>

#include "svb_internal.h"
#include "tc_common.cuh"

namespace svb {
namespace {

constexpr uint32_t kTmemCols = 512;      // two slots
constexpr uint32_t kSlotCols = 256;

// barrier of the data warps (named barrier 1) that also ANDs a predicate over them
__device__ __forceinline__ bool epi_sync_and(bool p)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred a, b;\n\t"
        "setp.ne.u32 a, %1, 0;\n\t"
        "bar.red.and.pred b, 1, %2, a;\n\t"
        "selp.u32 %0, 1, 0, b;\n\t}\n"
        : "=r"(r) : "r"(p ? 1u : 0u), "n"(FT_EPI_WARPS * 32) : "memory");
    return r != 0;
}

// CA consecutive 16-bit table entries (CA = 2, 4 or 8; 4-byte aligned) in one load
template <int CA>
__device__ __forceinline__ void load_u16(const uint16_t* t, uint32_t* out)
{
    if constexpr (CA == 8) {
        const uint4 q = *reinterpret_cast<const uint4*>(t);
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int i = 0; i < 4; i++) { out[2 * i] = w[i] & 0xFFFFu; out[2 * i + 1] = w[i] >> 16; }
    } else if constexpr (CA == 4) {
        const uint2 q = *reinterpret_cast<const uint2*>(t);
        out[0] = q.x & 0xFFFFu; out[1] = q.x >> 16; out[2] = q.y & 0xFFFFu; out[3] = q.y >> 16;
    } else {
        const uint32_t q = *reinterpret_cast<const uint32_t*>(t);
        out[0] = q & 0xFFFFu; out[1] = q >> 16;
    }
}

template <int K>
struct FusedSmem {
    static constexpr uint32_t tile_bytes = 4096u * 8u;                    // 32 KiB
    static constexpr uint32_t n_real = 1u << (K + 1);
    static constexpr uint32_t gate_bytes = 2u * n_real * n_real * 4u;     // [G_hi; G_lo]
    static constexpr uint32_t max_blocks = (uint32_t)fused_max_blocks(K);
    static constexpr uint32_t n_raw = (uint32_t)fused_raw_buffers(K);
    static constexpr uint32_t trans = 0;                                  // two transpose buffers
    static constexpr uint32_t raw = trans + 2 * tile_bytes;               // prefetch buffers
    static constexpr uint32_t gates = raw + n_raw * tile_bytes;
    static constexpr uint32_t blocks = gates + max_blocks * gate_bytes;
    static constexpr uint32_t pass = blocks + max_blocks * sizeof(FusedBlock);
    static constexpr uint32_t tbase = pass + sizeof(FusedPass);          // tile index -> base, 3 x 256
    static constexpr uint32_t misc = tbase + 3u * 256u * 8u;              // mbarriers, flags, counters
    static constexpr uint32_t total = misc + 128;
    static_assert(total <= 227u * 1024u, "shared memory of one CTA");
    // a second CTA on the SM would wait for the 512 TMEM columns this one holds
    static_assert(total > 114u * 1024u, "one CTA per SM");
    static_assert(gates % 128 == 0 && blocks % 16 == 0 && pass % 16 == 0 && tbase % 16 == 0 &&
                  misc % 16 == 0, "align");
};

template <int K>
__global__ void __launch_bounds__(FT_THREADS, 1)
k_fused(float2* __restrict__ sv, const FusedPass* __restrict__ passes,
        const FusedBlock* __restrict__ blocks, const float* __restrict__ gates, int pass_index,
        uint64_t tiles, int* __restrict__ err)
{
    constexpr int N = 1 << (K + 1);                 // real gate dimension = K extent
    constexpr int DN = 2 * N;                       // D columns per M block: [hi | lo products]
    constexpr int ROWS = 1 << (FT_TILE_BITS - K);   // rows of the state operand
    constexpr int MBLK = ROWS / 128;                // M = 128 blocks
    constexpr int KSTEPS = N / 8;                   // tf32 MMA K = 8
    constexpr int PARTS = FT_EPI_WARPS / 4;         // data warps per TMEM lane quadrant
    constexpr int CW = N / PARTS;                   // columns per thread and M block
    constexpr int CA = CW / 2;                      // amplitudes per thread and M block
    constexpr int CHUNKS = 2048 / (FT_EPI_WARPS * 32);   // 16-byte chunks of a tile per thread
    constexpr int CPR = (1 << K) / 2;               // 16-byte chunks per transpose row
    constexpr int EPI = FT_EPI_WARPS * 32;          // data threads
    constexpr uint32_t GATE_WORDS = 2u * N * N;
    constexpr uint32_t IDESC_W = umma_idesc_tf32(DN), IDESC_N = umma_idesc_tf32(N);
    constexpr uint32_t PLANE = (uint32_t)(MBLK * N);   // TMEM columns of one operand plane
    using L = FusedSmem<K>;
    constexpr uint32_t NR = L::n_raw;
    static_assert(2 * PLANE + MBLK * DN <= kSlotCols && 2 * kSlotCols <= kTmemCols, "TMEM slots");
    static_assert(CA % 2 == 0 && MBLK * CW * FT_EPI_WARPS == 256 && CHUNKS * EPI == 2048, "thread share of a tile");

    extern __shared__ __align__(128) unsigned char sm[];
    float2* trans = reinterpret_cast<float2*>(sm + L::trans);
    float2* raw = reinterpret_cast<float2*>(sm + L::raw);
    float* sg = reinterpret_cast<float*>(sm + L::gates);
    FusedBlock* sb = reinterpret_cast<FusedBlock*>(sm + L::blocks);
    FusedPass* sp = reinterpret_cast<FusedPass*>(sm + L::pass);
    uint64_t* tb = reinterpret_cast<uint64_t*>(sm + L::tbase);
    uint64_t* bar_mma = reinterpret_cast<uint64_t*>(sm + L::misc);   // per slot: MMAs done
    uint64_t* bar_ready = bar_mma + 2;                               // per slot: operands stored
    uint64_t* bar_load = bar_ready + 2;                              // per prefetch buffer
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::misc + 64);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::misc + 68);
    uint32_t* counts = reinterpret_cast<uint32_t*>(sm + L::misc + 72);  // [0,2) MMAs committed,
    // [2,4) MMAs consumed, [4,4+NR) loads issued, [6,6+NR) loads consumed

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool mma_warp = warp == FT_EPI_WARPS;
    const int quad = warp & 3;          // TMEM lane quadrant of a data warp
    const int part = warp >> 2;         // which part of the columns it handles
    const uint64_t my_tiles = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    // -- stage the pass, its blocks and their gate operands in shared memory
    {
        const uint4* src = reinterpret_cast<const uint4*>(passes + pass_index);
        uint4* dst = reinterpret_cast<uint4*>(sp);
        for (int w = tid; w < (int)(sizeof(FusedPass) / 16); w += FT_THREADS) dst[w] = src[w];
    }
    __syncthreads();
    const int nb = sp->n_blocks;
    const bool plan_ok = nb >= 1 && nb <= (int)L::max_blocks && sp->n_nonlocal <= FT_MAX_NONLOCAL;
    if (plan_ok) {
        const uint4* src = reinterpret_cast<const uint4*>(blocks + sp->block_begin);
        uint4* dst = reinterpret_cast<uint4*>(sb);
        for (int w = tid; w < nb * (int)(sizeof(FusedBlock) / 16); w += FT_THREADS) dst[w] = src[w];
        // tile index bits 8t..8t+7 -> their share of the tile's global base
        for (int i = tid; i < 3 * 256; i += FT_THREADS) {
            const int t = i >> 8;
            uint64_t base = 0;
            for (int b = 0; b < 8; b++) {
                const int q = 8 * t + b;
                if (q < sp->n_nonlocal && ((i >> b) & 1)) base |= 1ull << sp->nonlocal_q[q];
            }
            tb[i] = base;
        }
    }
    __syncthreads();
    for (int b = 0; plan_ok && b < nb; b++) {
        const uint4* src = reinterpret_cast<const uint4*>(gates + sb[b].gate_word);
        uint4* dst = reinterpret_cast<uint4*>(sg + b * GATE_WORDS);
        for (int w = tid; w < (int)(GATE_WORDS / 4); w += FT_THREADS) dst[w] = src[w];
    }
    if (tid == 0) {
        mbar_init(bar_mma, 1);
        mbar_init(bar_mma + 1, 1);
        mbar_init(bar_ready, FT_EPI_WARPS);
        mbar_init(bar_ready + 1, FT_EPI_WARPS);
        for (uint32_t i = 0; i < NR; i++) mbar_init(bar_load + i, EPI);
        *abort_flag = 0;
        for (int i = 0; i < 8; i++) counts[i] = 0;
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
    const FusedPass& P = *sp;
    const bool run = plan_ok && my_tiles > 0;

    // global amplitude offset of this CTA's j-th tile
    auto tile_base = [&](uint64_t j) {
        const uint64_t t = blockIdx.x + j * gridDim.x;
        return tb[t & 255u] | tb[256 + ((t >> 8) & 255u)] | tb[512 + ((t >> 16) & 255u)];
    };

    if (mma_warp) {
        // ---- the MMA warp: one lane issues each slot's blocks once its operands are stored
        if (lane == 0 && run) {
            const uint32_t g_a = smem_u32(sg);
            auto issue = [&](int s, int b) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t base = tmem + (uint32_t)s * kSlotCols;
                const uint32_t g = g_a + (uint32_t)b * GATE_WORDS * 4u;
#pragma unroll
                for (int mb = 0; mb < MBLK; mb++) {
                    const uint32_t d = base + 2u * PLANE + (uint32_t)(mb * DN);
                    const uint32_t ah = base + (uint32_t)(mb * N), al = ah + PLANE;
#pragma unroll
                    for (int k8 = 0; k8 < KSTEPS; k8++) {
                        // two 16-byte K chunks of the 2N-row operand per K step
                        const uint64_t dg = umma_desc(g + (uint32_t)k8 * 2u * (DN * 16u), DN * 16u, 128u);
                        mma_tf32_ts(d, ah + 8u * k8, dg, IDESC_W, k8 > 0 ? 1u : 0u);
                        mma_tf32_ts(d, al + 8u * k8, dg, IDESC_N, 1u);
                    }
                }
                mma_commit(bar_mma + s);
                counts[s]++;
            };
            uint32_t rpar0 = 0, rpar1 = 0;
            int blk0 = 0, blk1 = 0;
            bool act0 = true, act1 = my_tiles > 1;
            uint64_t next = act1 ? 2 : 1;
            bool live = mbar_wait_abort(bar_ready, 0, abort_flag);
            if (live) { rpar0 = 1; issue(0, 0); }
            if (live && act1) {
                live = mbar_wait_abort(bar_ready + 1, 0, abort_flag);
                if (live) { rpar1 = 1; issue(1, 0); }
            }
            // the data warps' order: slots alternate; a slot's next block, or block 0 of
            // its next tile
            auto step = [&](int s, bool& act, int& blk, uint32_t& rpar) {
                if (!act || !live) return;
                if (blk + 1 < nb) {
                    blk++;
                } else if (next < my_tiles) {
                    next++;
                    blk = 0;
                } else {
                    act = false;
                    return;
                }
                live = mbar_wait_abort(bar_ready + s, rpar, abort_flag);
                if (!live) return;
                rpar ^= 1u;
                issue(s, blk);
            };
            while (live && (act0 || act1)) {
                step(0, act0, blk0, rpar0);
                step(1, act1, blk1, rpar1);
            }
        }
    } else if (run) {
        // ---- the data warps
        const uint32_t lane_base = (uint32_t)(quad * 32) << 16;
        // the 16-byte chunks of a thread in a tile: chunk c = tid + EPI i is piece tid & 7 of
        // run (tid >> 3) + (EPI / 8) i (local index 16 run + 2 piece; local position 0 is
        // qubit 0, so a piece is two adjacent amplitudes)
        // Fixed for the pass: their global offsets within a tile, their slots in a raw
        // tile and where they sit in the output stage (with the swap of its two halves).
        uint64_t goff[CHUNKS];
        uint32_t rslot[CHUNKS], oslot[CHUNKS];
        {
            const uint64_t g_part = P.g_lo[(((tid >> 3) & 3) << 4) | ((tid & 7) << 1)];
#pragma unroll
            for (int i = 0; i < CHUNKS; i++) {
                const uint32_t c = (uint32_t)(tid + EPI * i);
                goff[i] = g_part + P.g_hi[(tid >> 5) + (EPI / 32) * i];
                rslot[i] = c ^ P.raw_xor[c >> 3];
                const uint32_t ox = P.out_xor[c >> 3];
                oslot[i] = ((c ^ (ox >> 1)) << 1) | (ox & 1u);
            }
        }

        // tile j into prefetch buffer j % NR (CHUNKS cp.async per thread, arriving on its mbarrier)
        auto issue_load = [&](uint64_t j) {
            const uint32_t rb = (uint32_t)(j % NR);
            const float2* src = sv + tile_base(j);
            float2* dst = raw + rb * 4096u;
#pragma unroll
            for (int i = 0; i < CHUNKS; i++) cp_async16(dst + 2 * rslot[i], src + goff[i]);
            cp_async_arrive(bar_load + rb);
            if (tid == 0) counts[4 + rb]++;
        };
        // rows n = 128 mb + 32 quad + lane, columns part * CW + [0, CW): hi/lo into
        // the A planes of slot s, then this warp's arrival on the slot's ready barrier
        auto put_rows = [&](int s, float (&v)[MBLK][CW]) {
            const uint32_t base = tmem + (uint32_t)s * kSlotCols + lane_base + (uint32_t)(part * CW);
#pragma unroll
            for (int mb = 0; mb < MBLK; mb++) {
                float h[CW], l[CW];
#pragma unroll
                for (int i = 0; i < CW; i++) split_tf32(v[mb][i], h[i], l[i]);
                tmem_st_cols<CW>(base + (uint32_t)(mb * N), h);
                tmem_st_cols<CW>(base + PLANE + (uint32_t)(mb * N), l);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_ready + s);
        };

        bool ok = true;
        uint32_t mpar0 = 0, mpar1 = 0, tsel = 0;
        int blk0 = 0, blk1 = 0;
        uint64_t tj0 = 0, tj1 = 0, next_j = 0;
        bool act0 = false, act1 = false;

        // a new tile in slot s: its block-0 rows gathered from the prefetch buffer
        auto start = [&](int s, uint64_t j) -> bool {
            const uint32_t rb = (uint32_t)(j % NR);
            const bool got = mbar_wait_abort(bar_load + rb, (uint32_t)((j / NR) & 1u), abort_flag);
            const float2* R = raw + rb * 4096u;
            const FusedBlock& B0 = sb[0];
            uint32_t asc[CA];
            load_u16<CA>(B0.a_sc + part * CA, asc);
            float v[MBLK][CW];
#pragma unroll
            for (int mb = 0; mb < MBLK; mb++) {
                const uint32_t n = (uint32_t)(128 * mb + 32 * quad + lane);
                const uint32_t rl = (uint32_t)B0.n_lo[n & 31u] ^ (uint32_t)B0.n_hi[n >> 5];
#pragma unroll
                for (int a2 = 0; a2 < CA; a2++) {
                    const float2 x = R[rl ^ asc[a2]];
                    v[mb][2 * a2] = x.x;
                    v[mb][2 * a2 + 1] = x.y;
                }
            }
            put_rows(s, v);
            // every thread's reads of the buffer are done before it is refilled
            if (!epi_sync_and(got)) return false;
            if (tid == 0) counts[6 + rb]++;
            if (j + NR < my_tiles) issue_load(j + NR);
            return true;
        };

        // one step of slot s: wait for its MMAs, then its next operand or its output
        auto step = [&](int s, bool& act, int& blk, uint64_t& tj, uint32_t& mpar) {
            if (!act || !ok) return;
            const bool got = mbar_wait_abort(bar_mma + s, mpar, abort_flag);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float v[MBLK][CW], w[MBLK][CW];
            const uint32_t dcol = tmem + (uint32_t)s * kSlotCols + lane_base + 2u * PLANE + (uint32_t)(part * CW);
#pragma unroll
            for (int mb = 0; mb < MBLK; mb++) {
                tmem_ld_cols<CW>(dcol + (uint32_t)(mb * DN), v[mb]);
                tmem_ld_cols<CW>(dcol + (uint32_t)(mb * DN + N), w[mb]);
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
#pragma unroll
            for (int mb = 0; mb < MBLK; mb++)
#pragma unroll
                for (int i = 0; i < CW; i++) v[mb][i] += w[mb][i];
            const FusedBlock& B = sb[blk];
            uint32_t na[CA];
            load_u16<CA>(B.nxt_a + part * CA, na);
            float2* T = trans + tsel * 4096u;
            tsel ^= 1u;
            // D rows into the transpose buffer: the next block's row order, or (last block)
            // local-index order as the output stage
#pragma unroll
            for (int mb = 0; mb < MBLK; mb++) {
                const uint32_t n = (uint32_t)(128 * mb + 32 * quad + lane);
                const uint32_t wn = (uint32_t)B.nxt_nlo[n & 31u] ^ (uint32_t)B.nxt_nhi[n >> 5];
#pragma unroll
                for (int a2 = 0; a2 < CA; a2++)
                    T[wn ^ na[a2]] = make_float2(v[mb][2 * a2], v[mb][2 * a2 + 1]);
            }
            if (!epi_sync_and(got)) { ok = false; return; }
            mpar ^= 1u;
            if (tid == 0) counts[2 + s]++;
            const float4* t4 = reinterpret_cast<const float4*>(T);
            if (blk + 1 < nb) {
                // this thread's rows of the next block, one 8-byte read per amplitude at its
                // transpose slot (the 16 lanes of a half warp, rows n..n+15, hit 16 bank
                // pairs: fused_slot puts row bits 0..2 on the chunk and row bit 3 on the word)
#pragma unroll
                for (int mb = 0; mb < MBLK; mb++) {
                    const uint32_t n = (uint32_t)(128 * mb + 32 * quad + lane);
#pragma unroll
                    for (int a2 = 0; a2 < CA; a2++) {
                        const float2 x = T[fused_slot(n, (uint32_t)(part * CA + a2), K)];
                        v[mb][2 * a2] = x.x;
                        v[mb][2 * a2 + 1] = x.y;
                    }
                }
                blk++;
                put_rows(s, v);
            } else {
                // the tile out in 16-byte pieces (4 threads per 64-byte run of the state)
                float2* dst = sv + tile_base(tj);
#pragma unroll
                for (int i = 0; i < CHUNKS; i++) {
                    float4 x = t4[oslot[i] >> 1];
                    if (oslot[i] & 1u) x = make_float4(x.z, x.w, x.x, x.y);
                    *reinterpret_cast<float4*>(dst + goff[i]) = x;
                }
                if (next_j < my_tiles) {
                    tj = next_j++;
                    blk = 0;
                    ok = start(s, tj);
                } else {
                    act = false;
                }
            }
        };

        for (uint64_t j = 0; j < NR && j < my_tiles; j++) issue_load(j);
        tj0 = next_j++;
        act0 = true;
        ok = start(0, tj0);
        if (ok && next_j < my_tiles) {
            tj1 = next_j++;
            act1 = true;
            ok = start(1, tj1);
        }
        while (ok && (act0 || act1)) {
            step(0, act0, blk0, tj0, mpar0);
            step(1, act1, blk1, tj1, mpar1);
        }
        if (!ok) *abort_flag = 1;
    }

    __syncthreads();
    if (!plan_ok && tid == 0) atomicExch(err, 1);
    if (*abort_flag && tid == 0) {
        atomicExch(err, 1);
        // let what is still in flight land before the memory goes away (bounded waits)
        for (int s = 0; s < 2; s++)
            for (uint32_t c = counts[2 + s]; c < counts[s]; c++) mbar_wait(bar_mma + s, c & 1u);
        for (uint32_t rb = 0; rb < NR; rb++)
            for (uint32_t c = counts[6 + rb]; c < counts[4 + rb]; c++) mbar_wait(bar_load + rb, c & 1u);
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
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        ctas[dev] = sms;                 // one CTA per SM (all of its tensor memory)
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

// The pair engine's per-tile machinery, shared by its one-circuit kernel
// (kernels_pairs.cu) and the batched-circuit kernel (circuit_batch.cu).
//
// A CTA of 256 threads holds a tile of 4,096 amplitudes, 16 complex<double> per thread.
// In the current layout lane bits 0 and 1 hold the block's two qubits, so the four lanes t
// with equal t >> 2 hold the four amplitudes a = t & 3 of one "vector", and the 8 lane
// groups of a warp hold 8 vectors.  For every two register slots the block is one m16n8k8
// f64 MMA,
//     D^T = X^T G'^T  (16 vectors x 8 outputs = 16 x 8 inputs . 8 x 8)
// (A fragment = the thread's real parts (K = 0..3) and imaginary parts (K = 4..7) of its
// two slots; B = the lane's two entries of the real 8x8 form G'), and the 4 accumulator
// registers a thread gets back are the real and imaginary parts of its own output
// amplitude a' = t & 3 in both slots.  So the tile never leaves the registers between
// blocks on the same pair.  A PO_SWAP exchanges a lane bit with a register bit by one warp
// shuffle per moved word; a PO_LPERM permutes the lane bits by one indexed shuffle of
// every word; a PO_RELAYOUT sends the tile through shared memory with the staged engine's
// XOR swizzle.
#pragma once
#include "staged_core.cuh"

namespace svb {
namespace {


constexpr int PR_THREADS = 1 << (PR_TILE_BITS - RB);    // 256
constexpr int PR_NR = 1 << RB;                          // 16

// D (16 x 8) = A (16 x 8) . B (8 x 8), f64.  Lane 4g + t holds A[g][t], A[g+8][t],
// A[g][t+4], A[g+8][t+4]; B[t][g], B[t+4][g]; and gets D[g][2t], D[g][2t+1], D[g+8][2t],
// D[g+8][2t+1].
__device__ __forceinline__ void dmma16(double& d0, double& d1, double& d2, double& d3, double a0, double a1,
                                       double a2, double a3, double b0, double b1)
{
    asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%10,%10,%10,%10};"
        : "=d"(d0), "=d"(d1), "=d"(d2), "=d"(d3)
        : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1), "d"(0.0));
}

// exchange lane bit L with register bit R: the element at (lane bit i, register bit j)
// becomes the one that was at (lane bit j, register bit i)
template <int L, int R>
__device__ __forceinline__ void swap_lr(double2* v)
{
    const bool hi = (threadIdx.x >> L) & 1;
#pragma unroll
    for (int k = 0; k < PR_NR; k++) {
        if (k & (1 << R)) continue;
        const int k1 = k | (1 << R);
        const double2 send = hi ? v[k] : v[k1];
        double2 recv;
        recv.x = __shfl_xor_sync(0xffffffffu, send.x, 1 << L);
        recv.y = __shfl_xor_sync(0xffffffffu, send.y, 1 << L);
        if (hi) v[k] = recv;
        else v[k1] = recv;
    }
}

template <int L>
__device__ __forceinline__ void swap_l(double2* v, int r)
{
    switch (r) {
    case 0: swap_lr<L, 0>(v); break;
    case 1: swap_lr<L, 1>(v); break;
    case 2: swap_lr<L, 2>(v); break;
    default: swap_lr<L, 3>(v); break;
    }
}

__device__ __forceinline__ void swap_any(double2* v, int lane, int r)
{
    switch (lane) {
    case 0: swap_l<0>(v, r); break;
    case 1: swap_l<1>(v, r); break;
    case 2: swap_l<2>(v, r); break;
    case 3: swap_l<3>(v, r); break;
    default: swap_l<4>(v, r); break;
    }
}

struct PairGOffs {
    uint64_t thr;
    uint64_t reg[RB];
};

__device__ __forceinline__ void pair_goffs(const DevStage& S, const uint8_t* local_q, int tid, PairGOffs& g)
{
    uint64_t t = 0;
#pragma unroll
    for (int b = 0; b < PR_TILE_BITS - RB; b++)
        if ((tid >> b) & 1) t |= 1ull << local_q[S.thr_pos[b]];
    g.thr = t;
#pragma unroll
    for (int i = 0; i < RB; i++) g.reg[i] = 1ull << local_q[S.reg_pos[i]];
}

__device__ __forceinline__ uint64_t pair_goff(const PairGOffs& g, int k)
{
    uint64_t r = g.thr;
#pragma unroll
    for (int i = 0; i < RB; i++)
        if ((k >> i) & 1) r |= g.reg[i];
    return r;
}

// A pass's ops, layouts and (when they fit) gate fragments in shared memory beside the
// tile, copied once per CTA and pass so that the op loop reads no global memory but the
// tile.  P is in shared memory already; ends with a barrier.
struct PairStaged {
    const PairOp* ops;
    const DevStage* lay;
    const double2* G;
    int n_ops;
    int n_lay;
};

__device__ __forceinline__ PairStaged pair_stage(unsigned char* smem_raw, const PairPass& P,
                                                 const PairOp* __restrict__ ops,
                                                 const DevStage* __restrict__ layouts,
                                                 const double2* __restrict__ gates, int tid)
{
    PairStaged S;
    S.n_ops = P.op_end - P.op_begin;
    S.n_lay = P.store_layout - P.load_layout + 1;
    PairOp* sops = reinterpret_cast<PairOp*>(smem_raw + (sizeof(double2) << PR_TILE_BITS));
    DevStage* slay = reinterpret_cast<DevStage*>(reinterpret_cast<unsigned char*>(sops) + 16 * (size_t)S.n_ops);
    double2* sg = reinterpret_cast<double2*>(reinterpret_cast<unsigned char*>(slay) +
                                             ((24 * (size_t)S.n_lay + 15) / 16) * 16);
    const uint4* o4 = reinterpret_cast<const uint4*>(ops + P.op_begin);
    for (int w = tid; w < S.n_ops; w += PR_THREADS) reinterpret_cast<uint4*>(sops)[w] = o4[w];
    const uint32_t* l4 = reinterpret_cast<const uint32_t*>(layouts + P.load_layout);
    for (int w = tid; w < S.n_lay * 6; w += PR_THREADS) reinterpret_cast<uint32_t*>(slay)[w] = l4[w];
    if (P.stage_gates) {
        const double2* g = gates + (size_t)P.gate_begin * 32;
        for (int w = tid; w < P.gate_count * 32; w += PR_THREADS) sg[w] = g[w];
    }
    __syncthreads();
    S.ops = sops;
    S.lay = slay;
    S.G = P.stage_gates ? sg : gates + (size_t)P.gate_begin * 32;
    return S;
}

// One tile of pass P: load, the pass's ops in order, store.  sv is the state the pass's
// offsets are relative to; sm the 64 KiB tile area of shared memory.
__device__ __forceinline__ void pair_tile(double2* __restrict__ sv, double2* sm, const PairPass& P,
                                          const PairStaged& S, const PairGOffs& gin, const PairGOffs& gout,
                                          uint64_t tile, int tid, int lane)
{
    const PairOp* sops = S.ops;
    const DevStage* slay = S.lay;
    const double2* G = S.G;
    const int n_ops = S.n_ops;
    uint64_t base = 0;
    for (int j = 0; j < P.n_nonlocal; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];
    double2 v[PR_NR];
#pragma unroll
    for (int k = 0; k < PR_NR; k++) v[k] = sv[base | pair_goff(gin, k)];
    for (int o = 0; o < n_ops; o++) {
        const PairOp op = sops[o];
        if (op.kind == PO_BLOCK) {
            static_assert(PR_MAX_COND == 2, "condition qubits of a block");
            int var = 0;
            if (op.ncond > 0) var |= (int)((base >> op.cond_q[0]) & 1ull);
            if (op.ncond > 1) var |= (int)((base >> op.cond_q[1]) & 1ull) << 1;
            const double2 g = G[(size_t)((int)op.gate - P.gate_begin + var) * 32 + lane];
            // two register slots per MMA: slot k as rows g, slot k + 1 as rows g + 8;
            // K = 8 takes the real parts (k < 4) and the imaginary parts (k >= 4)
#pragma unroll
            for (int k = 0; k < PR_NR; k += 2) {
                double d0, d1, d2, d3;
                dmma16(d0, d1, d2, d3, v[k].x, v[k + 1].x, v[k].y, v[k + 1].y, g.x, g.y);
                v[k].x = d0;
                v[k].y = d1;
                v[k + 1].x = d2;
                v[k + 1].y = d3;
            }
        } else if (op.kind == PO_SWAP) {
            swap_any(v, op.lane, op.reg);
        } else if (op.kind == PO_LPERM) {
            // lane bit b takes the element of lane bit from[b]: read every register
            // from the lane whose bit from[b] is this lane's bit b
            int src = 0;
#pragma unroll
            for (int b = 0; b < PR_LANE_BITS; b++) src |= ((lane >> b) & 1) << ((op.gate >> (3 * b)) & 7u);
#pragma unroll
            for (int k = 0; k < PR_NR; k++) {
                v[k].x = __shfl_sync(0xffffffffu, v[k].x, src);
                v[k].y = __shfl_sync(0xffffffffu, v[k].y, src);
            }
        } else {
            Slots from, to;
            make_slots<double, PR_TILE_BITS - RB>(slay[op.src - P.load_layout], tid, from);
            make_slots<double, PR_TILE_BITS - RB>(slay[op.layout - P.load_layout], tid, to);
#pragma unroll
            for (int k = 0; k < PR_NR; k++) sm[slot_of(from, k)] = v[k];
            __syncthreads();
#pragma unroll
            for (int k = 0; k < PR_NR; k++) v[k] = sm[slot_of(to, k)];
            __syncthreads();
        }
    }
#pragma unroll
    for (int k = 0; k < PR_NR; k++) sv[base | pair_goff(gout, k)] = v[k];
}

}  // namespace
}  // namespace svb

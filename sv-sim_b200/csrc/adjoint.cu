// Adjoint differentiation (no counterpart in the reference).
//
// E(p) = <psi| H |psi>, psi = U_K ... U_1 |0..0>, U_k the elementary ops of the
// circuit (the reference's composite sequences, lower.cpp).  After the forward pass
// lambda = H psi.  Walking k = K..1:
//     psi    <- U_k^dagger psi            (psi is now the state before op k)
//     g[k,i] =  Re <lambda| dU_k/d ang_i |psi>
//     lambda <- U_k^dagger lambda
// and dE/dp = 2 sum_{k,i,f} g[k,i] * d ang_i / d field_f * d field_f / d p.
// Only psi and lambda are held; to bound the drift of the reverse-propagated psi the
// forward pass stores checkpoints, and psi is reloaded from them on the way back.
// Every reduction is FP64 with a fixed order (per-block partials, then one pass).
// The forward pass runs on the pair engine (n >= 12; all segments planned before the
// first launch, so the GPU never waits for the host) or the staged engine below; the
// reverse sweep is tiled: its inverse ops
// are cut into passes of local qubits, and each tile of psi and lambda goes through a
// pass's ops in shared memory, leaving one derivative sum per tile and parameter slot.
#include <cmath>
#include <cstring>
#include <algorithm>
#include <string>

#include "gate_math.cuh"

namespace svb {

enum { EK_CONST = 0, EK_U3 = 1, EK_U2 = 2, EK_U1 = 3, EK_RX = 4, EK_RY = 5, EK_R = 6 };

namespace {

constexpr int ADJ_BLOCKS = 296;   // 2 x 148 SMs
constexpr int ADJ_THREADS = 256;


__device__ __forceinline__ double block_sum(double v, double* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    return s;
}

// ---- the reverse sweep, tiled -------------------------------------------------------
// The inverse ops in reverse order are cut into passes (select_passes) of AT_M local
// qubits.  A CTA loads a tile of psi and of lambda into shared memory, applies the pass's
// ops in order (for each: psi <- U^dagger psi, the derivative sums Re <lambda| dU |psi>,
// lambda <- U^dagger lambda) and writes the tile back; a differentiated op leaves one
// block-reduced sum per tile and slot in `partial` (row = slot, column = tile).
constexpr int AT_M = 10;                  // 1,024 amplitudes of psi and of lambda: 32 KiB
constexpr int AT_THREADS = 256;
constexpr int AT_MAX_LSLOTS = 128;   // derivative slots of one pass at most (a pass with more is split)

enum { AT_C1 = 0, AT_DIAG = 1, AT_CX = 2 };

struct AdjTileOp {
    uint8_t kind;      // AT_C1 (target local), AT_DIAG, AT_CX (target local)
    uint8_t p;         // local position of the target
    uint8_t c;         // AT_CX: local position of the control
    uint8_t flags;     // bit 0: the DIAG qubit is a tile bit; bit 1: the CX control is
    uint8_t nd;        // derivative slots (AT_C1 only)
    uint8_t tile_bit;  // tile-index bit of a tile-bit qubit
    uint8_t pad[2];
    int32_t pad2;
    int32_t lslot;     // its first derivative slot among the pass's slots (the global
                       // slot numbers are in the pass's table)
    double m[8];       // the inverse op: C1 2x2, or d0, d1 for DIAG
    double dm[3][8];   // derivative matrices, C1 layout
};
static_assert(sizeof(AdjTileOp) % 16 == 0, "AdjTileOp layout");

struct AdjTilePass {
    uint8_t nonlocal_q[64];
    uint64_t g_lo[64];         // local index bits 0-5 -> global offset
    uint64_t g_hi[32];         // local index bits 6-10 -> global offset
    int32_t n_nonlocal, op_begin, op_end;
    int32_t n_lslots;          // derivative slots of the pass's ops
    int32_t lslot_begin;       // their global slot numbers: lslots[lslot_begin + local slot]
    int32_t stage_begin, stage_end;   // k_adj_stages: the pass's register stages
    int32_t pad;
};
static_assert(sizeof(AdjTilePass) % 16 == 0, "AdjTilePass layout");

__global__ void __launch_bounds__(AT_THREADS, 3)
k_adj_tiles(double2* __restrict__ psi, double2* __restrict__ lam, const AdjTilePass* __restrict__ passes,
            int pass_index, const AdjTileOp* __restrict__ ops, const int32_t* __restrict__ lslots, int M,
            uint64_t tiles, double* __restrict__ partial)
{
    // shared memory: the psi and lambda tiles, then each warp's derivative sums per slot
    // of the pass (reduced over the warps once per tile)
    extern __shared__ __align__(16) double2 at_sm[];
    __shared__ AdjTilePass P;
    constexpr int WARPS = AT_THREADS / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    {
        const uint4* src = reinterpret_cast<const uint4*>(passes + pass_index);
        uint4* dst = reinterpret_cast<uint4*>(&P);
        for (int w = threadIdx.x; w < (int)(sizeof(AdjTilePass) / 16); w += AT_THREADS) dst[w] = src[w];
        __syncthreads();
    }
    const uint32_t T = 1u << M;
    double2* sp = at_sm;
    double2* sl = at_sm + T;
    double* wsum = reinterpret_cast<double*>(at_sm + 2 * T);      // [local slot][warp]
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        uint64_t base = 0;
        for (int j = 0; j < P.n_nonlocal; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];
        for (uint32_t l = threadIdx.x; l < T; l += AT_THREADS) {
            const uint64_t g = base + P.g_lo[l & 63u] + P.g_hi[l >> 6];
            sp[l] = psi[g];
            sl[l] = lam[g];
        }
        __syncthreads();
        for (int o = P.op_begin; o < P.op_end; o++) {
            const AdjTileOp& op = ops[o];
            const uint4 hdr = __ldg(reinterpret_cast<const uint4*>(&op));
            const int kind = hdr.x & 0xFFu, p = (hdr.x >> 8) & 0xFFu, flags = hdr.x >> 24;
            const int nd = hdr.y & 0xFFu, tbit = (hdr.y >> 8) & 0xFFu, lslot = (int)hdr.w;
            Coef<double> inv;
            {
                const double2* m2 = reinterpret_cast<const double2*>(op.m);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const double2 v = __ldg(m2 + j);
                    inv.m[2 * j] = v.x;
                    inv.m[2 * j + 1] = v.y;
                }
            }
            if (kind == AT_C1) {
                double acc[3] = {0.0, 0.0, 0.0};
                for (uint32_t i = threadIdx.x; i < T / 2; i += AT_THREADS) {
                    const uint32_t p0 = (uint32_t)insert_zero(i, p), p1 = p0 | (1u << p);
                    double2 s0 = sp[p0], s1 = sp[p1];
                    double2 l0 = sl[p0], l1 = sl[p1];
                    dense_pair<double>(F_C1, inv, s0, s1);
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        if (d >= nd) break;
                        double m[8];
                        const double2* m2 = reinterpret_cast<const double2*>(op.dm[d]);
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const double2 v = __ldg(m2 + j);
                            m[2 * j] = v.x;
                            m[2 * j + 1] = v.y;
                        }
                        const double u0r = m[0] * s0.x - m[1] * s0.y + m[2] * s1.x - m[3] * s1.y;
                        const double u0i = m[0] * s0.y + m[1] * s0.x + m[2] * s1.y + m[3] * s1.x;
                        const double u1r = m[4] * s0.x - m[5] * s0.y + m[6] * s1.x - m[7] * s1.y;
                        const double u1i = m[4] * s0.y + m[5] * s0.x + m[6] * s1.y + m[7] * s1.x;
                        acc[d] += l0.x * u0r + l0.y * u0i + l1.x * u1r + l1.y * u1i;
                    }
                    dense_pair<double>(F_C1, inv, l0, l1);
                    sp[p0] = s0; sp[p1] = s1;
                    sl[p0] = l0; sl[p1] = l1;
                }
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    if (d >= nd) break;
                    double v = acc[d];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0) wsum[(lslot + d) * WARPS + warp] = v;
                }
            } else if (kind == AT_DIAG) {
                const bool tile_bit = flags & 1;
                const bool one_tile = tile_bit && ((tile >> tbit) & 1ull);
                for (uint32_t l = threadIdx.x; l < T; l += AT_THREADS) {
                    const bool one = tile_bit ? one_tile : ((l >> p) & 1u);
                    double2 a = sp[l], b = sl[l];
                    if (one) { diag_one<double>(F_DIAG, inv, a); diag_one<double>(F_DIAG, inv, b); }
                    else { diag_zero<double>(F_DIAG, inv, a); diag_zero<double>(F_DIAG, inv, b); }
                    sp[l] = a;
                    sl[l] = b;
                }
            } else {
                const uint32_t pd = 1u << p;
                if (flags & 2) {
                    if ((tile >> tbit) & 1ull) {
                        for (uint32_t i = threadIdx.x; i < T / 2; i += AT_THREADS) {
                            const uint32_t p0 = (uint32_t)insert_zero(i, p), p1 = p0 | pd;
                            const double2 a0 = sp[p0], a1 = sp[p1], b0 = sl[p0], b1 = sl[p1];
                            sp[p0] = a1; sp[p1] = a0;
                            sl[p0] = b1; sl[p1] = b0;
                        }
                    }
                } else {
                    const int c = (hdr.x >> 16) & 0xFFu;
                    const int lo = c < p ? c : p, hi = c < p ? p : c;
                    for (uint32_t i = threadIdx.x; i < T / 4; i += AT_THREADS) {
                        const uint32_t b = (uint32_t)insert_zero(insert_zero(i, lo), hi) | (1u << c);
                        const uint32_t p0 = b, p1 = b | pd;
                        const double2 a0 = sp[p0], a1 = sp[p1], b0 = sl[p0], b1 = sl[p1];
                        sp[p0] = a1; sp[p1] = a0;
                        sl[p0] = b1; sl[p1] = b0;
                    }
                }
            }
            __syncthreads();
        }
        for (uint32_t l = threadIdx.x; l < T; l += AT_THREADS) {
            const uint64_t g = base + P.g_lo[l & 63u] + P.g_hi[l >> 6];
            psi[g] = sp[l];
            lam[g] = sl[l];
        }
        // the tile's derivative sums, warps added in a fixed order (the barrier after the
        // last op made every warp's sums visible)
        for (int j = threadIdx.x; j < P.n_lslots; j += AT_THREADS) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < WARPS; w++) v += wsum[j * WARPS + w];
            partial[(uint64_t)lslots[P.lslot_begin + j] * tiles + tile] = v;
        }
        __syncthreads();
    }
}

// ---- the reverse sweep with register stages (tiles of exactly AT_M = 10 qubits) ------
// The same passes as k_adj_tiles, but inside a pass the ops are grouped into stages whose
// dense and CX targets lie on 3 "register" positions of the tile: each of 128 threads
// keeps the 8 amplitudes of psi and of lambda that differ in those positions in
// registers, applies the stage's ops there, and the tile goes through shared memory once
// per stage instead of once per op (k_adj_tiles was bound by its shared-memory sweeps:
// L1 throughput 79%, FP64 pipe 21%).
constexpr int AS_THREADS = 1 << (AT_M - 3);   // 128
constexpr int AS_R = 8;                       // amplitudes of each state per thread

struct AdjStage {
    uint8_t rp[3];      // local positions held in register bits 0..2
    uint8_t tp[7];      // local positions of thread-index bits 0..6
    uint8_t pad[6];
    int32_t op_begin, op_end;
    int32_t pad2[2];
};
static_assert(sizeof(AdjStage) == 32, "AdjStage layout");

enum { AS_LOC_REG = 0, AS_LOC_THREAD = 1, AS_LOC_TILE = 2 };

struct AdjStageOp {
    uint8_t kind;      // AT_C1, AT_DIAG, AT_CX
    uint8_t j;         // C1 / CX: register bit of the target; DIAG: bit of the qubit in its location
    uint8_t c;         // CX: bit of the control in its location
    uint8_t loc;       // DIAG qubit / CX control: AS_LOC_REG, AS_LOC_THREAD or AS_LOC_TILE
    uint8_t nd;        // derivative slots (AT_C1)
    uint8_t pad[3];
    int32_t lslot;
    int32_t pad2;
    double m[8];
    double dm[3][8];
};
static_assert(sizeof(AdjStageOp) % 16 == 0, "AdjStageOp layout");

template <int J>
__device__ __forceinline__ void as_c1(double2* vp, double2* vl, const Coef<double>& inv, const double (*dm)[8],
                                      int nd, double* acc)
{
#pragma unroll
    for (int r = 0; r < AS_R; r++) {
        if (r & (1 << J)) continue;
        const int r1 = r | (1 << J);
        double2 s0 = vp[r], s1 = vp[r1];
        double2 l0 = vl[r], l1 = vl[r1];
        dense_pair<double>(F_C1, inv, s0, s1);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (d >= nd) break;
            const double* m = dm[d];
            const double u0r = m[0] * s0.x - m[1] * s0.y + m[2] * s1.x - m[3] * s1.y;
            const double u0i = m[0] * s0.y + m[1] * s0.x + m[2] * s1.y + m[3] * s1.x;
            const double u1r = m[4] * s0.x - m[5] * s0.y + m[6] * s1.x - m[7] * s1.y;
            const double u1i = m[4] * s0.y + m[5] * s0.x + m[6] * s1.y + m[7] * s1.x;
            acc[d] += l0.x * u0r + l0.y * u0i + l1.x * u1r + l1.y * u1i;
        }
        dense_pair<double>(F_C1, inv, l0, l1);
        vp[r] = s0;
        vp[r1] = s1;
        vl[r] = l0;
        vl[r1] = l1;
    }
}

template <int J>
__device__ __forceinline__ void as_swap_all(double2* vp, double2* vl)
{
#pragma unroll
    for (int r = 0; r < AS_R; r++) {
        if (r & (1 << J)) continue;
        const int r1 = r | (1 << J);
        const double2 a = vp[r], b = vl[r];
        vp[r] = vp[r1];
        vp[r1] = a;
        vl[r] = vl[r1];
        vl[r1] = b;
    }
}

template <int J, int C>
__device__ __forceinline__ void as_swap_ctrl(double2* vp, double2* vl)
{
#pragma unroll
    for (int r = 0; r < AS_R; r++) {
        if ((r & (1 << J)) || !(r & (1 << C))) continue;
        const int r1 = r | (1 << J);
        const double2 a = vp[r], b = vl[r];
        vp[r] = vp[r1];
        vp[r1] = a;
        vl[r] = vl[r1];
        vl[r1] = b;
    }
}

template <int J>
__device__ __forceinline__ void as_diag_reg(double2* vp, double2* vl, const Coef<double>& inv)
{
#pragma unroll
    for (int r = 0; r < AS_R; r++) {
        if (r & (1 << J)) {
            diag_one<double>(F_DIAG, inv, vp[r]);
            diag_one<double>(F_DIAG, inv, vl[r]);
        } else {
            diag_zero<double>(F_DIAG, inv, vp[r]);
            diag_zero<double>(F_DIAG, inv, vl[r]);
        }
    }
}

__global__ void __launch_bounds__(AS_THREADS, 3)
k_adj_stages(double2* __restrict__ psi, double2* __restrict__ lam, const AdjTilePass* __restrict__ passes,
             int pass_index, const AdjStage* __restrict__ stages, const AdjStageOp* __restrict__ ops,
             const int32_t* __restrict__ lslots, uint64_t tiles, double* __restrict__ partial)
{
    extern __shared__ __align__(16) double2 as_sm[];
    __shared__ AdjTilePass P;
    constexpr int WARPS = AS_THREADS / 32;
    constexpr uint32_t T = 1u << AT_M;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        const uint4* src = reinterpret_cast<const uint4*>(passes + pass_index);
        uint4* dst = reinterpret_cast<uint4*>(&P);
        for (int w = tid; w < (int)(sizeof(AdjTilePass) / 16); w += AS_THREADS) dst[w] = src[w];
        __syncthreads();
    }
    double2* sp = as_sm;
    double2* sl = as_sm + T;
    double* wsum = reinterpret_cast<double*>(as_sm + 2 * T);      // [local slot][warp]
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        uint64_t base = 0;
        for (int j = 0; j < P.n_nonlocal; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];
        for (uint32_t l = tid; l < T; l += AS_THREADS) {
            const uint64_t g = base + P.g_lo[l & 63u] + P.g_hi[l >> 6];
            sp[l] = psi[g];
            sl[l] = lam[g];
        }
        __syncthreads();
        for (int st = P.stage_begin; st < P.stage_end; st++) {
            const AdjStage S = stages[st];
            uint32_t tb = 0;
#pragma unroll
            for (int b = 0; b < 7; b++) tb |= (uint32_t)((tid >> b) & 1) << S.tp[b];
            const uint32_t o0 = 1u << S.rp[0], o1 = 1u << S.rp[1], o2 = 1u << S.rp[2];
            double2 vp[AS_R], vl[AS_R];
#pragma unroll
            for (int r = 0; r < AS_R; r++) {
                const uint32_t l = tb | ((r & 1) ? o0 : 0u) | ((r & 2) ? o1 : 0u) | ((r & 4) ? o2 : 0u);
                vp[r] = sp[l];
                vl[r] = sl[l];
            }
            for (int o = S.op_begin; o < S.op_end; o++) {
                const AdjStageOp& op = ops[o];
                const uint4 hdr = __ldg(reinterpret_cast<const uint4*>(&op));
                const int kind = hdr.x & 0xFFu, j = (hdr.x >> 8) & 0xFFu, c = (hdr.x >> 16) & 0xFFu;
                const int loc = hdr.x >> 24, nd = hdr.y & 0xFFu, lslot = (int)hdr.z;
                Coef<double> inv;
                {
                    const double2* m2 = reinterpret_cast<const double2*>(op.m);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const double2 v = __ldg(m2 + q);
                        inv.m[2 * q] = v.x;
                        inv.m[2 * q + 1] = v.y;
                    }
                }
                if (kind == AT_C1) {
                    double dm[3][8];
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        const double2* m2 = reinterpret_cast<const double2*>(op.dm[d]);
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const double2 v = d < nd ? __ldg(m2 + q) : make_double2(0.0, 0.0);
                            dm[d][2 * q] = v.x;
                            dm[d][2 * q + 1] = v.y;
                        }
                    }
                    double acc[3] = {0.0, 0.0, 0.0};
                    if (j == 0) as_c1<0>(vp, vl, inv, dm, nd, acc);
                    else if (j == 1) as_c1<1>(vp, vl, inv, dm, nd, acc);
                    else as_c1<2>(vp, vl, inv, dm, nd, acc);
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        if (d >= nd) break;
                        double v = acc[d];
#pragma unroll
                        for (int sh = 16; sh > 0; sh >>= 1) v += __shfl_xor_sync(0xffffffffu, v, sh);
                        if (lane == 0) wsum[(lslot + d) * WARPS + warp] = v;
                    }
                } else if (kind == AT_CX) {
                    if (loc == AS_LOC_REG) {
                        if (j == 0) { if (c == 1) as_swap_ctrl<0, 1>(vp, vl); else as_swap_ctrl<0, 2>(vp, vl); }
                        else if (j == 1) { if (c == 0) as_swap_ctrl<1, 0>(vp, vl); else as_swap_ctrl<1, 2>(vp, vl); }
                        else { if (c == 0) as_swap_ctrl<2, 0>(vp, vl); else as_swap_ctrl<2, 1>(vp, vl); }
                    } else {
                        const bool on = loc == AS_LOC_THREAD ? ((tid >> c) & 1) : ((tile >> c) & 1ull);
                        if (on) {
                            if (j == 0) as_swap_all<0>(vp, vl);
                            else if (j == 1) as_swap_all<1>(vp, vl);
                            else as_swap_all<2>(vp, vl);
                        }
                    }
                } else {                     // AT_DIAG
                    if (loc == AS_LOC_REG) {
                        if (j == 0) as_diag_reg<0>(vp, vl, inv);
                        else if (j == 1) as_diag_reg<1>(vp, vl, inv);
                        else as_diag_reg<2>(vp, vl, inv);
                    } else {
                        const bool one = loc == AS_LOC_THREAD ? ((tid >> j) & 1) : ((tile >> j) & 1ull);
#pragma unroll
                        for (int r = 0; r < AS_R; r++) {
                            if (one) {
                                diag_one<double>(F_DIAG, inv, vp[r]);
                                diag_one<double>(F_DIAG, inv, vl[r]);
                            } else {
                                diag_zero<double>(F_DIAG, inv, vp[r]);
                                diag_zero<double>(F_DIAG, inv, vl[r]);
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < AS_R; r++) {
                const uint32_t l = tb | ((r & 1) ? o0 : 0u) | ((r & 2) ? o1 : 0u) | ((r & 4) ? o2 : 0u);
                sp[l] = vp[r];
                sl[l] = vl[r];
            }
            __syncthreads();
        }
        for (uint32_t l = tid; l < T; l += AS_THREADS) {
            const uint64_t g = base + P.g_lo[l & 63u] + P.g_hi[l >> 6];
            psi[g] = sp[l];
            lam[g] = sl[l];
        }
        // the tile's derivative sums, warps added in a fixed order (the barrier after the
        // last stage made every warp's sums visible)
        for (int q = tid; q < P.n_lslots; q += AS_THREADS) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < WARPS; w++) v += wsum[q * WARPS + w];
            partial[(uint64_t)lslots[P.lslot_begin + q] * tiles + tile] = v;
        }
        __syncthreads();
    }
}

// out = sum_t coef_t P_t psi
__global__ void __launch_bounds__(256)
k_pauli_apply(const double2* __restrict__ psi, double2* __restrict__ out, uint64_t dim,
              const svb_pauli_term* __restrict__ terms, int n_terms)
{
    extern __shared__ svb_pauli_term sterms[];
    for (int t = threadIdx.x; t < n_terms; t += blockDim.x) sterms[t] = terms[t];
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
        double accr = 0.0, acci = 0.0;
        for (int t = 0; t < n_terms; t++) {
            const uint64_t j = i ^ sterms[t].x_mask;
            const double2 b = psi[j];
            double br = b.x, bi = b.y;
            if (__popcll(j & sterms[t].z_mask) & 1) { br = -br; bi = -bi; }
            double tr, ti;
            switch (__popcll(sterms[t].x_mask & sterms[t].z_mask) & 3) {
            case 0: tr = br; ti = bi; break;
            case 1: tr = -bi; ti = br; break;
            case 2: tr = -br; ti = -bi; break;
            default: tr = bi; ti = -br; break;
            }
            accr += sterms[t].coef * tr;
            acci += sterms[t].coef * ti;
        }
        out[i] = make_double2(accr, acci);
    }
}

__global__ void __launch_bounds__(256)
k_inner_re(const double2* __restrict__ a, const double2* __restrict__ b, uint64_t dim,
           double* __restrict__ partial)
{
    __shared__ double red[8];
    double acc = 0.0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
        const double2 x = a[i], y = b[i];
        acc += x.x * y.x + x.y * y.y;
    }
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// results[r] = sum of partial[r * stride + i], i < nblocks; one warp per result, fixed order
__global__ void k_reduce_rows(const double* __restrict__ partial, int nblocks, uint64_t stride, int rows,
                              double* __restrict__ results)
{
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= rows) return;
    double s = 0.0;
    for (int i = lane; i < nblocks; i += 32) s += partial[(size_t)row * stride + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) results[row] = s;
}

unsigned adj_grid(uint64_t items)
{
    const uint64_t need = (items + ADJ_THREADS - 1) / ADJ_THREADS;
    return (unsigned)std::min<uint64_t>(std::max<uint64_t>(need, 1), ADJ_BLOCKS);
}

// d M / d ang_i for the elementary kinds, C1 layout.  Returns false if the op has no
// derivative with respect to ang_i.
bool deriv_matrix(const EOp& e, int i, double* m)
{
    std::memset(m, 0, 8 * sizeof(double));
    const double S2I = 0.70710678118654752440;
    switch (e.kind) {
    case EK_U3: {
        const double th = e.ang[0], ph = e.ang[1], la = e.ang[2];
        const double c = std::cos(th / 2), s = std::sin(th / 2);
        if (i == 0) {
            m[0] = -0.5 * s;
            m[2] = -0.5 * std::cos(la) * c; m[3] = -0.5 * std::sin(la) * c;
            m[4] = 0.5 * std::cos(ph) * c;  m[5] = 0.5 * std::sin(ph) * c;
            m[6] = -0.5 * std::cos(ph + la) * s; m[7] = -0.5 * std::sin(ph + la) * s;
        } else if (i == 1) {
            m[4] = -std::sin(ph) * s; m[5] = std::cos(ph) * s;
            m[6] = -std::sin(ph + la) * c; m[7] = std::cos(ph + la) * c;
        } else {
            m[2] = std::sin(la) * s; m[3] = -std::cos(la) * s;
            m[6] = -std::sin(ph + la) * c; m[7] = std::cos(ph + la) * c;
        }
        return true;
    }
    case EK_U2: {
        const double ph = e.ang[1], la = e.ang[2];
        if (i == 1) {
            m[4] = -S2I * std::sin(ph); m[5] = S2I * std::cos(ph);
            m[6] = -S2I * std::sin(ph + la); m[7] = S2I * std::cos(ph + la);
            return true;
        }
        if (i == 2) {
            m[2] = S2I * std::sin(la); m[3] = -S2I * std::cos(la);
            m[6] = -S2I * std::sin(ph + la); m[7] = S2I * std::cos(ph + la);
            return true;
        }
        return false;
    }
    case EK_U1:
        if (i != 2) return false;
        m[6] = -std::sin(e.ang[2]);
        m[7] = std::cos(e.ang[2]);
        return true;
    case EK_RX: {
        if (i != 0) return false;
        const double c = std::cos(e.ang[0] / 2), s = std::sin(e.ang[0] / 2);
        m[0] = -0.5 * s; m[3] = -0.5 * c; m[5] = -0.5 * c; m[6] = -0.5 * s;
        return true;
    }
    case EK_RY: {
        if (i != 0) return false;
        const double c = std::cos(e.ang[0] / 2), s = std::sin(e.ang[0] / 2);
        m[0] = -0.5 * s; m[2] = -0.5 * c; m[4] = 0.5 * c; m[6] = -0.5 * s;
        return true;
    }
    default:
        return false;
    }
}

// U^dagger of an elementary op as an F_C1 / F_DIAG / F_CX op.
bool inverse_op(const EOp& e, EOp& inv)
{
    inv = e;
    const double S2I = 0.70710678118654752440;
    double* m = inv.m;
    auto c1 = [&](double a, double b, double c, double d, double e_, double f, double g, double h) {
        inv.form = F_C1;
        m[0] = a; m[1] = b; m[2] = c; m[3] = d; m[4] = e_; m[5] = f; m[6] = g; m[7] = h;
    };
    auto dg = [&](double a, double b, double c, double d) {
        inv.form = F_DIAG;
        std::memset(m, 0, 8 * sizeof(double));
        m[0] = a; m[1] = b; m[2] = c; m[3] = d;
    };
    switch (e.form) {
    case F_C1: c1(e.m[0], -e.m[1], e.m[4], -e.m[5], e.m[2], -e.m[3], e.m[6], -e.m[7]); return true;
    case F_X:  c1(0, 0, 1, 0, 1, 0, 0, 0); return true;
    case F_Y:  c1(0, 0, 0, -1, 0, 1, 0, 0); return true;
    case F_H:  c1(S2I, 0, S2I, 0, S2I, 0, -S2I, 0); return true;
    case F_W:  c1(S2I, 0, 0, S2I, 0, S2I, S2I, 0); return true;
    case F_RX: c1(e.m[0], 0, 0, -e.m[1], 0, -e.m[1], e.m[0], 0); return true;  // RX(-theta)
    case F_RY: c1(e.m[0], 0, e.m[2], 0, e.m[1], 0, e.m[3], 0); return true;   // transpose
    case F_Z:  dg(1, 0, -1, 0); return true;
    case F_S:  dg(1, 0, 0, -1); return true;
    case F_SDG: dg(1, 0, 0, 1); return true;
    case F_T:  dg(1, 0, S2I, -S2I); return true;
    case F_TDG: dg(1, 0, S2I, S2I); return true;
    case F_U1: dg(1, 0, e.m[0], -e.m[1]); return true;
    case F_DIAG: dg(e.m[0], -e.m[1], e.m[2], -e.m[3]); return true;
    case F_CX: return true;
    default: return false;   // F_R, F_SRN: not unitary
    }
}

}  // namespace

}  // namespace svb

using namespace svb;

namespace svb {
namespace {

// Appends the pair plan of one forward segment to `all`, shifting its indices; the
// kernel reads every index relative to its pass, so the passes of all segments can live
// in one set of device buffers.  False if the layout indices would overflow.
bool append_pair_plan(PairPlan& all, const PairPlan& seg)
{
    const int32_t op0 = (int32_t)all.ops.size(), lay0 = (int32_t)all.layouts.size();
    const int32_t g0 = (int32_t)(all.gates.size() / 64);
    if (all.layouts.size() + seg.layouts.size() > 65535) return false;
    for (PairPass P : seg.passes) {
        P.op_begin += op0;
        P.op_end += op0;
        P.load_layout += lay0;
        P.store_layout += lay0;
        P.gate_begin += g0;
        all.passes.push_back(P);
    }
    for (PairOp o : seg.ops) {
        if (o.kind == PO_BLOCK) o.gate += (uint32_t)g0;
        else if (o.kind == PO_RELAYOUT) {
            o.layout = (uint16_t)(o.layout + lay0);
            o.src = (uint16_t)(o.src + lay0);
        }
        all.ops.push_back(o);
    }
    all.layouts.insert(all.layouts.end(), seg.layouts.begin(), seg.layouts.end());
    all.gates.insert(all.gates.end(), seg.gates.begin(), seg.gates.end());
    all.stage_bytes = std::max(all.stage_bytes, seg.stage_bytes);
    all.n_blocks += seg.n_blocks;
    return true;
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Groups each pass's ops into register stages for k_adj_stages (passes of AT_M local
// qubits): ops are taken in order while their dense or CX targets fit 3 register
// positions; the stage's other 7 local positions are the thread-index bits.
void build_stages(std::vector<AdjTilePass>& tpasses, const std::vector<AdjTileOp>& tops,
                  std::vector<AdjStage>& stages, std::vector<AdjStageOp>& sops)
{
    for (AdjTilePass& P : tpasses) {
        P.stage_begin = (int32_t)stages.size();
        int32_t o = P.op_begin;
        while (o < P.op_end) {
            std::vector<int> rp;
            int32_t e = o;
            for (; e < P.op_end; e++) {
                const AdjTileOp& t = tops[e];
                if (t.kind != AT_C1 && t.kind != AT_CX) continue;
                if (std::find(rp.begin(), rp.end(), (int)t.p) != rp.end()) continue;
                if (rp.size() == 3) break;
                rp.push_back(t.p);
            }
            for (int q = 0; rp.size() < 3; q++)
                if (std::find(rp.begin(), rp.end(), q) == rp.end()) rp.push_back(q);
            AdjStage S;
            std::memset(&S, 0, sizeof(S));
            int nt = 0;
            for (int j = 0; j < 3; j++) S.rp[j] = (uint8_t)rp[j];
            for (int q = 0; q < AT_M; q++)
                if (std::find(rp.begin(), rp.end(), q) == rp.end()) S.tp[nt++] = (uint8_t)q;
            auto where = [&](int q, uint8_t& loc, uint8_t& bit) {
                for (int j = 0; j < 3; j++)
                    if (S.rp[j] == q) { loc = AS_LOC_REG; bit = (uint8_t)j; return; }
                for (int b = 0; b < 7; b++)
                    if (S.tp[b] == q) { loc = AS_LOC_THREAD; bit = (uint8_t)b; return; }
            };
            S.op_begin = (int32_t)sops.size();
            for (int32_t k = o; k < e; k++) {
                const AdjTileOp& t = tops[k];
                AdjStageOp so;
                std::memset(&so, 0, sizeof(so));
                so.kind = t.kind;
                so.nd = t.nd;
                so.lslot = t.lslot;
                std::memcpy(so.m, t.m, sizeof(so.m));
                std::memcpy(so.dm, t.dm, sizeof(so.dm));
                uint8_t loc = AS_LOC_REG;
                if (t.kind == AT_C1) {
                    where(t.p, loc, so.j);
                } else if (t.kind == AT_CX) {
                    where(t.p, loc, so.j);
                    if (t.flags & 2) { so.loc = AS_LOC_TILE; so.c = t.tile_bit; }
                    else where(t.c, so.loc, so.c);
                } else {
                    if (t.flags & 1) { so.loc = AS_LOC_TILE; so.j = t.tile_bit; }
                    else where(t.p, so.loc, so.j);
                }
                sops.push_back(so);
            }
            S.op_end = (int32_t)sops.size();
            stages.push_back(S);
            o = e;
        }
        P.stage_end = (int32_t)stages.size();
    }
}

}  // namespace
}  // namespace svb

extern "C" svb_status svb_adjoint(svb_sim* s, const svb_gate* gates, const svb_param_binding* bindings,
                                  size_t n_gates, uint32_t n_params, const svb_pauli_term* terms,
                                  size_t n_terms, double* energy, double* grad)
{
    if (!s) { set_error("svb_adjoint: NULL handle"); return SVB_ERR_INVALID; }
    if ((n_gates && (!gates || !bindings)) || (n_terms && !terms) || (n_params && !grad)) {
        set_error("svb_adjoint: NULL argument");
        return SVB_ERR_INVALID;
    }
    if (s->precision != SVB_FP64) {
        set_error("svb_adjoint: the adjoint runs on FP64 states");
        return SVB_ERR_UNSUPPORTED;
    }
    if (n_terms > 4096) { set_error("svb_adjoint: at most 4096 terms"); return SVB_ERR_INVALID; }
    for (size_t t = 0; t < n_terms; t++)
        if ((terms[t].x_mask | terms[t].z_mask) >> s->n) {
            set_error("svb_adjoint: observable acts on a qubit >= n_qubits");
            return SVB_ERR_INVALID;
        }
    for (size_t i = 0; i < n_gates; i++)
        for (int f = 0; f < 3; f++)
            if (bindings[i].idx[f] >= (int32_t)n_params) {
                set_error("svb_adjoint: binding of gate " + std::to_string(i) + " names parameter " +
                          std::to_string(bindings[i].idx[f]) + " >= n_params");
                return SVB_ERR_INVALID;
            }
    // validates and lowers the gates; the handle's own circuit and plan stay as they are
    std::vector<EOp> eops;
    svb_status rc = validate_and_lower(s, gates, n_gates, eops, nullptr);
    if (rc != SVB_OK) return rc;
    const int n = (int)s->n;
    const uint64_t dim = 1ull << n;
    const size_t K = eops.size();

    // derivative slots
    struct Slot { size_t k; int i; };
    std::vector<Slot> slots;
    std::vector<int> first_slot(K, -1), n_slot(K, 0);
    for (size_t k = 0; k < K; k++) {
        const EOp& e = eops[k];
        const svb_param_binding& b = bindings[e.gate];
        for (int i = 0; i < 3; i++) {
            bool used = false;
            for (int f = 0; f < 3; f++)
                if (b.idx[f] >= 0 && e.jac[i][f] != 0.0) used = true;
            if (!used) continue;
            if (e.kind == EK_R || e.kind == EK_CONST) {
                set_error("svb_adjoint: gate " + std::to_string(e.gate) + " has a bound angle on a "
                          "non-differentiable op (R is not unitary)");
                return SVB_ERR_UNSUPPORTED;
            }
            if (first_slot[k] < 0) first_slot[k] = (int)slots.size();
            slots.push_back({k, i});
            n_slot[k]++;
        }
        EOp inv;
        if (!inverse_op(e, inv)) {
            set_error("svb_adjoint: gate " + std::to_string(e.gate) + " is not unitary (R or SRN)");
            return SVB_ERR_UNSUPPORTED;
        }
    }

    cudaError_t err = cudaSuccess;
    AdjScratch& A = s->adj;
    const size_t sbytes = dim * sizeof(double2);
    // buffers live in the handle and are reused by later calls; large states give them
    // back at the end of the call
    const bool keep = sbytes <= (size_t(256) << 20);
    auto fail = [&](cudaError_t e, const char* what) {
        if (!keep) free_adjoint_scratch(A);
        set_error(std::string("svb_adjoint: ") + what + ": " + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? SVB_ERR_OOM : SVB_ERR_CUDA;
    };
    const size_t nslots = std::max<size_t>(slots.size(), 1);
    const int TM = std::min(n, AT_M);                 // local qubits of a reverse-sweep tile
    const uint64_t tiles = 1ull << (n - TM);
    const size_t eoff = slots.size() * tiles;         // the energy's partials follow the slots'
    if ((err = grow(A.lam, sbytes)) != cudaSuccess) return fail(err, "cudaMalloc(lambda)");
    if ((err = grow(A.partial, (nslots * tiles + ADJ_BLOCKS) * sizeof(double))) != cudaSuccess)
        return fail(err, "cudaMalloc(partials)");
    if ((err = grow(A.results, (nslots + 1) * sizeof(double))) != cudaSuccess)
        return fail(err, "cudaMalloc(results)");
    if ((err = grow(A.terms, std::max<size_t>(1, n_terms) * sizeof(svb_pauli_term))) != cudaSuccess)
        return fail(err, "cudaMalloc(terms)");
    if ((err = grow(A.final_state, sbytes)) != cudaSuccess) return fail(err, "cudaMalloc(final state)");
    double2* lam = static_cast<double2*>(A.lam.p);
    double* partial = static_cast<double*>(A.partial.p);
    double* results = static_cast<double*>(A.results.p);
    svb_pauli_term* dterms = static_cast<svb_pauli_term*>(A.terms.p);
    if (n_terms && (err = cudaMemcpy(dterms, terms, n_terms * sizeof(svb_pauli_term),
                                     cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(err, "terms upload");

    // checkpoints: up to 4 evenly spaced, if they fit in a quarter of free memory (the
    // device is asked once per state size; later calls reuse the answer)
    std::vector<void*> ckpts;
    std::vector<size_t> ckpt_at;   // op index where checkpoint c was taken (state before op)
    if (A.ck_count < 0 || A.ck_bytes != sbytes) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        size_t held = 0;
        for (const GrowBuf& b : A.ckpts) held += b.cap >= sbytes ? sbytes : 0;
        A.ck_count = (int)std::min<size_t>(4, (free_b + held) / 4 / sbytes);
        A.ck_bytes = sbytes;
    }
    int n_ck = A.ck_count;
    if (K < 64) n_ck = 0;
    if ((int)A.ckpts.size() < n_ck) A.ckpts.resize(n_ck);
    for (int c = 0; c < n_ck; c++) {
        if ((err = grow(A.ckpts[c], sbytes)) != cudaSuccess) { (void)cudaGetLastError(); break; }
        ckpts.push_back(A.ckpts[c].p);
        ckpt_at.push_back(K * (size_t)(c + 1) / (size_t)(n_ck + 1));
    }

    // the forward segments' pair plans, all built before anything is queued, so that the
    // GPU runs the whole forward pass without waiting for the host
    PairPlan fwd;
    std::vector<size_t> seg_pass_end;
    bool fwd_pairs = n >= PR_TILE_BITS;
    {
        size_t b0 = 0;
        for (size_t c = 0; fwd_pairs && c <= ckpts.size(); c++) {
            const size_t e0 = c < ckpts.size() ? ckpt_at[c] : K;
            std::vector<EOp> seg(eops.begin() + b0, eops.begin() + e0);
            PairPlan P;
            // the program-order cut only: this planning is on every gradient's path
            if (!plan_pairs(seg, n, P, nullptr, false) || !append_pair_plan(fwd, P)) fwd_pairs = false;
            seg_pass_end.push_back(fwd.passes.size());
            b0 = e0;
        }
    }
    // pinned staging: [forward plan | reverse plan | results]
    const size_t fwd_bytes = align_up(fwd.passes.size() * sizeof(PairPass)) +
                             align_up(fwd.ops.size() * sizeof(PairOp)) +
                             align_up(fwd.layouts.size() * sizeof(DevStage)) +
                             align_up(fwd.gates.size() * sizeof(double));
    // forward, segment by segment, checkpoint copies between them
    if ((err = launch_reset<double>(s->state, n, nullptr)) != cudaSuccess) return fail(err, "reset");
    if (fwd_pairs && !fwd.passes.empty()) {
        if ((err = grow_host(A.host_stage, fwd_bytes)) != cudaSuccess) return fail(err, "cudaMallocHost(stage)");
        if ((err = grow(A.pair_passes, fwd.passes.size() * sizeof(PairPass))) != cudaSuccess ||
            (err = grow(A.pair_ops, std::max<size_t>(1, fwd.ops.size()) * sizeof(PairOp))) != cudaSuccess ||
            (err = grow(A.pair_layouts, std::max<size_t>(1, fwd.layouts.size()) * sizeof(DevStage))) != cudaSuccess ||
            (err = grow(A.pair_gates, std::max<size_t>(2, fwd.gates.size()) * sizeof(double))) != cudaSuccess)
            return fail(err, "cudaMalloc(forward plan)");
        char* hs = static_cast<char*>(A.host_stage.p);
        size_t off = 0;
        auto stage = [&](const void* src, size_t bytes, void* dst) {
            if (bytes == 0 || err != cudaSuccess) return;
            std::memcpy(hs + off, src, bytes);
            err = cudaMemcpyAsync(dst, hs + off, bytes, cudaMemcpyHostToDevice, nullptr);
            off += align_up(bytes);
        };
        stage(fwd.passes.data(), fwd.passes.size() * sizeof(PairPass), A.pair_passes.p);
        stage(fwd.ops.data(), fwd.ops.size() * sizeof(PairOp), A.pair_ops.p);
        stage(fwd.layouts.data(), fwd.layouts.size() * sizeof(DevStage), A.pair_layouts.p);
        stage(fwd.gates.data(), fwd.gates.size() * sizeof(double), A.pair_gates.p);
        if (err != cudaSuccess) return fail(err, "forward plan upload");
        DevPairBuffers pb;
        pb.passes = static_cast<PairPass*>(A.pair_passes.p);
        pb.ops = static_cast<PairOp*>(A.pair_ops.p);
        pb.layouts = static_cast<DevStage*>(A.pair_layouts.p);
        pb.gates = static_cast<double*>(A.pair_gates.p);
        pb.stage_bytes = fwd.stage_bytes;
        size_t p0 = 0;
        for (size_t c = 0; c <= ckpts.size(); c++) {
            for (size_t p = p0; p < seg_pass_end[c] && err == cudaSuccess; p++)
                err = launch_pair_pass(s->state, n, (int)p, pb, nullptr);
            if (err != cudaSuccess) return fail(err, "forward pass");
            p0 = seg_pass_end[c];
            if (c < ckpts.size() &&
                (err = cudaMemcpyAsync(ckpts[c], s->state, sbytes, cudaMemcpyDeviceToDevice)) != cudaSuccess)
                return fail(err, "checkpoint");
        }
    } else if (fwd_pairs) {
        for (void* ck : ckpts)
            if ((err = cudaMemcpyAsync(ck, s->state, sbytes, cudaMemcpyDeviceToDevice)) != cudaSuccess)
                return fail(err, "checkpoint");
    } else {
        size_t begin = 0;
        for (size_t c = 0; c <= ckpts.size(); c++) {
            const size_t end = c < ckpts.size() ? ckpt_at[c] : K;
            std::vector<EOp> seg(eops.begin() + begin, eops.begin() + end);
            svb_status r2 = run_eops_fp64(n, s->state, seg, nullptr, A);
            if (r2 != SVB_OK) {
                if (!keep) free_adjoint_scratch(A);
                return r2;
            }
            if (c < ckpts.size() &&
                (err = cudaMemcpyAsync(ckpts[c], s->state, sbytes, cudaMemcpyDeviceToDevice)) != cudaSuccess)
                return fail(err, "checkpoint");
            begin = end;
        }
    }
    // psi(p), handed back in the handle at the end
    if ((err = cudaMemcpyAsync(A.final_state.p, s->state, sbytes, cudaMemcpyDeviceToDevice)) != cudaSuccess)
        return fail(err, "final state copy");
    // lambda = H psi, energy = Re <psi|lambda>
    const unsigned g = adj_grid(dim);
    if (n_terms)
        k_pauli_apply<<<g, 256, n_terms * sizeof(svb_pauli_term)>>>(
            static_cast<const double2*>(s->state), lam, dim, dterms, (int)n_terms);
    else
        err = cudaMemset(lam, 0, sbytes);
    k_inner_re<<<ADJ_BLOCKS, 256>>>(static_cast<const double2*>(s->state), lam, dim, partial + eoff);
    k_reduce_rows<<<1, 32>>>(partial + eoff, ADJ_BLOCKS, ADJ_BLOCKS, 1, results + slots.size());
    if ((err = cudaGetLastError()) != cudaSuccess) return fail(err, "energy");

    // reverse sweep, tiled: the inverse ops in reverse order, cut into passes of TM local
    // qubits; a pass never spans a checkpoint, after which psi is reloaded
    std::vector<AdjTilePass> tpasses;
    std::vector<AdjTileOp> tops;
    std::vector<int32_t> tslots;                      // per pass: global slot of each local slot
    int max_lslots = 0;
    struct Seg { size_t pass_end; int ck; };          // reload checkpoint ck after the passes
    std::vector<Seg> segs;
    {
        const int G = std::min(4, TM);
        size_t kk_hi = K;
        for (int ck = (int)ckpts.size() - 1;; ck--) {
            const size_t kk_lo = ck >= 0 ? ckpt_at[ck] : 0;
            std::vector<EOp> rev;
            std::vector<size_t> orig;
            for (size_t kk = kk_hi; kk-- > kk_lo;) {
                EOp inv;
                inverse_op(eops[kk], inv);
                if (n_slot[kk] > 0 && inv.form == F_DIAG) {
                    // a differentiated op needs its pairs local: as a general 2x2
                    const double d0r = inv.m[0], d0i = inv.m[1], d1r = inv.m[2], d1i = inv.m[3];
                    inv.form = F_C1;
                    const double c1[8] = {d0r, d0i, 0, 0, 0, 0, d1r, d1i};
                    std::memcpy(inv.m, c1, sizeof(c1));
                }
                rev.push_back(inv);
                orig.push_back(kk);
            }
            select_passes(rev, n, TM, G, [&](uint64_t L, const std::vector<int>& idx) {
                AdjTilePass P;
                std::memset(&P, 0, sizeof(P));
                int pos[64], tbit[64];
                uint8_t local_q[AT_M];
                int nl = 0, nn = 0;
                for (int q = 0; q < 64; q++) pos[q] = tbit[q] = -1;
                for (int q = 0; q < n; q++) {
                    if ((L >> q) & 1ull) { pos[q] = nl; local_q[nl++] = (uint8_t)q; }
                    else { tbit[q] = nn; P.nonlocal_q[nn++] = (uint8_t)q; }
                }
                P.n_nonlocal = nn;
                for (int j = 0; j < 64; j++)
                    for (int b2 = 0; b2 < 6 && b2 < TM; b2++)
                        if ((j >> b2) & 1) P.g_lo[j] |= 1ull << local_q[b2];
                for (int j = 0; j < 32; j++)
                    for (int b2 = 0; b2 < 5 && 6 + b2 < TM; b2++)
                        if ((j >> b2) & 1) P.g_hi[j] |= 1ull << local_q[6 + b2];
                P.op_begin = (int32_t)tops.size();
                P.lslot_begin = (int32_t)tslots.size();
                for (int i : idx) {
                    const EOp& e = rev[i];
                    const size_t kk = orig[i];
                    AdjTileOp t;
                    std::memset(&t, 0, sizeof(t));
                    if (e.form == F_CX) {
                        t.kind = AT_CX;
                        t.p = (uint8_t)pos[e.q];
                        if (pos[e.c] >= 0) t.c = (uint8_t)pos[e.c];
                        else { t.flags |= 2; t.tile_bit = (uint8_t)tbit[e.c]; }
                    } else if (e.form == F_DIAG) {
                        t.kind = AT_DIAG;
                        std::memcpy(t.m, e.m, sizeof(t.m));
                        if (pos[e.q] >= 0) t.p = (uint8_t)pos[e.q];
                        else { t.flags |= 1; t.tile_bit = (uint8_t)tbit[e.q]; }
                    } else {
                        if ((int)(tslots.size() - P.lslot_begin) + n_slot[kk] > AT_MAX_LSLOTS) {
                            // the warps' sums would not fit: the rest of the ops in a second
                            // pass over the same layout
                            P.op_end = (int32_t)tops.size();
                            P.n_lslots = (int32_t)tslots.size() - P.lslot_begin;
                            max_lslots = std::max(max_lslots, P.n_lslots);
                            tpasses.push_back(P);
                            P.op_begin = (int32_t)tops.size();
                            P.lslot_begin = (int32_t)tslots.size();
                        }
                        t.kind = AT_C1;
                        t.p = (uint8_t)pos[e.q];
                        std::memcpy(t.m, e.m, sizeof(t.m));
                        t.nd = (uint8_t)n_slot[kk];
                        t.lslot = (int32_t)tslots.size() - P.lslot_begin;
                        for (int d = 0; d < n_slot[kk]; d++) tslots.push_back(first_slot[kk] + d);
                        for (int d = 0; d < n_slot[kk]; d++) deriv_matrix(eops[kk], slots[first_slot[kk] + d].i, t.dm[d]);
                    }
                    tops.push_back(t);
                }
                P.op_end = (int32_t)tops.size();
                P.n_lslots = (int32_t)tslots.size() - P.lslot_begin;
                max_lslots = std::max(max_lslots, P.n_lslots);
                tpasses.push_back(P);
                return std::vector<int>{};
            });
            segs.push_back({tpasses.size(), ck});
            kk_hi = kk_lo;
            if (ck < 0) break;
        }
    }
    // register stages of the reverse passes (tiles of AT_M qubits)
    const bool staged_rev = TM == AT_M;
    std::vector<AdjStage> stages;
    std::vector<AdjStageOp> sops;
    if (staged_rev) build_stages(tpasses, tops, stages, sops);
    if ((err = grow(A.rev_stages, std::max<size_t>(1, stages.size()) * sizeof(AdjStage))) != cudaSuccess ||
        (err = grow(A.rev_sops, std::max<size_t>(1, sops.size()) * sizeof(AdjStageOp))) != cudaSuccess)
        return fail(err, "cudaMalloc(reverse plan)");
    if ((err = grow(A.rev_passes, std::max<size_t>(1, tpasses.size()) * sizeof(AdjTilePass))) != cudaSuccess)
        return fail(err, "cudaMalloc(reverse plan)");
    if ((err = grow(A.rev_ops, std::max<size_t>(1, tops.size()) * sizeof(AdjTileOp))) != cudaSuccess)
        return fail(err, "cudaMalloc(reverse plan)");
    if ((err = grow(A.rev_slots, std::max<size_t>(1, tslots.size()) * sizeof(int32_t))) != cudaSuccess)
        return fail(err, "cudaMalloc(reverse plan)");
    // the reverse plan goes through the pinned stage behind the forward plan (the forward
    // plan's copies may still be in flight, so its part of the stage is left alone); the
    // results come back into the stage's tail
    const size_t rev_bytes = align_up(tslots.size() * sizeof(int32_t)) +
                             align_up(tpasses.size() * sizeof(AdjTilePass)) +
                             (staged_rev ? align_up(stages.size() * sizeof(AdjStage)) +
                                               align_up(sops.size() * sizeof(AdjStageOp))
                                         : align_up(tops.size() * sizeof(AdjTileOp)));
    const size_t res_bytes = (slots.size() + 1) * sizeof(double);
    if (A.host_stage.cap < fwd_bytes + rev_bytes + res_bytes) {
        // growing would free memory the forward copies may still read: wait for them
        if ((err = cudaStreamSynchronize(nullptr)) != cudaSuccess) return fail(err, "forward pass");
        if ((err = grow_host(A.host_stage, fwd_bytes + rev_bytes + res_bytes)) != cudaSuccess)
            return fail(err, "cudaMallocHost(stage)");
    }
    {
        char* hs = static_cast<char*>(A.host_stage.p);
        size_t off = fwd_bytes;
        auto stage = [&](const void* src, size_t bytes, void* dst) {
            if (bytes == 0 || err != cudaSuccess) return;
            std::memcpy(hs + off, src, bytes);
            err = cudaMemcpyAsync(dst, hs + off, bytes, cudaMemcpyHostToDevice, nullptr);
            off += align_up(bytes);
        };
        stage(tslots.data(), tslots.size() * sizeof(int32_t), A.rev_slots.p);
        stage(tpasses.data(), tpasses.size() * sizeof(AdjTilePass), A.rev_passes.p);
        if (staged_rev) {
            stage(stages.data(), stages.size() * sizeof(AdjStage), A.rev_stages.p);
            stage(sops.data(), sops.size() * sizeof(AdjStageOp), A.rev_sops.p);
        } else {
            stage(tops.data(), tops.size() * sizeof(AdjTileOp), A.rev_ops.p);
        }
        if (err != cudaSuccess) return fail(err, "reverse plan upload");
    }
    double2* psi = static_cast<double2*>(s->state);
    if (staged_rev) {
        static int ctas_per_sm = 0, sms = 0;
        const size_t smem = (2 * sizeof(double2) << AT_M) + AT_MAX_LSLOTS * (AS_THREADS / 32) * sizeof(double);
        if (ctas_per_sm == 0) {
            if ((err = cudaFuncSetAttribute(k_adj_stages, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                    cudaSuccess ||
                (err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas_per_sm, k_adj_stages, AS_THREADS, smem)) !=
                    cudaSuccess ||
                (err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device)) != cudaSuccess)
                return fail(err, "reverse kernel setup");
            ctas_per_sm = std::max(ctas_per_sm, 1);
        }
        const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)ctas_per_sm * sms);
        const size_t dyn = (2 * sizeof(double2) << AT_M) + (size_t)max_lslots * (AS_THREADS / 32) * sizeof(double);
        size_t pi = 0;
        for (const Seg& sg : segs) {
            for (; pi < sg.pass_end; pi++)
                k_adj_stages<<<grid, AS_THREADS, dyn>>>(psi, lam, static_cast<const AdjTilePass*>(A.rev_passes.p),
                                                        (int)pi, static_cast<const AdjStage*>(A.rev_stages.p),
                                                        static_cast<const AdjStageOp*>(A.rev_sops.p),
                                                        static_cast<const int32_t*>(A.rev_slots.p), tiles, partial);
            if ((err = cudaGetLastError()) != cudaSuccess) return fail(err, "reverse pass");
            if (sg.ck >= 0 &&
                (err = cudaMemcpyAsync(psi, ckpts[sg.ck], sbytes, cudaMemcpyDeviceToDevice)) != cudaSuccess)
                return fail(err, "checkpoint reload");
        }
    } else {
        static int ctas_per_sm = 0, sms = 0;
        // the tiles and the warps' sums of up to AT_MAX_LSLOTS slots of a pass
        const size_t smem = (2 * sizeof(double2) << AT_M) + AT_MAX_LSLOTS * (AT_THREADS / 32) * sizeof(double);
        if (ctas_per_sm == 0) {
            if ((err = cudaFuncSetAttribute(k_adj_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                    cudaSuccess ||
                (err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas_per_sm, k_adj_tiles, AT_THREADS, smem)) !=
                    cudaSuccess ||
                (err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device)) != cudaSuccess)
                return fail(err, "reverse kernel setup");
            ctas_per_sm = std::max(ctas_per_sm, 1);
        }
        const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)ctas_per_sm * sms);
        const size_t dyn = (2 * sizeof(double2) << TM) + (size_t)max_lslots * (AT_THREADS / 32) * sizeof(double);
        size_t pi = 0;
        for (const Seg& sg : segs) {
            for (; pi < sg.pass_end; pi++)
                k_adj_tiles<<<grid, AT_THREADS, dyn>>>(psi, lam, static_cast<const AdjTilePass*>(A.rev_passes.p),
                                                       (int)pi, static_cast<const AdjTileOp*>(A.rev_ops.p),
                                                       static_cast<const int32_t*>(A.rev_slots.p), TM, tiles,
                                                       partial);
            if ((err = cudaGetLastError()) != cudaSuccess) return fail(err, "reverse pass");
            // psi is now the state before op ckpt_at[ck]: reload the stored copy
            if (sg.ck >= 0 &&
                (err = cudaMemcpyAsync(psi, ckpts[sg.ck], sbytes, cudaMemcpyDeviceToDevice)) != cudaSuccess)
                return fail(err, "checkpoint reload");
        }
    }
    if (!slots.empty())
        k_reduce_rows<<<(unsigned)((slots.size() * 32 + 255) / 256), 256>>>(partial, (int)tiles, tiles,
                                                                          (int)slots.size(), results);
    // results to the stage's tail, psi(p) back into the handle, then one wait
    double* host = reinterpret_cast<double*>(static_cast<char*>(A.host_stage.p) + fwd_bytes + rev_bytes);
    if ((err = cudaMemcpyAsync(host, results, res_bytes, cudaMemcpyDeviceToHost, nullptr)) != cudaSuccess)
        return fail(err, "results download");
    if ((err = cudaMemcpyAsync(s->state, A.final_state.p, sbytes, cudaMemcpyDeviceToDevice, nullptr)) != cudaSuccess)
        return fail(err, "final state restore");
    if ((err = cudaStreamSynchronize(nullptr)) != cudaSuccess) return fail(err, "adjoint");
    if (energy) *energy = host[slots.size()];
    for (uint32_t p = 0; p < n_params; p++) grad[p] = 0.0;
    for (size_t r = 0; r < slots.size(); r++) {
        const EOp& e = eops[slots[r].k];
        const svb_param_binding& b = bindings[e.gate];
        for (int f = 0; f < 3; f++)
            if (b.idx[f] >= 0 && e.jac[slots[r].i][f] != 0.0)
                grad[b.idx[f]] += 2.0 * host[r] * e.jac[slots[r].i][f] * b.coef[f];
    }
    if (!keep) free_adjoint_scratch(A);
    return SVB_OK;
}

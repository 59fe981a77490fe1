// The per-gate engine: one launch per elementary op, one streaming sweep over the
// affected amplitudes with 128-bit complex<double> (64-bit complex<float>) loads — the
// work of one OP_HEAD ... OP_TAIL block of the reference (svsim/src/svsim_nvgpu_sin.cuh
// :640-651) without its grid barrier.
//
// This file is compiled with -fmad=false (build.py): every product and sum of the gate
// expressions in gate_math.cuh is rounded on its own, in the order written, which is
// how the reference's CPU backends evaluate the same expressions
// (svsim_cpu_sin.hpp:602-1165; x86-64 without FMA contraction).  With the host-side
// coefficients of lower.cpp this makes the per-gate engine's FP64 states bit-identical
// to the reference CPU backend's for the same circuit.  The sweeps are HBM-bound, so
// the unfused multiply-adds cost nothing measurable.
#include "gate_math.cuh"

namespace svb {

// Each thread takes PG_UNROLL items per iteration (items u * stride apart, so a warp's
// accesses stay coalesced) and issues all their loads before any arithmetic: more bytes
// in flight per thread than one pair at a time.
constexpr int PG_UNROLL = 4;

template <typename T>
__global__ void __launch_bounds__(256)
k_eop_pairs(typename VecOf<T>::type* __restrict__ sv, uint64_t half, int q, int form,
            Coef<T> c)
{
    using V = typename VecOf<T>::type;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t qd = 1ull << q;
    const bool diag = form_is_diag(form);
    const bool both = !diag || form == F_DIAG;     // diagonal forms other than D leave |0> alone
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < half;
         i0 += PG_UNROLL * stride) {
        V a0[PG_UNROLL], a1[PG_UNROLL];
        uint64_t p0[PG_UNROLL];
#pragma unroll
        for (int u = 0; u < PG_UNROLL; u++) {
            const uint64_t i = i0 + (uint64_t)u * stride;
            p0[u] = insert_zero(i < half ? i : 0, q);
            if (i < half) {
                a1[u] = sv[p0[u] | qd];
                if (both) a0[u] = sv[p0[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < PG_UNROLL; u++) {
            if (i0 + (uint64_t)u * stride >= half) continue;
            if (diag) {
                diag_one<T>(form, c, a1[u]);
                if (form == F_DIAG) diag_zero<T>(form, c, a0[u]);
            } else {
                dense_pair<T>(form, c, a0[u], a1[u]);
            }
            sv[p0[u] | qd] = a1[u];
            if (both) sv[p0[u]] = a0[u];
        }
    }
}

// CX_GATE :779-811 — only the quarter of the state with ctrl = 1 moves.
template <typename T>
__global__ void __launch_bounds__(256)
k_cx(typename VecOf<T>::type* __restrict__ sv, uint64_t quarter, int c, int t)
{
    using V = typename VecOf<T>::type;
    const int lo = c < t ? c : t, hi = c < t ? t : c;
    const uint64_t cd = 1ull << c, td = 1ull << t;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < quarter;
         i0 += PG_UNROLL * stride) {
        V a0[PG_UNROLL], a1[PG_UNROLL];
        uint64_t b[PG_UNROLL];
#pragma unroll
        for (int u = 0; u < PG_UNROLL; u++) {
            const uint64_t i = i0 + (uint64_t)u * stride;
            b[u] = insert_zero(insert_zero(i < quarter ? i : 0, lo), hi) | cd;
            if (i < quarter) {
                a0[u] = sv[b[u]];
                a1[u] = sv[b[u] | td];
            }
        }
#pragma unroll
        for (int u = 0; u < PG_UNROLL; u++) {
            if (i0 + (uint64_t)u * stride >= quarter) continue;
            sv[b[u]] = a1[u];
            sv[b[u] | td] = a0[u];
        }
    }
}

static unsigned grid_for(uint64_t items, int threads)
{
    // enough CTAs to fill 148 SMs several times over, grid-stride beyond that
    const uint64_t need = (items + (uint64_t)threads * PG_UNROLL - 1) / ((uint64_t)threads * PG_UNROLL);
    const uint64_t cap = 148ull * 8;
    return (unsigned)(need < cap ? (need > 0 ? need : 1) : cap);
}

template <typename T>
cudaError_t launch_eop(void* state, int n, const EOp& op, cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    V* sv = static_cast<V*>(state);
    if (op.form == F_CX) {
        if (n < 2) return cudaErrorInvalidValue;
        const uint64_t quarter = 1ull << (n - 2);
        k_cx<T><<<grid_for(quarter, 256), 256, 0, s>>>(sv, quarter, (int)op.c, (int)op.q);
    } else {
        const uint64_t half = 1ull << (n - 1);
        Coef<T> c;
        for (int i = 0; i < 8; i++) c.m[i] = static_cast<T>(op.m[i]);
        k_eop_pairs<T><<<grid_for(half, 256), 256, 0, s>>>(sv, half, (int)op.q, (int)op.form, c);
    }
    return cudaGetLastError();
}

template cudaError_t launch_eop<double>(void*, int, const EOp&, cudaStream_t);
template cudaError_t launch_eop<float>(void*, int, const EOp&, cudaStream_t);

}  // namespace svb

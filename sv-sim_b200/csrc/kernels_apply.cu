// Gate-application kernels for sm_100a.
//
//  * k_eop_pairs / k_cx : the per-gate engine.  One launch per elementary op, one
//    streaming sweep over the affected amplitudes with 128-bit complex<double> (64-bit
//    complex<float>) loads — the work of one OP_HEAD ... OP_TAIL block of the
//    reference (svsim/src/svsim_nvgpu_sin.cuh:640-651) without its grid barrier.
//  * k_staged : the staged engine.  One launch per pass of the planner; every CTA owns
//    one tile of 2^M amplitudes (the M local qubits of the pass), keeps it in registers
//    (16 amplitudes per thread) and applies all ops of the pass to it, re-distributing
//    the tile through XOR-swizzled shared memory whenever the next ops target qubits
//    that are not in registers.  Each pass reads and writes the state exactly once.
#include <cstdio>

#include "staged_core.cuh"

namespace svb {

// ---------------------------------------------------------------------------------
// per-gate engine
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
k_eop_pairs(typename VecOf<T>::type* __restrict__ sv, uint64_t half, int q, int form,
            Coef<T> c)
{
    using V = typename VecOf<T>::type;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t qd = 1ull << q;
    const bool diag = form_is_diag(form);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += stride) {
        const uint64_t p0 = insert_zero(i, q);
        const uint64_t p1 = p0 | qd;
        if (diag) {
            V a1 = sv[p1];
            diag_one<T>(form, c, a1);
            sv[p1] = a1;
            if (form == F_DIAG) {
                V a0 = sv[p0];
                diag_zero<T>(form, c, a0);
                sv[p0] = a0;
            }
        } else {
            V a0 = sv[p0], a1 = sv[p1];
            dense_pair<T>(form, c, a0, a1);
            sv[p0] = a0;
            sv[p1] = a1;
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
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < quarter; i += stride) {
        const uint64_t b = insert_zero(insert_zero(i, lo), hi);
        const uint64_t p0 = b | cd, p1 = b | cd | td;
        const V a0 = sv[p0];
        const V a1 = sv[p1];
        sv[p0] = a1;
        sv[p1] = a0;
    }
}

static unsigned grid_for(uint64_t items, int threads)
{
    // enough CTAs to fill 148 SMs several times over, grid-stride beyond that
    const uint64_t need = (items + threads - 1) / threads;
    const uint64_t cap = 148ull * 16;
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

// ---------------------------------------------------------------------------------
// staged engine
// ---------------------------------------------------------------------------------

template <typename V, int NR>
__device__ __forceinline__ void relayout(V* sm, V* v, const Slots& from, const Slots& to)
{
#pragma unroll
    for (int k = 0; k < NR; k++) sm[slot_of(from, k)] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NR; k++) v[k] = sm[slot_of(to, k)];
    __syncthreads();
}

template <typename T, int M>
__global__ void __launch_bounds__(1 << (M - RB), (M - RB) <= 8 ? 2 : 1)
k_staged(typename VecOf<T>::type* __restrict__ sv, const DevPass* __restrict__ passes,
         const DevStage* __restrict__ stages, const DevOp* __restrict__ ops, int pass_index)
{
    using V = typename VecOf<T>::type;
    constexpr int TBITS = M - RB;
    constexpr int NR = 1 << RB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);

    const int tid = threadIdx.x;
    const DevPass& P = passes[pass_index];
    const uint64_t tile = blockIdx.x;
    uint64_t base = 0;
    const int nnl = P.n_nonlocal;
    for (int j = 0; j < nnl; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];

    const int s0 = P.stage_begin, s1 = P.stage_end;
    V v[NR];
    {
        GOffs g;
        make_goffs<TBITS>(stages[s0], P, tid, g);
#pragma unroll
        for (int k = 0; k < NR; k++) v[k] = sv[base | goff_of(g, k)];
    }
    Slots cur;
    make_slots<T, TBITS>(stages[s0], tid, cur);
    const DevStage* last = &stages[s0];
    for (int s = s0; s < s1; s++) {
        const DevStage& S = stages[s];
        if (s != s0) {
            Slots nxt;
            make_slots<T, TBITS>(S, tid, nxt);
            relayout<V, NR>(sm, v, cur, nxt);
            cur = nxt;
            last = &S;
        }
        const int ob = S.op_begin, oe = S.op_end;
        for (int o = ob; o < oe; o++) apply_devop<T>(ops + o, v, tid, base);
    }
    if (P.final_relayout) {
        Slots nxt;
        make_slots<T, TBITS>(P.store_layout, tid, nxt);
        relayout<V, NR>(sm, v, cur, nxt);
        last = &P.store_layout;
    }
    {
        GOffs g;
        make_goffs<TBITS>(*last, P, tid, g);
#pragma unroll
        for (int k = 0; k < NR; k++) sv[base | goff_of(g, k)] = v[k];
    }
}

template <typename T, int M>
static cudaError_t launch_staged_m(void* state, int n, int pass_index, const DevPlanBuffers& b,
                                   cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    static bool attr_done[64] = {false};   // per device
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = (size_t(1) << M) * sizeof(V);
    if (dev < 64 && !attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_staged<T, M>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_done[dev] = true;
    }
    const uint64_t tiles = 1ull << (n - M);
    k_staged<T, M><<<(unsigned)tiles, 1 << (M - RB), smem, s>>>(
        static_cast<V*>(state), b.passes, b.stages, b.ops, pass_index);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_staged_pass(void* state, int n, int M, int pass_index,
                               const DevPlanBuffers& b, cudaStream_t s)
{
    if (n < M) return cudaErrorInvalidValue;
    switch (M) {
    case 10: return launch_staged_m<T, 10>(state, n, pass_index, b, s);
    case 11: return launch_staged_m<T, 11>(state, n, pass_index, b, s);
    case 12: return launch_staged_m<T, 12>(state, n, pass_index, b, s);
    case 13:
        if constexpr (sizeof(T) == 4) return launch_staged_m<T, 13>(state, n, pass_index, b, s);
        return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------------
// state utilities
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void k_reset(typename VecOf<T>::type* sv, uint64_t dim)
{
    using V = typename VecOf<T>::type;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
        V z;
        z.x = (i == 0) ? T(1) : T(0);
        z.y = T(0);
        sv[i] = z;
    }
}

template <typename T>
cudaError_t launch_reset(void* state, int n, cudaStream_t s)
{
    const uint64_t dim = 1ull << n;
    k_reset<T><<<grid_for(dim, 256), 256, 0, s>>>(static_cast<typename VecOf<T>::type*>(state), dim);
    return cudaGetLastError();
}

template <typename T>
__global__ void k_soa_split(const typename VecOf<T>::type* __restrict__ sv, uint64_t count,
                            double* __restrict__ re, double* __restrict__ im)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const auto a = sv[i];
        if (re) re[i] = (double)a.x;
        if (im) im[i] = (double)a.y;
    }
}

template <typename T>
__global__ void k_soa_merge(typename VecOf<T>::type* __restrict__ sv, uint64_t count,
                            const double* __restrict__ re, const double* __restrict__ im)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        typename VecOf<T>::type a;
        a.x = (T)re[i];
        a.y = (T)im[i];
        sv[i] = a;
    }
}

template <typename T>
cudaError_t launch_soa_split(const void* state, uint64_t first, uint64_t count, double* re,
                             double* im, cudaStream_t s)
{
    const auto* sv = static_cast<const typename VecOf<T>::type*>(state) + first;
    k_soa_split<T><<<grid_for(count, 256), 256, 0, s>>>(sv, count, re, im);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_soa_merge(void* state, uint64_t first, uint64_t count, const double* re,
                             const double* im, cudaStream_t s)
{
    auto* sv = static_cast<typename VecOf<T>::type*>(state) + first;
    k_soa_merge<T><<<grid_for(count, 256), 256, 0, s>>>(sv, count, re, im);
    return cudaGetLastError();
}

#define SVB_INSTANTIATE(T)                                                                   \
    template cudaError_t launch_eop<T>(void*, int, const EOp&, cudaStream_t);                \
    template cudaError_t launch_staged_pass<T>(void*, int, int, int, const DevPlanBuffers&,   \
                                               cudaStream_t);                                \
    template cudaError_t launch_reset<T>(void*, int, cudaStream_t);                          \
    template cudaError_t launch_soa_split<T>(const void*, uint64_t, uint64_t, double*,       \
                                             double*, cudaStream_t);                         \
    template cudaError_t launch_soa_merge<T>(void*, uint64_t, uint64_t, const double*,       \
                                             const double*, cudaStream_t);
SVB_INSTANTIATE(double)
SVB_INSTANTIATE(float)

}  // namespace svb

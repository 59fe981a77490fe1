// Gate-application kernels for sm_100a.
//
//  * the per-gate engine (k_eop_pairs / k_cx) lives in kernels_pergate.cu, which is
//    compiled without FMA contraction.
//  * k_staged : the staged engine.  One launch per pass of the planner; every CTA owns
//    one tile of 2^M amplitudes (the M local qubits of the pass), keeps it in registers
//    (16 amplitudes per thread) and applies all ops of the pass to it, re-distributing
//    the tile through XOR-swizzled shared memory whenever the next ops target qubits
//    that are not in registers.  Each pass reads and writes the state exactly once.
#include <cstdio>
#include <cstdlib>

#include "staged_core.cuh"

namespace svb {

static unsigned grid_for(uint64_t items, int threads)
{
    // enough CTAs to fill 148 SMs several times over, grid-stride beyond that
    const uint64_t need = (items + (uint64_t)threads * 4 - 1) / ((uint64_t)threads * 4);
    const uint64_t cap = 148ull * 8;
    return (unsigned)(need < cap ? (need > 0 ? need : 1) : cap);
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

// In-place 2x2 complex update of one amplitude pair (C1 form) in inline PTX.  The
// four amplitude components are read-write operands, so every target variant of the
// dense-gate dispatch leaves its results in the registers it read them from.
__device__ __forceinline__ void c1_inplace(double2& a0, double2& a1, const Coef<double>& c,
                                           double ne0i, double ne1i, double ne2i, double ne3i)
{
    asm("{\n\t"
        ".reg .f64 r0, i0, r1;\n\t"
        "mul.rn.f64 r0, %4, %0;\n\t"
        "fma.rn.f64 r0, %12, %1, r0;\n\t"
        "fma.rn.f64 r0, %6, %2, r0;\n\t"
        "fma.rn.f64 r0, %13, %3, r0;\n\t"
        "mul.rn.f64 i0, %4, %1;\n\t"
        "fma.rn.f64 i0, %5, %0, i0;\n\t"
        "fma.rn.f64 i0, %6, %3, i0;\n\t"
        "fma.rn.f64 i0, %7, %2, i0;\n\t"
        "mul.rn.f64 r1, %8, %0;\n\t"
        "fma.rn.f64 r1, %14, %1, r1;\n\t"
        "fma.rn.f64 r1, %10, %2, r1;\n\t"
        "fma.rn.f64 r1, %15, %3, r1;\n\t"
        "mul.rn.f64 %3, %10, %3;\n\t"
        "fma.rn.f64 %3, %8, %1, %3;\n\t"
        "fma.rn.f64 %3, %9, %0, %3;\n\t"
        "fma.rn.f64 %3, %11, %2, %3;\n\t"
        "mov.f64 %0, r0;\n\t"
        "mov.f64 %1, i0;\n\t"
        "mov.f64 %2, r1;\n\t"
        "}"
        : "+d"(a0.x), "+d"(a0.y), "+d"(a1.x), "+d"(a1.y)
        : "d"(c.m[0]), "d"(c.m[1]), "d"(c.m[2]), "d"(c.m[3]), "d"(c.m[4]), "d"(c.m[5]),
          "d"(c.m[6]), "d"(c.m[7]), "d"(ne0i), "d"(ne1i), "d"(ne2i), "d"(ne3i));
}

template <typename T, typename V>
__device__ __forceinline__ void apply_devop_fast(const DevOp* __restrict__ opp, V* v, int tid,
                                                 uint64_t base)
{
    if constexpr (sizeof(T) == 8) {
        if (opp->form == F_C1) {
            const Coef<T> c = load_coef<T>(opp->m);
            const double ne0i = -c.m[1], ne1i = -c.m[3], ne2i = -c.m[5], ne3i = -c.m[7];
            for_pairs(opp->tgt, v, [&](V& a0, V& a1, int) { c1_inplace(a0, a1, c, ne0i, ne1i, ne2i, ne3i); });
            return;
        }
    }
    apply_devop<T>(opp, v, tid, base);
}

// Shared-memory layout of the staged kernel: the tile, then (VAR >= 1) the pass record,
// its stages and its ops, each region starting on a 16-byte boundary (the op
// coefficients are read and copied with 16-byte accesses).
constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
template <typename T, int M>
struct StagedSmem {
    static constexpr size_t tile = size_t(sizeof(typename VecOf<T>::type)) << M;
    static constexpr size_t pass_off = align16(tile);
    static constexpr size_t stages_off = align16(pass_off + sizeof(DevPass));
    static constexpr size_t ops_off = align16(stages_off + MAX_PASS_STAGES * sizeof(DevStage));
    static constexpr size_t total = align16(ops_off + MAX_PASS_OPS * sizeof(DevOp));
    static_assert(pass_off % 16 == 0 && stages_off % 16 == 0 && ops_off % 16 == 0, "alignment");
};

template <typename T, int M, int VAR>
__global__ void __launch_bounds__(1 << (M - RB), (M - RB) <= 8 ? 2 : 1)
k_staged(typename VecOf<T>::type* __restrict__ sv, const DevPass* __restrict__ passes,
         const DevStage* __restrict__ stages, const DevOp* __restrict__ ops, int pass_index,
         uint64_t tiles)
{
    using V = typename VecOf<T>::type;
    constexpr int TBITS = M - RB;
    constexpr int NR = 1 << RB;
    constexpr int NT = 1 << TBITS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);
    const int tid = threadIdx.x;

    // the pass description, its stages and its ops live in shared memory (VAR >= 1)
    const DevPass* Pp = passes + pass_index;
    const DevStage* S0 = stages;
    const DevOp* O0 = ops;
    int op_base = 0;
    if constexpr (VAR >= 1) {
        using L = StagedSmem<T, M>;
        DevPass* sP = reinterpret_cast<DevPass*>(smem_raw + L::pass_off);
        DevStage* sS = reinterpret_cast<DevStage*>(smem_raw + L::stages_off);
        DevOp* sO = reinterpret_cast<DevOp*>(smem_raw + L::ops_off);
        const DevPass& gP = passes[pass_index];
        const int sb = gP.stage_begin, se = gP.stage_end;
        const int ob = stages[sb].op_begin, oe = stages[se - 1].op_end;
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(&gP);
            uint32_t* dst = reinterpret_cast<uint32_t*>(sP);
            for (int w = tid; w < (int)(sizeof(DevPass) / 4); w += NT) dst[w] = src[w];
        }
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(stages + sb);
            uint32_t* dst = reinterpret_cast<uint32_t*>(sS);
            const int nw = (se - sb) * (int)(sizeof(DevStage) / 4);
            for (int w = tid; w < nw; w += NT) dst[w] = src[w];
        }
        {
            const uint4* src = reinterpret_cast<const uint4*>(ops + ob);
            uint4* dst = reinterpret_cast<uint4*>(sO);
            const int nw = (oe - ob) * (int)(sizeof(DevOp) / 16);
            for (int w = tid; w < nw; w += NT) dst[w] = src[w];
        }
        __syncthreads();
        Pp = sP;
        S0 = sS - sb;
        O0 = sO;
        op_base = ob;
    }
    const DevPass& P = *Pp;
    const int s0 = P.stage_begin, s1 = P.stage_end;
    const int nnl = P.n_nonlocal;

    for (uint64_t tile = blockIdx.x; tile < tiles; tile += (VAR >= 1 ? gridDim.x : tiles)) {
        uint64_t base = 0;
        for (int j = 0; j < nnl; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];

        V v[NR];
        {
            GOffs g;
            make_goffs<TBITS>(S0[s0], P, tid, g);
#pragma unroll
            for (int k = 0; k < NR; k++) v[k] = sv[base | goff_of(g, k)];
        }
        Slots cur;
        make_slots<T, TBITS>(S0[s0], tid, cur);
        const DevStage* last = &S0[s0];
        for (int s = s0; s < s1; s++) {
            const DevStage& S = S0[s];
            if (s != s0) {
                Slots nxt;
                make_slots<T, TBITS>(S, tid, nxt);
                relayout<V, NR>(sm, v, cur, nxt);
                cur = nxt;
                last = &S;
            }
            const int ob = S.op_begin - op_base, oe = S.op_end - op_base;
            for (int o = ob; o < oe; o++) {
                if constexpr (VAR == 2) apply_devop_fast<T>(O0 + o, v, tid, base);
                else apply_devop<T>(O0 + o, v, tid, base);
            }
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
}

static int staged_variant()
{
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SVB_STAGED_VARIANT");
        v = e ? std::atoi(e) : 2;
        if (v < 0 || v > 2) v = 2;
    }
    return v;
}

template <typename T, int M, int VAR>
static cudaError_t launch_staged_mv(void* state, int n, int pass_index, const DevPlanBuffers& b,
                                    cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    static int max_ctas[64] = {0};   // resident CTAs per device, 0 = not yet known
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = VAR >= 1 ? StagedSmem<T, M>::total : StagedSmem<T, M>::tile;
    if (dev < 64 && max_ctas[dev] == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_staged<T, M, VAR>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_staged<T, M, VAR>,
                                                          1 << (M - RB), smem);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        max_ctas[dev] = (per_sm > 0 ? per_sm : 1) * sms;
    }
    const uint64_t tiles = 1ull << (n - M);
    uint64_t grid = tiles;
    if (VAR >= 1 && dev < 64 && grid > (uint64_t)max_ctas[dev]) grid = (uint64_t)max_ctas[dev];
    k_staged<T, M, VAR><<<(unsigned)grid, 1 << (M - RB), smem, s>>>(
        static_cast<V*>(state), b.passes, b.stages, b.ops, pass_index, tiles);
    return cudaGetLastError();
}

template <typename T, int M>
static cudaError_t launch_staged_m(void* state, int n, int pass_index, const DevPlanBuffers& b,
                                   cudaStream_t s)
{
    switch (staged_variant()) {
    case 0: return launch_staged_mv<T, M, 0>(state, n, pass_index, b, s);
    case 1: return launch_staged_mv<T, M, 1>(state, n, pass_index, b, s);
    default: return launch_staged_mv<T, M, 2>(state, n, pass_index, b, s);
    }
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

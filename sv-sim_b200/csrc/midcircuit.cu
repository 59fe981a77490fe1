// Immediate-mode operations of the reference's Q#/QIR variant
// (svsim_qsharp/svsim_nvgpu_sin.cuh): gates with a control mask and mid-circuit Pauli
// measurement with collapse, applied to the handle's state on the GPU one call at a time.
//
//  * svb_apply_controlled: a 2x2 complex matrix on `target` for the amplitudes whose
//    control-mask bits are all 1 (the OP_HEAD_MASK rule, :680-690).  Only those pairs are
//    enumerated (both the target and the control bits are inserted into the pair index),
//    so a k-control gate touches 2^(n-k) amplitudes.
//  * svb_measure_qubit: Measure_GATE (:1486-1600).  The basis is changed (X: H; Y:
//    S^dagger then H), P(1) is summed in FP64 on the GPU, the outcome is 1 when the
//    caller's uniform r < P(1), the other half is zeroed and the kept half scaled by
//    1/sqrt(P(outcome)), and the basis change is undone (X: H; Y: H then S).
#include <algorithm>
#include <string>

#include "gate_math.cuh"

namespace svb {
namespace {

constexpr int MC_BLOCKS = REDUCE_BLOCKS;

// index of the i-th amplitude pair (target bit 0) with every control bit set; `bits` are
// the target and control positions in ascending order
__device__ __forceinline__ uint64_t mc_index(uint64_t i, const uint8_t* bits, int nb, uint64_t mask)
{
    uint64_t x = i;
    for (int b = 0; b < nb; b++) x = insert_zero(x, bits[b]);
    return x | mask;
}

struct McBits {
    uint8_t b[64];
    int n;
};

template <typename T>
__global__ void __launch_bounds__(256)
k_mc_apply(typename VecOf<T>::type* __restrict__ sv, uint64_t pairs, McBits bits, uint64_t mask, int target,
           Coef<T> c)
{
    using V = typename VecOf<T>::type;
    const uint64_t td = 1ull << target;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pairs;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p0 = mc_index(i, bits.b, bits.n, mask);
        V a0 = sv[p0], a1 = sv[p0 | td];
        dense_pair<T>(F_C1, c, a0, a1);
        sv[p0] = a0;
        sv[p0 | td] = a1;
    }
}

// FP64 partial sums of |a|^2 over the amplitudes with bit q set
template <typename T>
__global__ void __launch_bounds__(256)
k_prob_one(const typename VecOf<T>::type* __restrict__ sv, uint64_t half, int q, double* __restrict__ partial)
{
    __shared__ double red[8];
    double acc = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < half;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const auto a = sv[insert_zero(i, q) | (1ull << q)];
        acc += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
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

// out[0] = P(1) (fixed-order sum of the partials), out[1] = outcome (r < P(1))
__global__ void k_decide(const double* __restrict__ partial, int np, double r, double* __restrict__ out)
{
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += 32) s += partial[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) {
        out[0] = s;
        out[1] = (r < s) ? 1.0 : 0.0;
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_collapse(typename VecOf<T>::type* __restrict__ sv, uint64_t half, int q, const double* __restrict__ dec)
{
    using V = typename VecOf<T>::type;
    const double p1 = dec[0];
    const bool one = dec[1] != 0.0;
    const T f = static_cast<T>(1.0 / sqrt(one ? p1 : 1.0 - p1));
    V zero;
    zero.x = T(0);
    zero.y = T(0);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < half;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p0 = insert_zero(i, q), p1i = p0 | (1ull << q);
        V keep = sv[one ? p1i : p0];
        keep.x = keep.x * f;
        keep.y = keep.y * f;
        sv[one ? p1i : p0] = keep;
        sv[one ? p0 : p1i] = zero;
    }
}

unsigned grid_of(uint64_t items)
{
    const uint64_t need = (items + 255) / 256;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(need, 148ull * 8));
}

EOp basis_op(int form, int q)
{
    EOp e;
    e.form = (uint8_t)form;
    e.q = (uint32_t)q;          // H, S = diag(1, i), SDG = diag(1, -i): no coefficients
    return e;
}

template <typename T>
cudaError_t measure_qubit_t(Sim* s, int q, int pauli, double r, double* d_out, cudaStream_t st)
{
    using V = typename VecOf<T>::type;
    const int n = (int)s->n;
    V* sv = static_cast<V*>(s->state);
    const uint64_t half = 1ull << (n - 1);
    cudaError_t e = cudaSuccess;
    if (pauli == 1) e = launch_eop<T>(s->state, n, basis_op(F_H, q), st);
    if (pauli == 2) {
        e = launch_eop<T>(s->state, n, basis_op(F_SDG, q), st);
        if (e == cudaSuccess) e = launch_eop<T>(s->state, n, basis_op(F_H, q), st);
    }
    if (e != cudaSuccess) return e;
    k_prob_one<T><<<MC_BLOCKS, 256, 0, st>>>(sv, half, q, s->mscr.partial);
    k_decide<<<1, 32, 0, st>>>(s->mscr.partial, MC_BLOCKS, r, d_out);
    k_collapse<T><<<grid_of(half), 256, 0, st>>>(sv, half, q, d_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (pauli == 1) e = launch_eop<T>(s->state, n, basis_op(F_H, q), st);
    if (pauli == 2) {
        e = launch_eop<T>(s->state, n, basis_op(F_H, q), st);
        if (e == cudaSuccess) e = launch_eop<T>(s->state, n, basis_op(F_S, q), st);
    }
    return e;
}

}  // namespace
}  // namespace svb

using namespace svb;

extern "C" {

svb_status svb_apply_controlled(svb_sim* s, uint32_t target, uint64_t control_mask, const double* m, void* stream)
{
    if (!s || !m) { set_error("svb_apply_controlled: NULL argument"); return SVB_ERR_INVALID; }
    if (target >= s->n) { set_error("svb_apply_controlled: target >= n_qubits"); return SVB_ERR_INVALID; }
    if (s->n < 64 && (control_mask >> s->n)) {
        set_error("svb_apply_controlled: control mask names a qubit >= n_qubits");
        return SVB_ERR_INVALID;
    }
    if ((control_mask >> target) & 1ull) {
        set_error("svb_apply_controlled: the target is also a control");
        return SVB_ERR_INVALID;
    }
    McBits bits;
    bits.n = 0;
    for (uint32_t q = 0; q < s->n; q++)
        if (q == target || ((control_mask >> q) & 1ull)) bits.b[bits.n++] = (uint8_t)q;
    const uint64_t pairs = 1ull << (s->n - bits.n);
    cudaError_t e = cudaSetDevice(s->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (e == cudaSuccess) {
        if (s->precision == SVB_FP64) {
            Coef<double> c = load_coef<double>(m);
            k_mc_apply<double><<<grid_of(pairs), 256, 0, st>>>(static_cast<double2*>(s->state), pairs, bits,
                                                               control_mask, (int)target, c);
        } else {
            Coef<float> c = load_coef<float>(m);
            k_mc_apply<float><<<grid_of(pairs), 256, 0, st>>>(static_cast<float2*>(s->state), pairs, bits,
                                                              control_mask, (int)target, c);
        }
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_error(std::string("svb_apply_controlled: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return SVB_ERR_CUDA;
    }
    return SVB_OK;
}

svb_status svb_measure_qubit(svb_sim* s, uint32_t qubit, int pauli, double r, int* outcome, double* prob_one)
{
    if (!s) { set_error("svb_measure_qubit: NULL handle"); return SVB_ERR_INVALID; }
    if (qubit >= s->n) { set_error("svb_measure_qubit: qubit >= n_qubits"); return SVB_ERR_INVALID; }
    if (pauli < 0 || pauli > 2) { set_error("svb_measure_qubit: pauli must be 0 (Z), 1 (X) or 2 (Y)"); return SVB_ERR_INVALID; }
    cudaError_t e = cudaSetDevice(s->device);
    if (e == cudaSuccess && !s->mscr.partial) {
        e = cudaMalloc(&s->mscr.partial, REDUCE_BLOCKS * sizeof(double));
        if (e == cudaSuccess) s->mscr.cap_partial = REDUCE_BLOCKS;
    }
    if (e == cudaSuccess)
        e = s->precision == SVB_FP64 ? measure_qubit_t<double>(s, (int)qubit, pauli, r, s->d_small + 8, nullptr)
                                     : measure_qubit_t<float>(s, (int)qubit, pauli, r, s->d_small + 8, nullptr);
    double host[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(host, s->d_small + 8, sizeof(host), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_error(std::string("svb_measure_qubit: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return SVB_ERR_CUDA;
    }
    if (outcome) *outcome = host[1] != 0.0 ? 1 : 0;
    if (prob_one) *prob_one = host[0];
    return SVB_OK;
}

}  // extern "C"

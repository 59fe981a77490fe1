// Batched QAOA: many MaxCut instances of different sizes, each with its cost expectation
// and adjoint gradient, evaluated by one persistent cooperative launch that a CUDA graph
// replays (parameters in, launch, results out).
//
// Instance i has n_i qubits, a weighted graph and p layers (gamma_l, beta_l).  Its
// circuit in the reference gate set is H on every qubit, then per layer RZZ(-gamma w_e)
// on every edge and RX(2 beta) on every qubit.  The reference's RZZ is CX.U1(theta).CX
// (svsim_nvgpu_sin.cuh:1288-1294), which multiplies the amplitude of z by
// exp(i theta [z_a != z_b]); the edge layer is therefore the diagonal
// exp(-i gamma C(z)) with the MaxCut value C(z) = sum_e w_e [z_a != z_b], applied here as
// one phase per amplitude from a cost table built once per batch.  The mixer is the
// reference's RX (:1085-1100) with rx_real = cos(beta), rx_imag = -sin(beta).
//
// Tiles.  Every instance is cut into tiles of 2^M amplitudes (M = 12 FP64, 13 FP32:
// 64 KiB of state).  A layer takes two passes: the low pass holds qubits 0..M-1 (cost
// phase plus their RX), the high pass holds qubits 0..g-1 and M..n-1, g = 2M - n (the
// other RX).  Instances with n <= M are one tile and have no high pass.  The tiles of
// all instances in one pass form one phase of the launch; phases are separated by a
// grid barrier:
//   forward   F_low(l), F_high(l)          l = 0..p-1   (the last pass also forms the
//                                                        energy and lambda = C psi)
//   reverse   R_high(l), R_low(l)          l = p-1..0
// With psi and lambda taken at the point after layer l,
//   dE/dbeta_l = 2 Im <lambda| sum_q X_q |psi>,  dE/dgamma_l = 2 Im <lambda| C |psi>
// (mixer exp(-i beta sum X), cost layer exp(-i gamma C)); X_q commutes with every RX, so
// each pass adds the terms of the qubits it owns.
//
// Inside a tile.  512 threads hold 8 (FP64) or 16 (FP32) amplitudes each: 3 or 4 local
// bits live in registers, the 9 others come from the thread index.  Four stages move
// different local bits into registers (three exchanges through XOR-swizzled shared
// memory); the first stage loads from HBM and the last stores, both with the five lane
// bits on local bits 0..4, so a warp moves runs of 32 consecutive local amplitudes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "svb_internal.h"

namespace svb {
namespace {

constexpr int QB_THREADS = 512;
constexpr int QB_MAX_EDGES = 512;
constexpr unsigned kBarrierSpinLimit = 1u << 24;     // x >= 64 ns sleeps: > 1 s per barrier

template <typename T> struct QbCfg;
template <> struct QbCfg<double> {
    static constexpr int M = 12, RB = 3, NR = 8, SB = 3;
    // local bit held in register slot j during stage s
    static constexpr __host__ __device__ int reg_bit(int s, int j) { return s == 0 ? 9 + j : 3 * (s - 1) + j; }
    static constexpr __host__ __device__ bool owns(int, int) { return true; }
};
template <> struct QbCfg<float> {
    static constexpr int M = 13, RB = 4, NR = 16, SB = 4;
    static constexpr __host__ __device__ int reg_bit(int s, int j)
    {
        return s == 0 ? 9 + j : (s < 3 ? 4 * (s - 1) + j : 8 + j);
    }
    // stage 3 holds bits 8..11 but only bit 8 is new there
    static constexpr __host__ __device__ bool owns(int s, int j) { return s < 3 || j == 0; }
};

struct QaoaDesc {
    uint64_t state_off;      // first amplitude of the instance in the batch buffers
    uint64_t item_off;       // first tile of the instance within a pass
    uint32_t n;
    uint32_t pad;
};

struct QaoaArgs {
    void* psi;
    void* lam;
    const void* cost;            // C(z): double for FP64 batches, float for FP32
    const QaoaDesc* inst;
    const uint32_t* item_inst;   // [item]: the instance a tile belongs to
    const double* gammas;        // [inst][p]
    const double* mix;           // [inst][p] x (cos beta, -sin beta), from the host
    double* partial;             // [item][1 + 3p]: energy, dgamma_l, dbeta_l (low), dbeta_l (high)
    double* energy;              // [inst]
    double* grad;                // [inst][2p]: dE/dgamma_0..p-1, dE/dbeta_0..p-1
    unsigned* barrier;           // [0] arrival counter (zeroed before each launch), [1] error flag
    int n_inst;
    int p;
    uint64_t n_items;
};

template <typename T> struct AmpOf;
template <> struct AmpOf<double> { using type = double2; };
template <> struct AmpOf<float> { using type = float2; };

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier with a bounded wait.  The launch is cooperative, so every block is
// resident and the wait ends; if it does not within the limit, the error flag is set and
// the block goes on (the host then reports the launch as failed).
__device__ __forceinline__ void grid_barrier(unsigned* bar, unsigned target)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        unsigned spins = 0;
        while (ld_acquire(bar) < target) {
            if (++spins > kBarrierSpinLimit || ld_acquire(bar + 1) != 0u) {
                atomicOr(bar + 1, 1u);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

// two block sums in one pass (red holds 2 * QB_THREADS / 32 doubles); thread 0 gets both
__device__ __forceinline__ void block_sum2(double v, double w, double* red, double& sv, double& sw)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
        w += __shfl_xor_sync(0xffffffffu, w, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = v;
        red[QB_THREADS / 32 + (threadIdx.x >> 5)] = w;
    }
    __syncthreads();
    sv = 0;
    sw = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < QB_THREADS / 32; i++) {
            sv += red[i];
            sw += red[QB_THREADS / 32 + i];
        }
}

__device__ __forceinline__ double block_sum(double v, double* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < QB_THREADS / 32; w++) s += red[w];
    return s;
}

// thread-index bits deposited on the local bits that stage S does not hold in registers
template <typename T, int S>
__device__ __forceinline__ uint32_t thread_base(uint32_t tid)
{
    using C = QbCfg<T>;
    uint32_t out = 0;
    int k = 0;
#pragma unroll
    for (int b = 0; b < C::M; b++) {
        bool reg = false;
#pragma unroll
        for (int j = 0; j < C::RB; j++) reg |= (C::reg_bit(S, j) == b);
        if (!reg) {
            out |= ((tid >> k) & 1u) << b;
            k++;
        }
    }
    return out;
}

template <typename T, int S>
__device__ __forceinline__ constexpr uint32_t reg_off(int k)
{
    using C = QbCfg<T>;
    uint32_t o = 0;
    for (int j = 0; j < C::RB; j++) o |= uint32_t((k >> j) & 1) << C::reg_bit(S, j);
    return o;
}

template <typename T>
__device__ __forceinline__ uint32_t swz(uint32_t l)
{
    using C = QbCfg<T>;
    return l ^ ((l >> C::SB) & ((1u << C::SB) - 1));
}

// amplitude index within the instance of local index l of one tile
struct TileMap {
    uint64_t base;      // tile offset
    int g;              // high pass: local bits below g stay, bits >= g move up to M..n-1
    int shift;
    bool high;
    __device__ __forceinline__ uint64_t z(uint32_t l) const
    {
        if (!high) return base | l;
        const uint64_t lo = l & ((1u << g) - 1);
        return base | lo | (uint64_t(l >> g) << (g + shift));
    }
};

template <typename V, typename T>
__device__ __forceinline__ void rx_pair(V& a0, V& a1, T c, T s)
{
    // RX_GATE body with rx_real = c, rx_imag = s
    const T a0r = a0.x, a0i = a0.y, a1r = a1.x, a1i = a1.y;
    a0.x = (c * a0r) - (s * a1i);
    a0.y = (c * a0i) + (s * a1r);
    a1.x = -(s * a0i) + (c * a1r);
    a1.y = +(s * a0r) + (c * a1i);
}

// Im(conj(l) p), in the state's precision (sums are widened to FP64 once per stage)
template <typename V>
__device__ __forceinline__ auto im_conj_mul(const V& l, const V& p) -> decltype(l.x)
{
    return l.x * p.y - l.y * p.x;
}

// RX on every owned register slot of stage S whose local bit lies in [jb, je).  On the
// reverse sweep the X-derivative terms are added first and the inverse RX goes to both
// psi and lambda.
template <typename T, int S, bool REV>
__device__ __forceinline__ void stage_rx(typename AmpOf<T>::type* ps, typename AmpOf<T>::type* ls,
                                         int jb, int je, T c, T s, double& part_b)
{
    using C = QbCfg<T>;
    T acc = T(0);
#pragma unroll
    for (int j = 0; j < C::RB; j++) {
        if (!C::owns(S, j)) continue;
        const int bit = C::reg_bit(S, j);
        if (bit < jb || bit >= je) continue;
#pragma unroll
        for (int k = 0; k < C::NR; k++) {
            if (k & (1 << j)) continue;
            const int k1 = k | (1 << j);
            if (REV) {
                acc += im_conj_mul(ls[k], ps[k1]) + im_conj_mul(ls[k1], ps[k]);
                rx_pair(ps[k], ps[k1], c, T(-s));
                rx_pair(ls[k], ls[k1], c, T(-s));
            } else {
                rx_pair(ps[k], ps[k1], c, s);
            }
        }
    }
    if (REV) part_b += static_cast<double>(acc);
}

template <typename T, int SF, int ST>
__device__ __forceinline__ void exchange(typename AmpOf<T>::type* r, typename AmpOf<T>::type* buf,
                                         uint32_t tb_from, uint32_t tb_to)
{
    using C = QbCfg<T>;
#pragma unroll
    for (int k = 0; k < C::NR; k++) buf[swz<T>(tb_from | reg_off<T, SF>(k))] = r[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < C::NR; k++) r[k] = buf[swz<T>(tb_to | reg_off<T, ST>(k))];
}

// psi and lambda through their two buffers behind one barrier
template <typename T, int SF, int ST>
__device__ __forceinline__ void exchange2(typename AmpOf<T>::type* p, typename AmpOf<T>::type* l,
                                          typename AmpOf<T>::type* bp, typename AmpOf<T>::type* bl,
                                          uint32_t tb_from, uint32_t tb_to)
{
    using C = QbCfg<T>;
#pragma unroll
    for (int k = 0; k < C::NR; k++) {
        const uint32_t a = swz<T>(tb_from | reg_off<T, SF>(k));
        bp[a] = p[k];
        bl[a] = l[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < C::NR; k++) {
        const uint32_t a = swz<T>(tb_to | reg_off<T, ST>(k));
        p[k] = bp[a];
        l[k] = bl[a];
    }
}

__device__ __forceinline__ void cis(double ang, double& cr, double& ci) { sincos(ang, &ci, &cr); }
__device__ __forceinline__ void cis(float ang, float& cr, float& ci) { sincosf(ang, &ci, &cr); }

template <typename V, typename T>
__device__ __forceinline__ V cmul(const V& a, T cr, T ci)
{
    V b;
    b.x = cr * a.x - ci * a.y;
    b.y = cr * a.y + ci * a.x;
    return b;
}

template <typename T>
__global__ void __launch_bounds__(QB_THREADS, 1) k_qaoa(QaoaArgs A)
{
    using C = QbCfg<T>;
    using V = typename AmpOf<T>::type;
    constexpr int M = C::M, NR = C::NR;
    extern __shared__ __align__(16) unsigned char sm[];
    V* bp = reinterpret_cast<V*>(sm);
    V* bl = bp + (1u << M);
    double* red = reinterpret_cast<double*>(bl + (1u << M));

    V* psi = static_cast<V*>(A.psi);
    V* lam = static_cast<V*>(A.lam);
    const T* cost = static_cast<const T*>(A.cost);
    const int P = A.p;
    const int nq = 1 + 3 * P;
    const uint32_t tb0 = thread_base<T, 0>(threadIdx.x), tb1 = thread_base<T, 1>(threadIdx.x);
    const uint32_t tb2 = thread_base<T, 2>(threadIdx.x), tb3 = thread_base<T, 3>(threadIdx.x);

    V ps[NR], ls[NR];
    unsigned bar_target = 0;
    for (int ph = 0; ph < 4 * P; ph++) {
        const bool fwd = ph < 2 * P;
        const int r = fwd ? ph : ph - 2 * P;
        const int layer = fwd ? r / 2 : P - 1 - r / 2;
        const bool high = fwd ? (r & 1) : !(r & 1);
        for (uint64_t item = blockIdx.x; item < A.n_items; item += gridDim.x) {
            const int lo = (int)A.item_inst[item];
            const QaoaDesc D = A.inst[lo];
            const int n = (int)D.n;
            if (high && n <= M) continue;               // one-tile instance: no high pass
            const uint64_t t = item - D.item_off;
            const uint32_t size = n < M ? (1u << n) : (1u << M);
            TileMap tm;
            tm.high = high;
            tm.g = 2 * M - n;
            tm.shift = M - tm.g;
            tm.base = high ? (t << tm.g) : (t << M);
            const int jb = high ? tm.g : 0;
            const int je = high ? M : min(n, M);
            const bool last_fwd = fwd && layer == P - 1 && (high || n <= M);
            const double gamma = A.gammas[lo * P + layer];
            const T c = static_cast<T>(A.mix[2 * (lo * P + layer)]), s = static_cast<T>(A.mix[2 * (lo * P + layer) + 1]);
            const T gam = static_cast<T>(gamma);
            V* gp = psi + D.state_off;
            V* gl = lam + D.state_off;
            const T* gc = cost + D.state_off;
            double part_e = 0, part_g = 0, part_b = 0;

            // stage 0: HBM -> registers
            if (fwd && layer == 0 && !high) {
                T amp = T(1);
                for (int q = 0; q < n; q++) amp = static_cast<T>(0.70710678118654752440) * amp;
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    const uint32_t l = tb0 | reg_off<T, 0>(k);
                    ps[k].x = l < size ? amp : T(0);
                    ps[k].y = T(0);
                }
            } else {
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    const uint32_t l = tb0 | reg_off<T, 0>(k);
                    const bool ok = l < size;
                    const uint64_t z = tm.z(l);
                    V zero;
                    zero.x = T(0);
                    zero.y = T(0);
                    ps[k] = ok ? gp[z] : zero;
                    if (!fwd) ls[k] = ok ? gl[z] : zero;
                }
            }
            if (fwd && !high) {                         // cost layer exp(-i gamma C(z))
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    const uint32_t l = tb0 | reg_off<T, 0>(k);
                    const T cz = l < size ? gc[tm.z(l)] : T(0);
                    T cr, ci;
                    cis(-gam * cz, cr, ci);
                    ps[k] = cmul(ps[k], cr, ci);
                }
            }
            // stages 0..3: mixer on the owned bits, with exchanges between stages
            if (fwd) {
                // the exchanges alternate between the two buffers (lambda's is free on the
                // forward sweep), so a buffer is written again only after a barrier that
                // every read of it precedes
                stage_rx<T, 0, false>(ps, ls, jb, je, c, s, part_b);
                exchange<T, 0, 1>(ps, bp, tb0, tb1);
                stage_rx<T, 1, false>(ps, ls, jb, je, c, s, part_b);
                exchange<T, 1, 2>(ps, bl, tb1, tb2);
                stage_rx<T, 2, false>(ps, ls, jb, je, c, s, part_b);
                exchange<T, 2, 3>(ps, bp, tb2, tb3);
                stage_rx<T, 3, false>(ps, ls, jb, je, c, s, part_b);
            } else {
                stage_rx<T, 0, true>(ps, ls, jb, je, c, s, part_b);
                exchange2<T, 0, 1>(ps, ls, bp, bl, tb0, tb1);
                stage_rx<T, 1, true>(ps, ls, jb, je, c, s, part_b);
                __syncthreads();
                exchange2<T, 1, 2>(ps, ls, bp, bl, tb1, tb2);
                stage_rx<T, 2, true>(ps, ls, jb, je, c, s, part_b);
                __syncthreads();
                exchange2<T, 2, 3>(ps, ls, bp, bl, tb2, tb3);
                stage_rx<T, 3, true>(ps, ls, jb, je, c, s, part_b);
            }
            // stage 3: diagonal work on the final layout, then registers -> HBM
            if (last_fwd) {
                T acc = T(0);
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    const uint32_t l = tb3 | reg_off<T, 3>(k);
                    const T cz = l < size ? gc[tm.z(l)] : T(0);
                    const T pr = ps[k].x, pi = ps[k].y;
                    acc += cz * (pr * pr + pi * pi);
                    ls[k].x = cz * pr;
                    ls[k].y = cz * pi;
                }
                part_e = static_cast<double>(acc);
            }
            if (!fwd && !high) {
                T acc = T(0);
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    const uint32_t l = tb3 | reg_off<T, 3>(k);
                    const T cz = l < size ? gc[tm.z(l)] : T(0);
                    acc += cz * im_conj_mul(ls[k], ps[k]);
                    T cr, ci;
                    cis(gam * cz, cr, ci);
                    ps[k] = cmul(ps[k], cr, ci);
                    ls[k] = cmul(ls[k], cr, ci);
                }
                part_g = static_cast<double>(acc);
            }
            const bool store_psi = fwd || layer > 0 || high;
            const bool store_lam = (!fwd && store_psi) || last_fwd;
            if (store_psi) {
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    const uint32_t l = tb3 | reg_off<T, 3>(k);
                    if (l < size) {
                        const uint64_t z = tm.z(l);
                        gp[z] = ps[k];
                        if (store_lam) gl[z] = ls[k];
                    }
                }
            }
            double* pt = A.partial + item * (uint64_t)nq;
            if (last_fwd) {
                const double v = block_sum(part_e, red);
                if (threadIdx.x == 0) pt[0] = v;
            }
            if (!fwd) {
                double vb, vg;
                block_sum2(part_b, part_g, red, vb, vg);
                if (threadIdx.x == 0) {
                    pt[1 + (high ? 2 * P : P) + layer] = 2.0 * vb;
                    if (!high) pt[1 + layer] = 2.0 * vg;
                }
            }
            __syncthreads();
        }
        bar_target += gridDim.x;
        grid_barrier(A.barrier, bar_target);
    }
    // per-instance sums over the instance's tiles, one warp per (instance, quantity)
    const uint64_t warps = (uint64_t)gridDim.x * (QB_THREADS / 32);
    const uint64_t wid = ((uint64_t)blockIdx.x * QB_THREADS + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nout = 1 + 2 * P;
    for (uint64_t job = wid; job < (uint64_t)A.n_inst * nout; job += warps) {
        const int ii = (int)(job / nout), q = (int)(job % nout);
        const uint64_t i0 = A.inst[ii].item_off;
        const uint64_t i1 = ii + 1 < A.n_inst ? A.inst[ii + 1].item_off : A.n_items;
        double s = 0;
        for (uint64_t it = i0 + lane; it < i1; it += 32) {
            const double* pt = A.partial + it * (uint64_t)nq;
            if (q == 0) s += pt[0];
            else if (q <= P) s += pt[q];
            else s += pt[q] + pt[q + P];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if (q == 0) A.energy[ii] = s;
            else A.grad[(size_t)ii * 2 * P + (q - 1)] = s;
        }
    }
}

// C(z) = sum_e w_e [z_a != z_b] for every amplitude of every instance, summed in edge order
template <typename T>
__global__ void k_cost_table(const QaoaDesc* inst, int n_inst, const uint32_t* edge_off,
                             const uint32_t* edges, const double* w, uint64_t total, T* cost)
{
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < total;
         a += (uint64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_inst;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (inst[mid].state_off <= a) lo = mid; else hi = mid;
        }
        const uint64_t z = a - inst[lo].state_off;
        double c = 0;
        for (uint32_t e = edge_off[lo]; e < edge_off[lo + 1]; e++) {
            const uint32_t ab = edges[e];
            if (((z >> (ab & 0xffffu)) ^ (z >> (ab >> 16))) & 1ull) c += w[e];
        }
        cost[a] = static_cast<T>(c);
    }
}

}  // namespace
// One CTA arrives at a grid barrier whose target (two arrivals) is never reached: the
// bounded wait of grid_barrier gives up and raises bar[1] (the batched kernels' error flag).
__global__ void k_grid_barrier_probe(unsigned* bar)
{
    grid_barrier(bar, 2u);
}

cudaError_t launch_grid_barrier_probe(unsigned* bar, cudaStream_t s)
{
    k_grid_barrier_probe<<<1, 32, 0, s>>>(bar);
    return cudaGetLastError();
}

}  // namespace svb

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
using namespace svb;

struct svb_qaoa_batch {
    int device = 0;
    int precision = SVB_FP64;
    int M = 12;
    uint32_t n_inst = 0, p = 0;
    uint64_t n_items = 0, total_amps = 0;
    double moved_bytes = 0;
    void* psi = nullptr;
    void* lam = nullptr;
    void* cost = nullptr;
    QaoaDesc* d_inst = nullptr;
    uint32_t* d_item_inst = nullptr; // instance of each tile of a pass
    double* d_params = nullptr;      // gammas, betas, then (cos beta, -sin beta) pairs
    double* d_partial = nullptr;
    double* d_out = nullptr;         // energies then gradients
    unsigned* d_bar = nullptr;       // barrier counter, error flag
    double* h_params = nullptr;      // pinned
    double* h_out = nullptr;         // pinned
    unsigned* h_err = nullptr;       // pinned
    size_t smem = 0;
    int grid = 0;
    bool graphed = false;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
};

namespace {

void free_batch(svb_qaoa_batch* b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->stream) cudaStreamDestroy(b->stream);
    cudaFree(b->psi);
    cudaFree(b->lam);
    cudaFree(b->cost);
    cudaFree(b->d_inst);
    cudaFree(b->d_item_inst);
    cudaFree(b->d_params);
    cudaFree(b->d_partial);
    cudaFree(b->d_out);
    cudaFree(b->d_bar);
    cudaFreeHost(b->h_params);
    cudaFreeHost(b->h_out);
    cudaFreeHost(b->h_err);
    delete b;
}

template <typename T>
cudaError_t setup_kernel(svb_qaoa_batch* b)
{
    using V = typename AmpOf<T>::type;
    b->smem = 2 * (sizeof(V) << QbCfg<T>::M) + 2 * (QB_THREADS / 32) * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_qaoa<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_qaoa<T>, QB_THREADS, b->smem)) != cudaSuccess)
        return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    b->grid = per_sm * sms;
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_batch(svb_qaoa_batch* b, cudaStream_t s)
{
    QaoaArgs a;
    a.psi = b->psi;
    a.lam = b->lam;
    a.cost = b->cost;
    a.inst = b->d_inst;
    a.item_inst = b->d_item_inst;
    a.gammas = b->d_params;
    a.mix = b->d_params + (size_t)2 * b->n_inst * b->p;
    a.partial = b->d_partial;
    a.energy = b->d_out;
    a.grad = b->d_out + b->n_inst;
    a.barrier = b->d_bar;
    a.n_inst = (int)b->n_inst;
    a.p = (int)b->p;
    a.n_items = b->n_items;
    cudaError_t e = cudaMemsetAsync(b->d_bar, 0, 2 * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel((const void*)k_qaoa<T>, dim3(b->grid), dim3(QB_THREADS), args,
                                       b->smem, s);
}

cudaError_t launch_any(svb_qaoa_batch* b, cudaStream_t s)
{
    return b->precision == SVB_FP64 ? launch_batch<double>(b, s) : launch_batch<float>(b, s);
}

// host pinned params -> device, launch, device results and error flag -> host pinned
cudaError_t enqueue_run(svb_qaoa_batch* b, cudaStream_t s)
{
    const size_t np = (size_t)4 * b->n_inst * b->p;
    const size_t no = (size_t)b->n_inst * (1 + 2 * b->p);
    cudaError_t e = cudaMemcpyAsync(b->d_params, b->h_params, np * 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    if ((e = launch_any(b, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b->h_out, b->d_out, no * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    return cudaMemcpyAsync(b->h_err, b->d_bar + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
}

svb_status cuda_fail(const std::string& where, cudaError_t e)
{
    set_error(where + ": " + cudaGetErrorString(e));
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? SVB_ERR_OOM : SVB_ERR_CUDA;
}

}  // namespace

extern "C" {

svb_status svb_qaoa_create(int device, int precision, uint32_t n_instances, const uint32_t* n_qubits,
                           const uint32_t* edge_offsets, const uint32_t* edges, const double* weights,
                           uint32_t p, svb_qaoa_batch** out)
{
    if (!out) { set_error("svb_qaoa_create: out is NULL"); return SVB_ERR_INVALID; }
    *out = nullptr;
    if (!n_qubits || !edge_offsets || n_instances == 0 || p == 0 || p > 64) {
        set_error("svb_qaoa_create: need at least one instance, 1 <= p <= 64 and non-NULL arrays");
        return SVB_ERR_INVALID;
    }
    if (precision != SVB_FP64 && precision != SVB_FP32) {
        set_error("svb_qaoa_create: precision must be SVB_FP64 or SVB_FP32");
        return SVB_ERR_INVALID;
    }
    if (edge_offsets[0] != 0) { set_error("svb_qaoa_create: edge_offsets[0] must be 0"); return SVB_ERR_INVALID; }
    // two passes of 2^M-amplitude tiles cover every qubit when n <= 2M
    const uint32_t max_n = 2u * (precision == SVB_FP64 ? QbCfg<double>::M : QbCfg<float>::M);
    for (uint32_t i = 0; i < n_instances; i++) {
        const uint32_t n = n_qubits[i];
        if (edge_offsets[i + 1] < edge_offsets[i] || edge_offsets[i + 1] - edge_offsets[i] > (uint32_t)QB_MAX_EDGES ||
            n < 2 || n > max_n) {
            set_error("svb_qaoa_create: instance " + std::to_string(i) + " needs 2.." + std::to_string(max_n) +
                      " qubits and at most " + std::to_string(QB_MAX_EDGES) + " edges");
            return SVB_ERR_INVALID;
        }
        for (uint32_t e = edge_offsets[i]; e < edge_offsets[i + 1]; e++) {
            if (!edges || !weights || edges[2 * e] >= n || edges[2 * e + 1] >= n || edges[2 * e] == edges[2 * e + 1]) {
                set_error("svb_qaoa_create: instance " + std::to_string(i) + " has an edge outside [0, n) or a loop");
                return SVB_ERR_INVALID;
            }
        }
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail("svb_qaoa_create", e);
    svb_qaoa_batch* b = new svb_qaoa_batch();
    b->device = device;
    b->precision = precision;
    b->M = precision == SVB_FP64 ? QbCfg<double>::M : QbCfg<float>::M;
    b->n_inst = n_instances;
    b->p = p;
    const size_t amp_bytes = precision == SVB_FP64 ? 16 : 8;
    const size_t cost_bytes = precision == SVB_FP64 ? 8 : 4;
    std::vector<QaoaDesc> desc(n_instances);
    uint64_t amps = 0, items = 0;
    double moved = 0;
    for (uint32_t i = 0; i < n_instances; i++) {
        const int n = (int)n_qubits[i];
        desc[i].state_off = amps;
        desc[i].item_off = items;
        desc[i].n = (uint32_t)n;
        desc[i].pad = 0;
        const double A = double(1ull << n) * amp_bytes, Cb = double(1ull << n) * cost_bytes;
        // state and cost bytes one evaluation reads and writes (forward, lambda, reverse)
        moved += (n > b->M ? (12.0 * p - 2) : (6.0 * p - 2)) * A + (2.0 * p + 1) * Cb;
        amps += 1ull << n;
        items += n <= b->M ? 1ull : (1ull << (n - b->M));
    }
    b->n_items = items;
    b->total_amps = amps;
    b->moved_bytes = moved;
    const uint32_t E = edge_offsets[n_instances];
    std::vector<uint32_t> packed(std::max<uint32_t>(E, 1), 0);
    std::vector<uint32_t> eoff(edge_offsets, edge_offsets + n_instances + 1);
    for (uint32_t k = 0; k < E; k++) packed[k] = edges[2 * k] | (edges[2 * k + 1] << 16);
    const uint32_t nq = 1 + 3 * p, nout = 1 + 2 * p;

    auto fail = [&](const char* what, cudaError_t err) {
        const svb_status st = cuda_fail(std::string("svb_qaoa_create: ") + what, err);
        free_batch(b);
        return st;
    };
    uint32_t *d_eoff = nullptr, *d_edges = nullptr;
    double* d_w = nullptr;
    auto free_tmp = [&]() { cudaFree(d_eoff); cudaFree(d_edges); cudaFree(d_w); };
    if ((e = cudaMalloc(&b->psi, amps * amp_bytes)) != cudaSuccess) return fail("state", e);
    if ((e = cudaMalloc(&b->lam, amps * amp_bytes)) != cudaSuccess) return fail("co-state", e);
    if ((e = cudaMalloc(&b->cost, amps * cost_bytes)) != cudaSuccess) return fail("cost table", e);
    if ((e = cudaMalloc(&b->d_inst, desc.size() * sizeof(QaoaDesc))) != cudaSuccess) return fail("alloc", e);
    if ((e = cudaMalloc(&b->d_params, (size_t)4 * n_instances * p * 8)) != cudaSuccess) return fail("alloc", e);
    if ((e = cudaMalloc(&b->d_partial, items * nq * 8)) != cudaSuccess) return fail("alloc", e);
    if ((e = cudaMalloc(&b->d_out, (size_t)n_instances * nout * 8)) != cudaSuccess) return fail("alloc", e);
    if ((e = cudaMalloc(&b->d_bar, 2 * sizeof(unsigned))) != cudaSuccess) return fail("alloc", e);
    if ((e = cudaMallocHost(&b->h_params, (size_t)4 * n_instances * p * 8)) != cudaSuccess) return fail("alloc", e);
    if ((e = cudaMallocHost(&b->h_out, (size_t)n_instances * nout * 8)) != cudaSuccess) return fail("alloc", e);
    if ((e = cudaMallocHost(&b->h_err, sizeof(unsigned))) != cudaSuccess) return fail("alloc", e);
    std::memset(b->h_params, 0, (size_t)4 * n_instances * p * 8);
    if ((e = cudaMemcpy(b->d_inst, desc.data(), desc.size() * sizeof(QaoaDesc), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail("upload", e);
    {
        std::vector<uint32_t> item_inst(std::max<uint64_t>(items, 1), 0);
        for (uint32_t i = 0; i < n_instances; i++) {
            const uint64_t end = i + 1 < n_instances ? desc[i + 1].item_off : items;
            for (uint64_t t = desc[i].item_off; t < end; t++) item_inst[t] = i;
        }
        if ((e = cudaMalloc(&b->d_item_inst, item_inst.size() * 4)) != cudaSuccess) return fail("alloc", e);
        if ((e = cudaMemcpy(b->d_item_inst, item_inst.data(), item_inst.size() * 4, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return fail("upload", e);
    }
    // the high-pass entries of one-tile instances are never written: zero them once
    if ((e = cudaMemset(b->d_partial, 0, items * nq * 8)) != cudaSuccess) return fail("memset", e);
    if ((e = cudaMalloc(&d_eoff, eoff.size() * 4)) != cudaSuccess ||
        (e = cudaMalloc(&d_edges, packed.size() * 4)) != cudaSuccess ||
        (e = cudaMalloc(&d_w, std::max<uint32_t>(E, 1) * 8)) != cudaSuccess) {
        free_tmp();
        return fail("alloc", e);
    }
    if ((e = cudaMemcpy(d_eoff, eoff.data(), eoff.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d_edges, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (E && (e = cudaMemcpy(d_w, weights, (size_t)E * 8, cudaMemcpyHostToDevice)) != cudaSuccess)) {
        free_tmp();
        return fail("upload", e);
    }
    const int cgrid = 148 * 8;
    if (precision == SVB_FP64)
        k_cost_table<double><<<cgrid, 256>>>(b->d_inst, (int)n_instances, d_eoff, d_edges, d_w, amps,
                                             static_cast<double*>(b->cost));
    else
        k_cost_table<float><<<cgrid, 256>>>(b->d_inst, (int)n_instances, d_eoff, d_edges, d_w, amps,
                                            static_cast<float*>(b->cost));
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    free_tmp();
    if (e != cudaSuccess) return fail("cost table", e);
    e = precision == SVB_FP64 ? setup_kernel<double>(b) : setup_kernel<float>(b);
    if (e != cudaSuccess) return fail("kernel setup", e);
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail("stream", e);
    // capture the whole evaluation; without a graph the same sequence is issued per call
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const cudaError_t le = enqueue_run(b, b->stream);
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (le == cudaSuccess && ce == cudaSuccess && g &&
            cudaGraphInstantiate(&b->graph, g, 0) == cudaSuccess)
            b->graphed = true;
        else
            b->graph = nullptr;
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
    }
    *out = b;
    return SVB_OK;
}

svb_status svb_qaoa_run(svb_qaoa_batch* b, const double* gammas, const double* betas, double* energies,
                        double* grads)
{
    if (!b || !gammas || !betas) { set_error("svb_qaoa_run: NULL argument"); return SVB_ERR_INVALID; }
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) return cuda_fail("svb_qaoa_run", e);
    const size_t np = (size_t)b->n_inst * b->p;
    std::memcpy(b->h_params, gammas, np * 8);
    std::memcpy(b->h_params + np, betas, np * 8);
    for (size_t i = 0; i < np; i++) {             // the mixer's RX(2 beta) coefficients
        b->h_params[2 * np + 2 * i] = std::cos(betas[i]);
        b->h_params[2 * np + 2 * i + 1] = -std::sin(betas[i]);
    }
    *b->h_err = 0;
    e = b->graphed ? cudaGraphLaunch(b->graph, b->stream) : enqueue_run(b, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail("svb_qaoa_run", e);
    if (*b->h_err) {
        set_error("svb_qaoa_run: a grid barrier timed out; results are invalid");
        return SVB_ERR_STATE;
    }
    if (energies) std::memcpy(energies, b->h_out, b->n_inst * 8);
    if (grads) std::memcpy(grads, b->h_out + b->n_inst, np * 2 * 8);
    return SVB_OK;
}

svb_status svb_qaoa_launch(svb_qaoa_batch* b, void* stream)
{
    if (!b) { set_error("svb_qaoa_launch: NULL batch"); return SVB_ERR_INVALID; }
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = launch_any(b, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail("svb_qaoa_launch", e);
    return SVB_OK;
}

svb_status svb_qaoa_info(const svb_qaoa_batch* b, svb_qaoa_stats* info)
{
    if (!b || !info) { set_error("svb_qaoa_info: NULL argument"); return SVB_ERR_INVALID; }
    info->n_instances = b->n_inst;
    info->p = b->p;
    info->tile_bits = (uint32_t)b->M;
    info->graphed = b->graphed ? 1 : 0;
    info->total_amplitudes = b->total_amps;
    info->tiles_per_pass = b->n_items;
    info->moved_bytes = b->moved_bytes;
    info->grid = (uint32_t)b->grid;
    info->reserved = 0;
    return SVB_OK;
}

svb_status svb_qaoa_destroy(svb_qaoa_batch* b)
{
    if (!b) return SVB_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_batch(b);
    return SVB_OK;
}

}  // extern "C"

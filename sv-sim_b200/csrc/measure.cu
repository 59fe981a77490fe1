// FP64 probability reductions and measurement sampling on the GPU.
//
// The reference samples on the host (svsim/src/svsim_nvgpu_sin.cuh:359-383): it copies
// the whole state back, builds a sequential inclusive scan S of |a|^2 (2^n+1 doubles),
// and for each shot keeps the j with S_j <= r < S_{j+1} (0 if none) by a linear scan.
// Here the same rule is evaluated on the device without a 2^n scan array:
//   1. k_block_sums   one warp per block of 4096 amplitudes; the block is walked in
//                     128 coalesced chunks of 32, each chunk summed by a fixed
//                     butterfly, chunk sums accumulated in index order (FP64);
//   2. k_scan_single  exclusive scan of the block sums (plus the total);
//   3. k_sample       one warp per shot: binary search of the block prefix, then the
//                     same chunk walk as step 1 from the block's prefix until the chunk
//                     holding r, then a warp inclusive scan inside that chunk.
// Every partial sum is non-negative, so the resulting prefix sums are non-decreasing
// in the index, and the sample is the first index whose inclusive sum exceeds r.
#include "gate_math.cuh"

namespace svb {
namespace {

constexpr int BLOCK_AMPS = 1 << MEAS_BLOCK_BITS;   // 4096
constexpr int CHUNKS = BLOCK_AMPS / 32;            // 128

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ double prob_at(const typename VecOf<T>::type* sv, uint64_t dim, uint64_t i)
{
    if (i >= dim) return 0.0;
    const auto a = sv[i];
    const double r = (double)a.x, m = (double)a.y;
    return (r * r) + (m * m);
}

template <typename T>
__global__ void __launch_bounds__(256)
k_block_sums(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim, uint64_t nblocks,
             double* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t b = warp; b < nblocks; b += nwarps) {
        const uint64_t base = b * BLOCK_AMPS;
        double acc = 0.0;
        for (int c = 0; c < CHUNKS; c++) {
            const uint64_t i0 = base + (uint64_t)c * 32;
            if (i0 >= dim) break;
            acc += warp_sum(prob_at<T>(sv, dim, i0 + lane));
        }
        if (lane == 0) out[b] = acc;
    }
}

// Exclusive scan of `in[0..count)` into out[0..count], out[count] = total.  One block
// of 1024 threads: each owns a contiguous segment (sequential sums), the segment
// totals are scanned across the block, then each segment is rewritten.
__global__ void __launch_bounds__(1024)
k_scan_single(const double* __restrict__ in, uint64_t count, double* __restrict__ out)
{
    __shared__ double wsum[32];
    const int t = threadIdx.x;
    const uint64_t seg = (count + 1023) / 1024;
    const uint64_t b = (uint64_t)t * seg;
    const uint64_t e = b + seg < count ? b + seg : count;
    double local = 0.0;
    for (uint64_t i = b; i < e; i++) local += in[i];
    // block exclusive scan of `local`
    const int lane = t & 31, w = t >> 5;
    double incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        double x = wsum[lane];
        double xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        wsum[lane] = xi - x;   // exclusive over warps
    }
    __syncthreads();
    double run = wsum[w] + (incl - local);
    for (uint64_t i = b; i < e; i++) {
        out[i] = run;
        run += in[i];
    }
    if (t == 1023) out[count] = wsum[31] + incl;
}

template <typename T>
__global__ void __launch_bounds__(256)
k_sample(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim, uint64_t nblocks,
         const double* __restrict__ prefix, const double* __restrict__ uniforms, uint32_t shots,
         uint64_t* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const uint64_t shot = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (shot >= shots) return;
    const double r = uniforms[shot];
    const double total = prefix[nblocks];
    uint64_t result = 0;
    if (r >= 0.0 && r < total) {
        uint64_t lo = 0, hi = nblocks;   // prefix[lo] <= r < prefix[hi]
        while (hi - lo > 1) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (prefix[mid] <= r) lo = mid;
            else hi = mid;
        }
        const uint64_t base = lo * BLOCK_AMPS;
        double acc = prefix[lo];
        uint64_t last_nonzero = base;
        bool found = false;
        for (int c = 0; c < CHUNKS && !found; c++) {
            const uint64_t i0 = base + (uint64_t)c * 32;
            if (i0 >= dim) break;
            const double p = prob_at<T>(sv, dim, i0 + lane);
            const double s = warp_sum(p);
            const unsigned nz = __ballot_sync(0xffffffffu, p > 0.0);
            if (acc + s > r) {
                double incl = p;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const double y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const unsigned hit = __ballot_sync(0xffffffffu, p > 0.0 && acc + incl > r);
                if (hit) {
                    result = i0 + (__ffs(hit) - 1);
                    found = true;
                } else {
                    acc += s;
                }
            } else {
                acc += s;
            }
            if (nz) last_nonzero = i0 + (31 - __clz(nz));
        }
        // r fell in a rounding gap at the end of the block: the last populated index
        if (!found) result = last_nonzero;
    }
    if (lane == 0) out[shot] = result;
}

template <typename T>
__global__ void __launch_bounds__(256)
k_pauli_expect(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim,
               const svb_pauli_term* __restrict__ terms, int n_terms, double* __restrict__ partial)
{
    extern __shared__ svb_pauli_term sterms[];
    __shared__ double red[8];
    for (int t = threadIdx.x; t < n_terms; t += blockDim.x) sterms[t] = terms[t];
    __syncthreads();
    double acc = 0.0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
        const auto a = sv[i];
        const double ar = (double)a.x, ai = (double)a.y;
        for (int t = 0; t < n_terms; t++) {
            const uint64_t xm = sterms[t].x_mask, zm = sterms[t].z_mask;
            const uint64_t j = i ^ xm;
            const auto b = sv[j];
            double br = (double)b.x, bi = (double)b.y;
            if (__popcll(j & zm) & 1) { br = -br; bi = -bi; }
            double tr, ti;
            switch (__popcll(xm & zm) & 3) {     // i^(number of Y factors)
            case 0: tr = br; ti = bi; break;
            case 1: tr = -bi; ti = br; break;
            case 2: tr = -br; ti = -bi; break;
            default: tr = bi; ti = -br; break;
            }
            acc += sterms[t].coef * (ar * tr + ai * ti);
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        partial[blockIdx.x] = s;
    }
}

__global__ void k_sum_partials(const double* __restrict__ partial, int count, double* __restrict__ out)
{
    // one warp, fixed order: deterministic
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += 32) s += partial[i];
    s = warp_sum(s);
    if (threadIdx.x == 0) *out = s;
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(256)
k_compare(const typename VecOf<TA>::type* __restrict__ a, const typename VecOf<TB>::type* __restrict__ b,
          uint64_t dim, double* __restrict__ partial)
{
    __shared__ double red[5][8];
    double re = 0, im = 0, na = 0, nb = 0, mx = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
        const double ar = (double)a[i].x, ai = (double)a[i].y;
        const double br = (double)b[i].x, bi = (double)b[i].y;
        re += ar * br + ai * bi;            // conj(a) b
        im += ar * bi - ai * br;
        na += ar * ar + ai * ai;
        nb += br * br + bi * bi;
        const double dr = ar - br, di = ai - bi;
        mx = fmax(mx, sqrt(dr * dr + di * di));
    }
    double v[5] = {re, im, na, nb, mx};
#pragma unroll
    for (int q = 0; q < 5; q++) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = (q == 4) ? fmax(x, y) : x + y;
        }
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        const int q = threadIdx.x;
        double x = red[q][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) x = (q == 4) ? fmax(x, red[q][w]) : x + red[q][w];
        partial[(size_t)q * gridDim.x + blockIdx.x] = x;
    }
}

__global__ void k_compare_final(const double* __restrict__ partial, int blocks, double* __restrict__ out)
{
    if (threadIdx.x != 0) return;
    double v[5] = {0, 0, 0, 0, 0};
    for (int q = 0; q < 5; q++)
        for (int i = 0; i < blocks; i++) {
            const double x = partial[(size_t)q * blocks + i];
            v[q] = (q == 4) ? fmax(v[q], x) : v[q] + x;
        }
    for (int q = 0; q < 5; q++) out[q] = v[q];
}

}  // namespace

template <typename TA, typename TB>
cudaError_t compare_device(const void* a, const void* b, int n, double* d_out5, double* d_partial5,
                           cudaStream_t s)
{
    const uint64_t dim = 1ull << n;
    k_compare<TA, TB><<<REDUCE_BLOCKS, 256, 0, s>>>(static_cast<const typename VecOf<TA>::type*>(a),
                                                   static_cast<const typename VecOf<TB>::type*>(b), dim,
                                                   d_partial5);
    k_compare_final<<<1, 32, 0, s>>>(d_partial5, REDUCE_BLOCKS, d_out5);
    return cudaGetLastError();
}
template cudaError_t compare_device<double, double>(const void*, const void*, int, double*, double*, cudaStream_t);
template cudaError_t compare_device<double, float>(const void*, const void*, int, double*, double*, cudaStream_t);
template cudaError_t compare_device<float, double>(const void*, const void*, int, double*, double*, cudaStream_t);
template cudaError_t compare_device<float, float>(const void*, const void*, int, double*, double*, cudaStream_t);

size_t measure_scratch_doubles(int n)
{
    const uint64_t dim = 1ull << n;
    return (size_t)((dim + BLOCK_AMPS - 1) / BLOCK_AMPS);
}

template <typename T>
static cudaError_t block_prefix(const void* state, int n, MeasureScratch& scr, cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    const uint64_t dim = 1ull << n;
    const uint64_t nb = measure_scratch_doubles(n);
    const uint64_t warps_needed = nb;
    unsigned blocks = (unsigned)((warps_needed * 32 + 255) / 256);
    if (blocks > 148u * 16) blocks = 148u * 16;
    k_block_sums<T><<<blocks, 256, 0, s>>>(static_cast<const V*>(state), dim, nb, scr.block_sums);
    k_scan_single<<<1, 1024, 0, s>>>(scr.block_sums, nb, scr.block_prefix);
    return cudaGetLastError();
}

template <typename T>
cudaError_t measure_device(const void* state, int n, const double* d_uniforms, uint32_t shots,
                           uint64_t* d_samples, double* d_total, MeasureScratch& scr, cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    const uint64_t dim = 1ull << n;
    const uint64_t nb = measure_scratch_doubles(n);
    cudaError_t e = block_prefix<T>(state, n, scr, s);
    if (e != cudaSuccess) return e;
    if (shots > 0) {
        const unsigned blocks = (unsigned)(((uint64_t)shots * 32 + 255) / 256);
        k_sample<T><<<blocks, 256, 0, s>>>(static_cast<const V*>(state), dim, nb, scr.block_prefix,
                                           d_uniforms, shots, d_samples);
    }
    if (d_total)
        e = cudaMemcpyAsync(d_total, scr.block_prefix + nb, sizeof(double),
                            cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <typename T>
cudaError_t expectation_device(const void* state, int n, const svb_pauli_term* d_terms, int n_terms,
                               double* d_out, double* d_partial, cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    const uint64_t dim = 1ull << n;
    const size_t smem = sizeof(svb_pauli_term) * (size_t)n_terms;
    k_pauli_expect<T><<<REDUCE_BLOCKS, 256, smem, s>>>(static_cast<const V*>(state), dim, d_terms,
                                                        n_terms, d_partial);
    k_sum_partials<<<1, 32, 0, s>>>(d_partial, REDUCE_BLOCKS, d_out);
    return cudaGetLastError();
}

#define SVB_MEAS_INST(T)                                                                    \
    template cudaError_t measure_device<T>(const void*, int, const double*, uint32_t,       \
                                           uint64_t*, double*, MeasureScratch&, cudaStream_t); \
    template cudaError_t expectation_device<T>(const void*, int, const svb_pauli_term*, int, \
                                               double*, double*, cudaStream_t);
SVB_MEAS_INST(double)
SVB_MEAS_INST(float)

}  // namespace svb

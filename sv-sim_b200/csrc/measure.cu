// FP64 probability reductions and measurement sampling on the GPU.
//
// The reference samples on the host (svsim/src/svsim_nvgpu_sin.cuh:359-383): it copies
// the whole state back, builds the sequential inclusive scan S_0 = 0,
// S_{i+1} = fl(S_i + p_i) with p_i = fl(fl(re_i*re_i) + fl(im_i*im_i)) (2^n+1 doubles),
// and for each shot keeps the j with S_j <= r < S_{j+1} (0 if none).  The samples here
// are those of that exact S, bit for bit, without a sequential pass and without a 2^n
// scan array.
//
// Why a parallel pass can give the sequential sums exactly: while S stays inside one
// binade [2^e, 2^(e+1)), every value S takes is an integer multiple m of the grid unit
// u = 2^(e-52) (m in [2^52, 2^53)), and fl(S + p) = (m + round(p/u)) u, where round is
// to the nearest integer — unless p/u has a fractional part of exactly one half (a
// tie: round-half-even then depends on the last bit of m) or m + p/u reaches 2^53 (the
// sum leaves the binade and the grid doubles).  So a run of elements without ties
// that stays in the binade advances m by an exact integer sum of per-element
// roundings, which adds up in any order.  Ties and binade crossings (at most a few
// dozen crossings, S being non-decreasing) are added one element at a time with
// IEEE adds in index order.
//
// Passes (B = 4096 amplitudes per block, 64 blocks per superblock):
//   1. k_block_sums   approximate FP64 block sums (any order) -> k_scan_single gives
//                     an approximate prefix, used only to guess each block's binade;
//   2. k_cdf_blocks   per block: the exact integer sum D_b of round(p_i/u) on the
//                     guessed binade's grid, or "zero block" / "no delta" (a tie, a
//                     guessed crossing, or no normal start);
//   3. k_cdf_super    per superblock: the sum of its blocks' D_b when they share one
//                     binade, else "no delta";
//   4. k_cdf_chain    one warp walks the superblocks in order from S = 0: a delta
//                     applies when S is in its binade and stays there (checked on the
//                     exact S), otherwise the warp descends to blocks and, where a
//                     block's delta does not apply either, to chunks of 32 elements
//                     (chunk_scan_exact);
//   5. k_cdf_fill     the exact S at every block start of the superblocks the chain
//                     did not descend into;
//   6. k_sample_exact one warp per shot: binary search over the exact block starts,
//                     then chunk_scan_exact through the block to the first index whose
//                     inclusive S exceeds r.
// Every step computes the reference's sequential values themselves, so equal inputs
// give the reference's samples whatever the summation order of pass 1.
#include "gate_math.cuh"

namespace svb {
namespace {

constexpr int BLOCK_AMPS = 1 << MEAS_BLOCK_BITS;   // 4096
constexpr int CHUNKS = BLOCK_AMPS / 32;            // 128
constexpr int SUPER_BLOCKS = 1 << MEAS_SUPER_BITS; // 64
constexpr uint64_t FRAC_MASK = (1ull << 52) - 1;
constexpr uint64_t HIDDEN = 1ull << 52;
constexpr uint64_t M_MAX = (1ull << 53) - 1;       // largest grid count inside one binade
// A block or superblock entry: bits 0..52 hold the delta D in grid units, bits 53..63
// the biased exponent code of its binade (e + 1023, in [1, 2046]); code 0 = no delta
// (its D field is then 1 if no probability of the range is NaN), code 2047 = every
// probability of the range is zero.
constexpr uint32_t CODE_NONE = 0, CODE_ZERO = 2047;

__device__ __forceinline__ uint64_t pack_entry(uint64_t d, uint32_t code) { return (uint64_t)code << 53 | d; }
__device__ __forceinline__ uint32_t entry_code(uint64_t w) { return (uint32_t)(w >> 53); }
__device__ __forceinline__ uint64_t entry_delta(uint64_t w) { return w & M_MAX; }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// |a_i|^2 as the reference forms it (svsim_nvgpu_sin.cuh:362-365): both products
// rounded, then added; never contracted into an FMA.
template <typename T>
__device__ __forceinline__ double prob_at(const typename VecOf<T>::type* sv, uint64_t dim, uint64_t i)
{
    if (i >= dim) return 0.0;
    const auto a = sv[i];
    const double r = (double)a.x, m = (double)a.y;
    return __dadd_rn(__dmul_rn(r, r), __dmul_rn(m, m));
}

// Binade code of a positive normal double (e + 1023), or 0 for 0, subnormals, inf,
// NaN and negatives; *m receives its significand as an integer in [2^52, 2^53).
__device__ __forceinline__ uint32_t binade_of(double s, uint64_t* m)
{
    const uint64_t b = (uint64_t)__double_as_longlong(s);
    const uint32_t code = (uint32_t)(b >> 52);      // sign bit included: negatives give >= 2048
    if (code == 0 || code >= 2047) return 0;
    *m = (b & FRAC_MASK) | HIDDEN;
    return code;
}

__device__ __forceinline__ double from_grid(uint32_t code, uint64_t m)   // m in [2^52, 2^53)
{
    return __longlong_as_double((long long)(((uint64_t)code << 52) | (m - HIDDEN)));
}

// p / 2^(e-52) rounded to the nearest integer, for p >= 0 (e = code - 1023).  *ok is
// cleared on a tie (fraction exactly 1/2) and for NaN or inf.  Exact integer
// arithmetic on p's significand.
__device__ __forceinline__ uint64_t grid_units(double p, uint32_t code, bool* ok)
{
    const uint64_t b = (uint64_t)__double_as_longlong(p);
    const int pb = (int)((b >> 52) & 0x7ff);
    if (pb == 0x7ff) { *ok = false; return 0; }
    uint64_t mp = b & FRAC_MASK;
    int ep = -1022;
    if (pb != 0) { mp |= HIDDEN; ep = pb - 1023; }
    const int sh = ((int)code - 1023) - ep;          // p / u = mp * 2^-sh
    if (sh < 0) {                                    // p >= 2^53 u: leaves the binade
        if (mp != 0) *ok = false;
        return 0;
    }
    if (sh == 0) {                                   // p / u = mp
        if (mp >= HIDDEN) *ok = false;
        return mp;
    }
    if (sh >= 64) return 0;                          // p / u < 2^-11
    const uint64_t ip = mp >> sh;
    const uint64_t fr = mp & ((1ull << sh) - 1);
    const uint64_t half = 1ull << (sh - 1);
    if (fr == half) *ok = false;
    return ip + (fr > half ? 1 : 0);
}

// S advanced by `d` grid units of binade `code`, if S lies in that binade and stays
// there; returns false (S unchanged) otherwise.
__device__ __forceinline__ bool advance(double* s, uint32_t code, uint64_t d)
{
    uint64_t m;
    if (binade_of(*s, &m) != code || code == 0) return false;
    if (d > M_MAX - m) return false;
    *s = from_grid(code, m + d);
    return true;
}

// The reference's inclusive sums over one chunk of 32 consecutive elements, exactly:
// lane l receives S_{j0+l+1} given s_in = S_{j0} (warp-uniform) and its own p.
// Integer grid deltas when no lane ties and the chunk stays in s_in's binade; else
// 32 IEEE adds in index order, evaluated by every lane.
__device__ __forceinline__ double chunk_scan_exact(double s_in, double p, int lane)
{
    uint64_t m;
    const uint32_t code = binade_of(s_in, &m);
    if (code != 0) {
        bool ok = true;
        const uint64_t d = grid_units(p, code, &ok);
        uint64_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint64_t total = __shfl_sync(0xffffffffu, incl, 31);
        if (__all_sync(0xffffffffu, ok) && total <= M_MAX - m) return from_grid(code, m + incl);
    } else if (s_in == 0.0 && __all_sync(0xffffffffu, p == 0.0)) {
        return 0.0;
    }
    double s = s_in, mine = 0.0;
#pragma unroll 8
    for (int k = 0; k < 32; k++) {
        s = __dadd_rn(s, __shfl_sync(0xffffffffu, p, k));
        if (k == lane) mine = s;
    }
    return mine;
}

template <typename T>
__device__ double walk_block(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim, uint64_t b,
                             double s, int lane)
{
    const uint64_t base = b * BLOCK_AMPS;
    for (int c = 0; c < CHUNKS; c++) {
        const uint64_t i0 = base + (uint64_t)c * 32;
        if (i0 >= dim) break;
        const double incl = chunk_scan_exact(s, prob_at<T>(sv, dim, i0 + lane), lane);
        s = __shfl_sync(0xffffffffu, incl, 31);
    }
    return s;
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

// Pass 2: one warp per block.  The binade guess is that of the approximate prefix at
// the block's start; a block whose approximate end lies in another binade is left
// without a delta (the chain adds it element by element).
template <typename T>
__global__ void __launch_bounds__(256)
k_cdf_blocks(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim, uint64_t nblocks,
             const double* __restrict__ approx, uint64_t* __restrict__ entry)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t b = warp; b < nblocks; b += nwarps) {
        uint64_t m0, m1;
        const uint32_t c0 = binade_of(approx[b], &m0);
        const uint32_t c1 = binade_of(approx[b + 1], &m1);
        const uint32_t code = (c0 != 0 && c0 == c1) ? c0 : 0;
        const uint64_t base = b * BLOCK_AMPS;
        uint64_t acc = 0;
        bool ok = true, nonzero = false, nan_free = true;
        for (int c = 0; c < CHUNKS; c++) {
            const uint64_t i0 = base + (uint64_t)c * 32;
            if (i0 >= dim) break;
            const double p = prob_at<T>(sv, dim, i0 + lane);
            nonzero |= (p != 0.0);
            nan_free &= (p == p);
            if (code != 0) acc += grid_units(p, code, &ok);
        }
        nonzero = __any_sync(0xffffffffu, nonzero);
        nan_free = __all_sync(0xffffffffu, nan_free);
        ok = __all_sync(0xffffffffu, ok);
        acc = warp_sum_u64(acc);               // < 4096 * 2^52: no wrap
        if (lane == 0) {
            uint64_t w = pack_entry(nan_free ? 1 : 0, CODE_NONE);
            if (!nonzero) w = pack_entry(0, CODE_ZERO);
            else if (code != 0 && ok && acc < HIDDEN) w = pack_entry(acc, code);
            entry[b] = w;
        }
    }
}

// Pass 3: one thread per superblock.
__global__ void __launch_bounds__(256)
k_cdf_super(const uint64_t* __restrict__ entry, uint64_t nblocks, uint64_t nsuper,
            uint64_t* __restrict__ sentry)
{
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsuper) return;
    const uint64_t b0 = s * SUPER_BLOCKS;
    const uint64_t b1 = b0 + SUPER_BLOCKS < nblocks ? b0 + SUPER_BLOCKS : nblocks;
    uint32_t code = CODE_ZERO;
    uint64_t d = 0;
    bool ok = true, nan_free = true;
    for (uint64_t b = b0; b < b1; b++) {
        const uint64_t w = entry[b];
        const uint32_t c = entry_code(w);
        if (c == CODE_ZERO) continue;
        if (c == CODE_NONE) {
            ok = false;
            nan_free = nan_free && entry_delta(w) == 1;
            continue;
        }
        if (code != CODE_ZERO && c != code) ok = false;
        code = c;
        d += entry_delta(w);                   // each < 2^52, at most 64 of them
        if (d >= HIDDEN) ok = false;
    }
    sentry[s] = ok ? pack_entry(code == CODE_ZERO ? 0 : d, code) : pack_entry(nan_free ? 1 : 0, CODE_NONE);
}

// S can no longer change over a range: S is NaN, or S is +inf and no probability of
// the range is NaN.
__device__ __forceinline__ bool stuck(double s, uint64_t w)
{
    if (s != s) return true;
    return isinf(s) && (entry_code(w) != CODE_NONE || entry_delta(w) == 1);
}

// Pass 4: one warp.  Entries are read 32 at a time (one per lane) and broadcast, so
// the chain waits on memory once per 32 superblocks or blocks.  desc[s] = 1 marks a
// superblock whose block starts the chain wrote itself.
template <typename T>
__global__ void __launch_bounds__(32)
k_cdf_chain(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim, uint64_t nblocks,
            uint64_t nsuper, const uint64_t* __restrict__ entry, const uint64_t* __restrict__ sentry,
            double* __restrict__ start, double* __restrict__ sstart, uint32_t* __restrict__ desc)
{
    const int lane = threadIdx.x;
    double s_val = 0.0;
    for (uint64_t g = 0; g < nsuper; g += 32) {
        const uint64_t mine = g + lane < nsuper ? sentry[g + lane] : 0;
        const uint64_t cnt = nsuper - g < 32 ? nsuper - g : 32;
        for (uint64_t k = 0; k < cnt; k++) {
            const uint64_t sidx = g + k;
            const uint64_t w = __shfl_sync(0xffffffffu, mine, (int)k);
            if (lane == 0) sstart[sidx] = s_val;
            const uint32_t code = entry_code(w);
            if (code == CODE_ZERO || stuck(s_val, w) ||
                (code != CODE_NONE && advance(&s_val, code, entry_delta(w)))) {
                if (lane == 0) desc[sidx] = 0;
                continue;
            }
            if (lane == 0) desc[sidx] = 1;
            const uint64_t b0 = sidx * SUPER_BLOCKS;
            const uint64_t b1 = b0 + SUPER_BLOCKS < nblocks ? b0 + SUPER_BLOCKS : nblocks;
            for (uint64_t h = b0; h < b1; h += 32) {
                const uint64_t bm = h + lane < b1 ? entry[h + lane] : 0;
                const uint64_t bc = b1 - h < 32 ? b1 - h : 32;
                for (uint64_t j = 0; j < bc; j++) {
                    const uint64_t b = h + j;
                    const uint64_t wb = __shfl_sync(0xffffffffu, bm, (int)j);
                    if (lane == 0) start[b] = s_val;
                    const uint32_t cb = entry_code(wb);
                    if (cb == CODE_ZERO || stuck(s_val, wb)) continue;
                    if (cb != CODE_NONE && advance(&s_val, cb, entry_delta(wb))) continue;
                    s_val = walk_block<T>(sv, dim, b, s_val, lane);
                }
            }
        }
    }
    if (lane == 0) {
        start[nblocks] = s_val;
        sstart[nsuper] = s_val;
    }
}

// Pass 5: one thread per superblock the chain did not descend into; its blocks'
// deltas all apply (they share the superblock's binade and their sum stays in it).
__global__ void __launch_bounds__(256)
k_cdf_fill(const uint64_t* __restrict__ entry, uint64_t nblocks, uint64_t nsuper,
           const double* __restrict__ sstart, const uint32_t* __restrict__ desc,
           double* __restrict__ start)
{
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsuper || desc[s]) return;
    const uint64_t b0 = s * SUPER_BLOCKS;
    const uint64_t b1 = b0 + SUPER_BLOCKS < nblocks ? b0 + SUPER_BLOCKS : nblocks;
    double v = sstart[s];
    for (uint64_t b = b0; b < b1; b++) {
        start[b] = v;
        const uint64_t w = entry[b];
        const uint32_t c = entry_code(w);
        if (c != CODE_ZERO && c != CODE_NONE && v == v) advance(&v, c, entry_delta(w));
    }
}

// Pass 6: one warp per shot.  start[] holds the reference's S at every block start
// (start[nblocks] = S_{2^n}); the block with start[b] <= r < start[b+1] is walked with
// the exact chunk sums until the first index j whose S_{j+1} exceeds r, which is the
// reference's j with S_j <= r < S_{j+1}.  Shots with no such j (r >= S_{2^n}, r < 0 or
// NaN) give 0 as in the reference.
template <typename T>
__global__ void __launch_bounds__(256)
k_sample_exact(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim, uint64_t nblocks,
               const double* __restrict__ start, const double* __restrict__ uniforms, uint32_t shots,
               uint64_t* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const uint64_t shot = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (shot >= shots) return;
    const double r = uniforms[shot];
    uint64_t result = 0;
    if (r >= 0.0 && r < start[nblocks]) {
        uint64_t lo = 0, hi = nblocks;   // start[lo] <= r < start[hi]
        while (hi - lo > 1) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (start[mid] <= r) lo = mid;
            else hi = mid;
        }
        const uint64_t base = lo * BLOCK_AMPS;
        double s = start[lo];
        result = ~0ull;                  // replaced below: start[lo+1] > r is met inside the block
        for (int c = 0; c < CHUNKS; c++) {
            const uint64_t i0 = base + (uint64_t)c * 32;
            if (i0 >= dim) break;
            const double incl = chunk_scan_exact(s, prob_at<T>(sv, dim, i0 + lane), lane);
            const unsigned hit = __ballot_sync(0xffffffffu, incl > r);
            if (hit) {
                result = i0 + (uint64_t)(__ffs(hit) - 1);
                break;
            }
            s = __shfl_sync(0xffffffffu, incl, 31);
        }
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

size_t measure_scratch_doubles(int n) { return (size_t)measure_layout(n).doubles; }

template <typename T>
cudaError_t measure_device(const void* state, int n, const double* d_uniforms, uint32_t shots,
                           uint64_t* d_samples, double* d_total, MeasureScratch& scr, cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    const MeasureLayout L = measure_layout(n);
    if (!scr.cdf || scr.cap_doubles < L.doubles) return cudaErrorInvalidValue;
    const V* sv = static_cast<const V*>(state);
    const uint64_t dim = 1ull << n;
    double* base = scr.cdf;
    uint64_t* entry = reinterpret_cast<uint64_t*>(base + L.off_entry);
    double* start = base + L.off_start;
    uint64_t* sentry = reinterpret_cast<uint64_t*>(base + L.off_sentry);
    double* sstart = base + L.off_sstart;
    uint32_t* desc = reinterpret_cast<uint32_t*>(base + L.off_desc);
    // 1. approximate block sums (into the entry array) and their prefix (into start)
    unsigned blocks = (unsigned)((L.nblocks * 32 + 255) / 256);
    if (blocks > 148u * 16) blocks = 148u * 16;
    k_block_sums<T><<<blocks, 256, 0, s>>>(sv, dim, L.nblocks, base + L.off_entry);
    k_scan_single<<<1, 1024, 0, s>>>(base + L.off_entry, L.nblocks, start);
    // 2-5. exact block starts
    k_cdf_blocks<T><<<blocks, 256, 0, s>>>(sv, dim, L.nblocks, start, entry);
    const unsigned sb = (unsigned)((L.nsuper + 255) / 256);
    k_cdf_super<<<sb, 256, 0, s>>>(entry, L.nblocks, L.nsuper, sentry);
    k_cdf_chain<T><<<1, 32, 0, s>>>(sv, dim, L.nblocks, L.nsuper, entry, sentry, start, sstart, desc);
    k_cdf_fill<<<sb, 256, 0, s>>>(entry, L.nblocks, L.nsuper, sstart, desc, start);
    // 6. samples
    if (shots > 0) {
        const unsigned sblocks = (unsigned)(((uint64_t)shots * 32 + 255) / 256);
        k_sample_exact<T><<<sblocks, 256, 0, s>>>(sv, dim, L.nblocks, start, d_uniforms, shots, d_samples);
    }
    cudaError_t e = cudaSuccess;
    if (d_total)
        e = cudaMemcpyAsync(d_total, start + L.nblocks, sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <typename T>
cudaError_t norm2_device(const void* state, int n, double* d_total, MeasureScratch& scr, cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    const MeasureLayout L = measure_layout(n);
    if (!scr.cdf || scr.cap_doubles < L.doubles) return cudaErrorInvalidValue;
    double* base = scr.cdf;
    unsigned blocks = (unsigned)((L.nblocks * 32 + 255) / 256);
    if (blocks > 148u * 16) blocks = 148u * 16;
    k_block_sums<T><<<blocks, 256, 0, s>>>(static_cast<const V*>(state), 1ull << n, L.nblocks, base + L.off_entry);
    k_scan_single<<<1, 1024, 0, s>>>(base + L.off_entry, L.nblocks, base + L.off_start);
    cudaError_t e = cudaMemcpyAsync(d_total, base + L.off_start + L.nblocks, sizeof(double),
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
    template cudaError_t norm2_device<T>(const void*, int, double*, MeasureScratch&, cudaStream_t); \
    template cudaError_t expectation_device<T>(const void*, int, const svb_pauli_term*, int, \
                                               double*, double*, cudaStream_t);
SVB_MEAS_INST(double)
SVB_MEAS_INST(float)

}  // namespace svb

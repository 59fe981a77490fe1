// Device helpers shared by the fused tensor-core kernels (kernels_fused.cu,
// kernels_fused6.cu): shared-memory and instruction descriptors of tcgen05.mma, bounded
// mbarrier waits, tensor-memory loads and stores, the split of an FP32 value into the two
// TF32 terms the MMAs read, and 16-byte cp.async copies.
#pragma once

#include <cstdint>

namespace svb {
namespace {

constexpr uint32_t kSuspendNs = 20000;          // longest sleep of one mbarrier try
constexpr uint64_t kWaitNs = 2000000000ull;     // a wait gives up after 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// canonical K-major, no-swizzle shared-memory descriptor
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;                 // descriptor version (sm_100)
    return d;                               // base offset 0, LBO mode 0, no swizzle
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc_tf32(uint32_t n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// one try: the warp sleeps (issuing nothing) until the phase completes or kSuspendNs pass
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done) : "r"(a), "r"(parity), "r"(kSuspendNs) : "memory");
    return done != 0;
}

// bounded wait: gives up after kWaitNs
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    if (mbar_try(a, parity)) return true;
    const uint64_t t0 = global_ns();
    while (global_ns() - t0 < kWaitNs)
        if (mbar_try(a, parity)) return true;
    return false;
}

// x = hi + lo for the MMA: hi is x itself, of which the MMA reads only the top 19 bits
// (x truncated to TF32), and lo is the exact remainder x - trunc(x), which the MMA in turn
// truncates to TF32.  What that second truncation drops is below 2^-22 of |x| and biased
// towards zero; the closing FP64 renormalisation of a fused run removes the resulting
// uniform shrink (rounding lo to nearest instead costs two more instructions per value
// on the kernels' critical path, for no measurable change in fidelity).
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo)
{
    hi = x;
    lo = x - __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);   // exact
}

// 8 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v)
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}


// D[tmem] (+)= A[tmem] . B[smem]
__device__ __forceinline__ void mma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                            uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                 :: "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])),
                    "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])),
                    "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
                 : "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
        :: "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
           "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
           "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
           "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
           "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
           "r"(__float_as_uint(v[15]))
        : "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float* v)
{
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 4; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st4(uint32_t taddr, const float* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};"
                 :: "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])),
                    "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3]))
                 : "memory");
}

// W consecutive TMEM columns of this warp's 32 lanes (W = 4, 8, 16 or 32)
template <int W>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, float* v)
{
    if constexpr (W == 4) {
        tmem_ld4(taddr, v);
    } else if constexpr (W == 8) {
        tmem_ld8(taddr, v);
    } else {
#pragma unroll
        for (int c = 0; c < W; c += 16) tmem_ld16(taddr + (uint32_t)c, v + c);
    }
}

template <int W>
__device__ __forceinline__ void tmem_st_cols(uint32_t taddr, const float* v)
{
    if constexpr (W == 4) {
        tmem_st4(taddr, v);
    } else if constexpr (W == 8) {
        tmem_st8(taddr, v);
    } else {
#pragma unroll
        for (int c = 0; c < W; c += 16) tmem_st16(taddr + (uint32_t)c, v + c);
    }
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

// bounded wait that also gives up once *abort is set; a wait that runs out sets it
__device__ __forceinline__ bool mbar_wait_abort(uint64_t* bar, uint32_t parity, volatile int* abort)
{
    const uint32_t a = smem_u32(bar);
    if (mbar_try(a, parity)) return true;
    const uint64_t t0 = global_ns();
    while (global_ns() - t0 < kWaitNs) {
        if (mbar_try(a, parity)) return true;
        if (*abort) return false;
    }
    *abort = 1;
    return false;
}

// 16 bytes global -> shared, asynchronous (L2 only)
__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_u32(dst)), "l"(src) : "memory");
}

// 8 bytes global -> shared, asynchronous
__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(smem_u32(dst)), "l"(src) : "memory");
}

// arrive on the mbarrier once all of this thread's earlier cp.async copies have landed
__device__ __forceinline__ void cp_async_arrive(uint64_t* bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}

}  // namespace
}  // namespace svb

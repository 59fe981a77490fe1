// Per-thread logic of the staged engine's tile kernel (k_staged in kernels_apply.cu):
// shared-memory swizzle, layout decoding and the application of one planned op to the
// 16 register-held amplitudes of a thread.  Host-callable as well, so that tests can
// execute a plan on the CPU with exactly the kernel's index arithmetic.
#pragma once

#include "gate_math.cuh"

namespace svb {

// XOR swizzle of a local index into a shared-memory slot.  The low G bits are
// XOR-ed with the fold of every higher G-bit group, so a layout whose lowest G lane
// bits sit at positions with distinct residues mod G touches 2^G distinct 16-byte
// (FP64) or 8-byte (FP32) bank groups per phase: conflict-free.
template <typename T> struct Swz;
template <> struct Swz<double> {
    static constexpr int G = 3;
    SVB_HD static uint32_t f(uint32_t l) {
        const uint32_t x = l >> 3;
        return l ^ ((x ^ (x >> 3) ^ (x >> 6) ^ (x >> 9)) & 7u);
    }
};
template <> struct Swz<float> {
    static constexpr int G = 4;
    SVB_HD static uint32_t f(uint32_t l) {
        const uint32_t x = l >> 4;
        return l ^ ((x ^ (x >> 4) ^ (x >> 8)) & 15u);
    }
};

struct Slots {
    uint32_t thr;          // swizzled shared slot of the thread part of the index
    uint32_t reg[RB];      // swizzled slot of each register bit
};

template <typename T, int TBITS>
SVB_HD void make_slots(const DevStage& S, int tid, Slots& o)
{
    uint32_t lt = 0;
#pragma unroll
    for (int b = 0; b < TBITS; b++)
        if ((tid >> b) & 1) lt |= 1u << S.thr_pos[b];
    o.thr = Swz<T>::f(lt);
#pragma unroll
    for (int i = 0; i < RB; i++) o.reg[i] = Swz<T>::f(1u << S.reg_pos[i]);
}

SVB_HD uint32_t slot_of(const Slots& s, int k)
{
    uint32_t r = s.thr;
#pragma unroll
    for (int i = 0; i < RB; i++)
        if ((k >> i) & 1) r ^= s.reg[i];
    return r;
}

// Global offsets of a layout (only needed while loading and storing a tile).
struct GOffs {
    uint64_t thr;
    uint64_t reg[RB];
};

template <int TBITS>
SVB_HD void make_goffs(const DevStage& S, const DevPass& P, int tid, GOffs& o)
{
    uint64_t gt = 0;
#pragma unroll
    for (int b = 0; b < TBITS; b++)
        if ((tid >> b) & 1) gt |= 1ull << P.local_q[S.thr_pos[b]];
    o.thr = gt;
#pragma unroll
    for (int i = 0; i < RB; i++) o.reg[i] = 1ull << P.local_q[S.reg_pos[i]];
}

SVB_HD uint64_t goff_of(const GOffs& g, int k)
{
    uint64_t r = g.thr;
#pragma unroll
    for (int i = 0; i < RB; i++)
        if ((k >> i) & 1) r |= g.reg[i];
    return r;
}

template <int TB, typename V, typename F>
SVB_HD void pairs_tb(V* v, F&& f)
{
#pragma unroll
    for (int k = 0; k < (1 << RB); k++)
        if (!(k & (1 << TB))) f(v[k], v[k | (1 << TB)], k);
}

template <typename V, typename F>
SVB_HD void for_pairs(int tb, V* v, F&& f)
{
    switch (tb) {
    case 0: pairs_tb<0>(v, f); break;
    case 1: pairs_tb<1>(v, f); break;
    case 2: pairs_tb<2>(v, f); break;
    default: pairs_tb<3>(v, f); break;
    }
}

template <int TB, typename V, typename F1, typename F0>
SVB_HD void split_tb(V* v, F1&& f1, F0&& f0)
{
#pragma unroll
    for (int k = 0; k < (1 << RB); k++) {
        if (k & (1 << TB)) f1(v[k]);
        else f0(v[k]);
    }
}

// Apply f1 to elements whose register bit `tb` is 1 and f0 to the others.
template <typename V, typename F1, typename F0>
SVB_HD void for_split(int tb, V* v, F1&& f1, F0&& f0)
{
    switch (tb) {
    case 0: split_tb<0>(v, f1, f0); break;
    case 1: split_tb<1>(v, f1, f0); break;
    case 2: split_tb<2>(v, f1, f0); break;
    default: split_tb<3>(v, f1, f0); break;
    }
}

template <typename T, int FORM, typename V>
SVB_HD void dense_all(int tgt, const Coef<T>& c, V* v)
{
    for_pairs(tgt, v, [&](V& a0, V& a1, int) { dense_pair<T>(FORM, c, a0, a1); });
}

template <typename T, int FORM, typename V>
SVB_HD void diag_all(int loc_kind, int loc_bit, bool uni, const Coef<T>& c, V* v)
{
    if (loc_kind == LOC_REG) {
        for_split(loc_bit, v, [&](V& a) { diag_one<T>(FORM, c, a); },
                  [&](V& a) { diag_zero<T>(FORM, c, a); });
    } else if (uni) {
#pragma unroll
        for (int k = 0; k < (1 << RB); k++) diag_one<T>(FORM, c, v[k]);
    } else if (FORM == F_DIAG) {
#pragma unroll
        for (int k = 0; k < (1 << RB); k++) diag_zero<T>(FORM, c, v[k]);
    }
}

template <typename T, typename V>
SVB_HD void apply_devop(const DevOp* __restrict__ opp, V* v, int tid,
                                            uint64_t base)
{
    const int form = opp->form;
    const int tgt = opp->tgt;
    const int loc_kind = opp->loc_kind;
    const int loc_bit = opp->loc_bit;
    bool uni = true;   // value of a thread- or tile-located qubit
    if (loc_kind == LOC_THR) uni = (tid >> loc_bit) & 1;
    else if (loc_kind == LOC_TILE) uni = (base >> opp->tile_qubit) & 1;

    if (form == F_CX) {
        if (loc_kind == LOC_REG) {
            const int cb = loc_bit;
            for_pairs(tgt, v, [&](V& a0, V& a1, int k) {
                const bool on = (k >> cb) & 1;
                const V x0 = a0, x1 = a1;
                a0 = on ? x1 : x0;
                a1 = on ? x0 : x1;
            });
        } else if (uni) {
            for_pairs(tgt, v, [&](V& a0, V& a1, int) { const V t = a0; a0 = a1; a1 = t; });
        }
        return;
    }
    const Coef<T> c = load_coef<T>(opp->m);
    switch (form) {
    case F_C1:  dense_all<T, F_C1>(tgt, c, v); break;
    case F_X:   dense_all<T, F_X>(tgt, c, v); break;
    case F_Y:   dense_all<T, F_Y>(tgt, c, v); break;
    case F_H:   dense_all<T, F_H>(tgt, c, v); break;
    case F_SRN: dense_all<T, F_SRN>(tgt, c, v); break;
    case F_W:   dense_all<T, F_W>(tgt, c, v); break;
    case F_RX:  dense_all<T, F_RX>(tgt, c, v); break;
    case F_RY:  dense_all<T, F_RY>(tgt, c, v); break;
    case F_Z:   diag_all<T, F_Z>(loc_kind, loc_bit, uni, c, v); break;
    case F_S:   diag_all<T, F_S>(loc_kind, loc_bit, uni, c, v); break;
    case F_SDG: diag_all<T, F_SDG>(loc_kind, loc_bit, uni, c, v); break;
    case F_T:   diag_all<T, F_T>(loc_kind, loc_bit, uni, c, v); break;
    case F_TDG: diag_all<T, F_TDG>(loc_kind, loc_bit, uni, c, v); break;
    case F_R:   diag_all<T, F_R>(loc_kind, loc_bit, uni, c, v); break;
    case F_U1:  diag_all<T, F_U1>(loc_kind, loc_bit, uni, c, v); break;
    case F_DIAG: diag_all<T, F_DIAG>(loc_kind, loc_bit, uni, c, v); break;
    default: break;
    }
}

}  // namespace svb

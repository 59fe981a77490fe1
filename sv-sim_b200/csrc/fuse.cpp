// Gate fusion for the fused tensor-core engine (FP32 states).
//
// The elementary-op stream (the reference's gate sequences, lower.cpp) is cut into
// passes over tiles of 2^FT_TILE_BITS amplitudes, as the staged engine does, except that
// every qubit an op touches must be local to the pass.  Inside a pass the ops are
// grouped into blocks acting on at most k qubits; each block is multiplied out on the
// host in FP64 into one 2^k x 2^k complex matrix, written as the real 2^(k+1) square
// [[Re,-Im],[Im,Re]] interleaved by (index, re/im), split into a TF32 "hi" part and an
// FP32 "lo" remainder, and laid out in the tensor core's canonical K-major shared-memory
// format.  The kernel (kernels_fused.cu) applies a pass's blocks to a tile in shared
// memory with tcgen05 MMAs: D = X_hi G_hi^T + X_hi G_lo^T + X_lo G_hi^T.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>

#include "svb_internal.h"

namespace svb {
namespace {

using cplx = std::complex<double>;
inline uint64_t bit(int q) { return 1ull << q; }

uint64_t op_qubits(const EOp& e)
{
    return e.form == F_CX ? (bit(e.q) | bit(e.c)) : bit(e.q);
}

// Applies one elementary op to a 2^k complex vector whose bit i is global qubit tq[i].
void apply_small(const EOp& e, const int* pos_of_q, std::vector<cplx>& v)
{
    const size_t dim = v.size();
    const double S2I = 0.70710678118654752440;
    const double* m = e.m;
    if (e.form == F_CX) {
        const size_t cb = size_t(1) << pos_of_q[e.c], tb = size_t(1) << pos_of_q[e.q];
        for (size_t i = 0; i < dim; i++)
            if ((i & cb) && !(i & tb)) std::swap(v[i], v[i | tb]);
        return;
    }
    const size_t qb = size_t(1) << pos_of_q[e.q];
    for (size_t i = 0; i < dim; i++) {
        if (i & qb) continue;
        const cplx a0 = v[i], a1 = v[i | qb];
        cplx b0 = a0, b1 = a1;
        const cplx I(0, 1);
        switch (e.form) {
        case F_C1: b0 = cplx(m[0], m[1]) * a0 + cplx(m[2], m[3]) * a1;
                   b1 = cplx(m[4], m[5]) * a0 + cplx(m[6], m[7]) * a1; break;
        case F_X:  b0 = a1; b1 = a0; break;
        case F_Y:  b0 = -I * a1; b1 = I * a0; break;
        case F_H:  b0 = S2I * (a0 + a1); b1 = S2I * (a0 - a1); break;
        case F_W:  b0 = S2I * (a0 - I * a1); b1 = S2I * (-I * a0 + a1); break;
        case F_RX: b0 = m[0] * a0 + I * m[1] * a1; b1 = I * m[1] * a0 + m[0] * a1; break;
        case F_RY: b0 = m[0] * a0 + m[1] * a1; b1 = m[2] * a0 + m[3] * a1; break;
        case F_Z:  b1 = -a1; break;
        case F_S:  b1 = I * a1; break;
        case F_SDG: b1 = -I * a1; break;
        case F_T:  b1 = cplx(S2I, S2I) * a1; break;
        case F_TDG: b1 = cplx(S2I, -S2I) * a1; break;
        case F_R:  b1 = I * m[0] * a1; break;
        case F_U1: b1 = cplx(m[0], m[1]) * a1; break;
        case F_DIAG: b0 = cplx(m[0], m[1]) * a0; b1 = cplx(m[2], m[3]) * a1; break;
        default: break;   // F_SRN is rejected before fusion
        }
        v[i] = b0;
        v[i | qb] = b1;
    }
}

float tf32_hi(float x)
{
    // round to nearest (ties away) at 10 explicit mantissa bits
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u = (u + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// byte offset of element (row, kk) in the canonical K-major, no-swizzle layout with
// `rows` rows: 8-row x 16-byte core matrices, 128-byte row-group stride (SBO) and
// rows*16-byte K-chunk stride (LBO)
inline uint32_t kmajor_offset(uint32_t row, uint32_t kk, uint32_t rows)
{
    return (kk >> 2) * (rows * 16u) + (row >> 3) * 128u + (row & 7u) * 16u + (kk & 3u) * 4u;
}

}  // namespace

bool fusable(const std::vector<EOp>& ops)
{
    for (const EOp& e : ops)
        if (e.form == F_SRN) return false;
    return true;
}

void plan_fused(const std::vector<EOp>& ops, int n, int k, FusedPlan& plan)
{
    plan = FusedPlan{};
    plan.k = k;
    const int M = FT_TILE_BITS, G = FT_LOW_BITS;
    const int rows = 1 << (M - k);
    const int N = 1 << (k + 1);
    const size_t N_ops = ops.size();
    const uint64_t all = (n >= 64) ? ~0ull : (bit(n) - 1);
    std::vector<char> done(N_ops, 0);
    size_t first = 0;
    std::vector<int> taken, remaining, rest, blk;
    for (;;) {
        while (first < N_ops && done[first]) first++;
        if (first == N_ops) break;
        // -- local qubits of the pass: every qubit of an op must be local
        uint64_t L = (n == M) ? all : (bit(G) - 1);
        int nL = (n == M) ? n : G;
        uint64_t blocked = 0;
        taken.clear();
        for (size_t i = first; i < N_ops; i++) {
            if (done[i]) continue;
            const uint64_t t = op_qubits(ops[i]);
            if (t & blocked) { blocked |= t; if (blocked == all) break; continue; }
            const uint64_t need = t & ~L;
            const int add = __builtin_popcountll(need);
            if (nL + add > M) { blocked |= t; if (blocked == all) break; continue; }
            L |= need;
            nL += add;
            taken.push_back((int)i);
            done[i] = 1;
        }
        for (int q = 0; nL < M && q < n; q++)
            if (!((L >> q) & 1)) { L |= bit(q); nL++; }

        FusedPass P;
        std::memset(&P, 0, sizeof(P));
        int pos_of[64];
        for (int q = 0; q < 64; q++) pos_of[q] = -1;
        int nl = 0, nn = 0;
        for (int q = 0; q < n; q++) {
            if ((L >> q) & 1) { pos_of[q] = nl; P.local_q[nl++] = (uint8_t)q; }
            else P.nonlocal_q[nn++] = (uint8_t)q;
        }
        P.n_nonlocal = nn;
        for (int j = 0; j < 64; j++) {
            uint64_t lo = 0, hi = 0;
            for (int b = 0; b < 6; b++) {
                if ((j >> b) & 1) {
                    lo |= bit(P.local_q[b]);
                    hi |= bit(P.local_q[6 + b]);
                }
            }
            P.g_lo[j] = lo;
            P.g_hi[j] = hi;
        }
        P.block_begin = (int32_t)plan.blocks.size();

        // -- blocks: up to k qubits each, commuting ops pulled forward
        struct BlockOps { std::vector<int> tq; std::vector<int> ops; };
        std::vector<BlockOps> pblocks;
        remaining = taken;
        while (!remaining.empty() && (int)pblocks.size() < fused_max_blocks(k)) {
            uint64_t S = 0;
            uint64_t blk_blocked = 0;
            blk.clear();
            rest.clear();
            for (int i : remaining) {
                const uint64_t t = op_qubits(ops[i]);
                if (t & blk_blocked) { blk_blocked |= t; rest.push_back(i); continue; }
                if (__builtin_popcountll(S | t) <= k) {
                    S |= t;
                    blk.push_back(i);
                } else {
                    blk_blocked |= t;
                    rest.push_back(i);
                }
            }
            // targets: the block's qubits, padded with other local qubits to exactly k
            std::vector<int> tq;
            for (int q = 0; q < n; q++)
                if ((S >> q) & 1) tq.push_back(q);
            for (int p = 0; (int)tq.size() < k && p < M; p++) {
                const int q = P.local_q[p];
                if (!((S >> q) & 1)) { tq.push_back(q); S |= bit(q); }
            }
            pblocks.push_back({tq, blk});
            remaining.swap(rest);
        }
        const int nblocks = (int)pblocks.size();

        // Bit orderings.  The threads that write block f's operand have lane bits 0..3 on
        // the local positions W_f (the tile loader's positions 1..4 for f = 0, otherwise
        // row bits 0..3 of block f-1).  Their 8-byte stores are conflict-free when W_f lands
        // on {target bit 0, row bits 0..2} of block f, so those come first.
        std::vector<std::vector<int>> T(nblocks), C(nblocks);
        std::vector<int> W = {1, 2, 3, 4};
        for (int f = 0; f < nblocks; f++) {
            uint32_t tmask = 0;
            for (int q : pblocks[f].tq) tmask |= 1u << pos_of[q];
            std::vector<int>& t = T[f];
            std::vector<int>& c = C[f];
            for (int p : W)
                if (((tmask >> p) & 1) && t.empty()) t.push_back(p);
            for (int p = 0; p < M; p++)
                if (((tmask >> p) & 1) && std::find(t.begin(), t.end(), p) == t.end()) t.push_back(p);
            for (int p : W)
                if (!((tmask >> p) & 1)) c.push_back(p);
            for (int p = 0; p < M; p++)
                if (!((tmask >> p) & 1) && std::find(c.begin(), c.end(), p) == c.end()) c.push_back(p);
            W.assign(c.begin(), c.begin() + 4);
        }

        // per-block tables; offsets are additive over disjoint bit groups of the local index
        auto operand_word = [&](int f, uint32_t l) -> uint32_t {
            uint32_t row = 0, a = 0;
            for (int i = 0; i < k; i++)
                if ((l >> T[f][i]) & 1) a |= 1u << i;
            for (size_t i = 0; i < C[f].size(); i++)
                if ((l >> C[f][i]) & 1) row |= 1u << i;
            return kmajor_offset(row, 2 * a, rows) / 4;
        };
        std::vector<FusedBlock> fb(nblocks);
        for (int f = 0; f < nblocks; f++) {
            FusedBlock& B = fb[f];
            std::memset(&B, 0, sizeof(B));
            for (int a = 0; a < 64; a++) {
                uint32_t l = 0;
                for (int i = 0; i < k; i++)
                    if ((a >> i) & 1) l |= 1u << T[f][i];
                B.a_sc[a] = (uint16_t)(a < (1 << k) ? l : 0);
            }
            for (int j = 0; j < 32; j++) {
                uint32_t l = 0;
                for (int i = 0; i < 5 && i < (int)C[f].size(); i++)
                    if ((j >> i) & 1) l |= 1u << C[f][i];
                B.n_lo[j] = (uint16_t)l;
            }
            for (int j = 0; j < 16; j++) {
                uint32_t l = 0;
                for (int i = 0; i < 4 && 5 + i < (int)C[f].size(); i++)
                    if ((j >> i) & 1) l |= 1u << C[f][5 + i];
                B.n_hi[j] = (uint16_t)l;
            }
            for (int j = 0; j < 64; j++) {
                B.off_lo[j] = operand_word(f, (uint32_t)j);
                B.off_hi[j] = operand_word(f, (uint32_t)j << 6);
            }
        }
        for (int f = 0; f < nblocks; f++) {
            FusedBlock& B = fb[f];
            const bool last = (f == nblocks - 1);
            auto nxt = [&](uint32_t l) -> uint32_t { return last ? l : operand_word(f + 1, l); };
            for (int a = 0; a < 64; a++) B.nxt_a[a] = nxt(B.a_sc[a]);
            for (int j = 0; j < 32; j++) B.nxt_nlo[j] = nxt(B.n_lo[j]);
            for (int j = 0; j < 16; j++) B.nxt_nhi[j] = nxt(B.n_hi[j]);
        }

        // block matrices: gate operand B[m'][kk] for the real form, hi and lo planes
        for (int f = 0; f < nblocks; f++) {
            // qubit -> bit of the block's matrix index, in the order of T[f]
            int tpos[64];
            for (int q = 0; q < 64; q++) tpos[q] = -1;
            for (int i = 0; i < k; i++) tpos[P.local_q[T[f][i]]] = i;
            const int d = 1 << k;
            std::vector<cplx> U((size_t)d * d), col(d);
            for (int c = 0; c < d; c++) {
                std::fill(col.begin(), col.end(), cplx(0, 0));
                col[c] = 1.0;
                for (int i : pblocks[f].ops) apply_small(ops[i], tpos, col);
                for (int r = 0; r < d; r++) U[(size_t)r * d + c] = col[r];
            }
            FusedBlock& B = fb[f];
            const size_t plane = (size_t)N * N;
            B.gate_word = (uint32_t)plan.gates.size();
            plan.gates.resize(plan.gates.size() + 2 * plane);
            float* hi = plan.gates.data() + B.gate_word;
            float* lo = hi + plane;
            for (int mp = 0; mp < N; mp++) {
                const int ar = mp >> 1, cr = mp & 1;
                for (int kk = 0; kk < N; kk++) {
                    const int ac = kk >> 1, cc = kk & 1;
                    const cplx u = U[(size_t)ar * d + ac];
                    double val;
                    if (cr == 0) val = cc == 0 ? u.real() : -u.imag();
                    else val = cc == 0 ? u.imag() : u.real();
                    // hi = val to TF32, lo = the remainder to TF32 (both rounded to
                    // nearest, so the pair carries ~21 bits of the FP64 entry, unbiased)
                    const float h = tf32_hi((float)val);
                    const uint32_t w = kmajor_offset(mp, kk, N) / 4;
                    hi[w] = h;
                    lo[w] = tf32_hi((float)(val - (double)h));
                }
            }
            plan.blocks.push_back(B);
        }
        for (int i : remaining) done[i] = 0;   // did not fit in this pass's blocks
        P.n_blocks = nblocks;
        plan.passes.push_back(P);
    }
    (void)rows;
}

}  // namespace svb

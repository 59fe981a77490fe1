// Gate fusion for the fused tensor-core engine (FP32 states).
//
// The elementary-op stream (the reference's gate sequences, lower.cpp) is cut into
// passes over tiles of 2^FT_TILE_BITS amplitudes, as the staged engine does, except that
// every qubit an op touches must be local to the pass.  Inside a pass the ops are
// grouped into blocks acting on at most k qubits; each block is multiplied out on the
// host in FP64 into one 2^k x 2^k complex matrix, written as the real 2^(k+1) square
// [[Re,-Im],[Im,Re]] interleaved by (index, re/im), split into TF32 G_hi and G_lo (both
// rounded to nearest from the FP64 value) and stored as one 2N-row operand (G_hi rows,
// then G_lo rows) in the tensor core's canonical K-major shared-memory format.  The plan
// also fixes, per pass and block, the bit orders and the XOR-combined tables through which
// the kernel (kernels_fused.cu) moves a tile between blocks, chosen so that its
// shared-memory transposes are free of bank conflicts.
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

// seeds tried per block (the first open ops that can move to the front); fewer for the
// six-qubit blocks, whose passes are many (n = 30: 148 passes with 8 seeds, 146 with 32 at
// four times the planning time)
constexpr size_t kSeedWindow = 32;
constexpr size_t kSeedWindow6 = 8;

void plan_fused(const std::vector<EOp>& ops, int n, int k, FusedPlan& plan)
{
    plan = FusedPlan{};
    plan.k = k;
    const int M = FT_TILE_BITS, G = FT_LOW_BITS;
    const int N = 1 << (k + 1);
    const size_t N_ops = ops.size();
    const uint64_t all = (n >= 64) ? ~0ull : (bit(n) - 1);
    std::vector<char> done(N_ops, 0);
    size_t first = 0;
    std::vector<int> remaining, rest, blk;
    for (;;) {
        while (first < N_ops && done[first]) first++;
        if (first == N_ops) break;
        // -- the pass's blocks first, then its local qubits.  A block grows in program
        // order from a seed set of qubits over every op not yet placed: an op joins while
        // the block stays within k qubits, the pass within M local qubits (the G lowest
        // always among them), and none of its qubits is held by an op left out before it
        // (so the ops left out commute past the block).  Seeds: the first open op and each
        // of the next ones that could move to the front (no earlier open op shares a
        // qubit); the block that takes the most ops is kept.  Up to fused_max_blocks(k)
        // blocks per pass; the pass's local qubits are their union, padded from the lowest.
        // (n = 30, k = 5: 69 passes and 186 blocks, against 81 and 227 for a pass cut in
        // program order with blocks grown from the first op.)
        uint64_t L = (n == M) ? all : (bit(G) - 1);
        remaining.clear();
        for (size_t i = first; i < N_ops; i++)
            if (!done[i]) remaining.push_back((int)i);
        struct Grown { uint64_t S; std::vector<int> ops; };
        std::vector<Grown> grown;
        auto grow = [&](uint64_t S0, std::vector<int>& b, std::vector<int>& r) {
            uint64_t S = S0, held = 0;
            b.clear();
            r.clear();
            for (size_t x = 0; x < remaining.size(); x++) {
                const int i = remaining[x];
                const uint64_t t = op_qubits(ops[i]);
                if (!(t & held) && __builtin_popcountll(S | t) <= k && __builtin_popcountll(L | S | t) <= M) {
                    S |= t;
                    b.push_back(i);
                } else {
                    held |= t;
                    r.push_back(i);
                    if (held == all) {               // nothing later can join
                        r.insert(r.end(), remaining.begin() + (long)x + 1, remaining.end());
                        break;
                    }
                }
            }
            return S;
        };
        {
            std::vector<int> b2, r2;
            while ((int)grown.size() < fused_max_blocks(k) && !remaining.empty()) {
                uint64_t S = grow(0, blk, rest);
                uint64_t front = op_qubits(ops[remaining[0]]);
                for (size_t c = 1; c < remaining.size() && c < kSeedWindow; c++) {
                    const uint64_t t = op_qubits(ops[remaining[c]]);
                    if (t & front) { front |= t; continue; }
                    front |= t;
                    if (__builtin_popcountll(L | t) > M) continue;
                    const uint64_t S2 = grow(t, b2, r2);
                    if (b2.size() > blk.size()) {
                        blk.swap(b2);
                        rest.swap(r2);
                        S = S2;
                    }
                }
                if (blk.empty()) break;
                L |= S;
                for (int i : blk) done[i] = 1;
                grown.push_back({S, blk});
                remaining.swap(rest);
            }
        }
        int nL = __builtin_popcountll(L);
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

        // -- the blocks' targets: their qubits, padded with other local qubits to exactly k
        struct BlockOps { std::vector<int> tq; std::vector<int> ops; };
        std::vector<BlockOps> pblocks;
        for (const Grown& gb : grown) {
            uint64_t S = gb.S;
            std::vector<int> tq;
            for (int q = 0; q < n; q++)
                if ((S >> q) & 1) tq.push_back(q);
            for (int p = 0; (int)tq.size() < k && p < M; p++) {
                const int q = P.local_q[p];
                if (!((S >> q) & 1)) { tq.push_back(q); S |= bit(q); }
            }
            pblocks.push_back({tq, gb.ops});
        }
        const int nblocks = (int)pblocks.size();

        // Bit orderings, chosen so that the kernel's 8-byte shared-memory accesses are
        // conflict-free: the 16 lanes of a half warp (local positions = row bits 0..3 of
        // the accessing block) must land on 16 distinct bank pairs (word bits 0..3).
        //  * Block f > 0 is written from block f-1's rows: W = C[f-1][0..3] is matched onto
        //    the four bank-pair images of fused_slot (image i from target slot tslot[i] or
        //    row slot cslot[i]); a perfect matching always exists.
        //  * Block 0 is gathered from the raw tile and the last block writes the output
        //    stage; both layouts are chosen afterwards to fit (raw_xor, out_xor below).
        //    Block 0 puts position 0 (the only source of word bit 0 in the raw tile) on a
        //    row lane when it is a row.
        std::vector<std::vector<int>> T(nblocks), C(nblocks);
        const int tslot[4] = {0, 1, 2, k >= 4 ? 3 : -1};
        const int cslot[4] = {3, k >= 4 ? 0 : 1, k >= 4 ? 1 : 2, k >= 4 ? 2 : 0};
        for (int f = 0; f < nblocks; f++) {
            uint32_t tmask = 0;
            for (int q : pblocks[f].tq) tmask |= 1u << pos_of[q];
            auto is_target = [&](int p) { return ((tmask >> p) & 1) != 0; };
            std::vector<int>& t = T[f];
            std::vector<int>& c = C[f];
            t.assign(k, -1);
            c.assign(M - k, -1);
            std::vector<char> used(M, 0);
            if (f > 0) {
                const int* W = C[f - 1].data();
                int perm[4] = {0, 1, 2, 3}, best[4] = {0, 1, 2, 3}, best_ok = -1;
                do {
                    int good = 0;
                    for (int j = 0; j < 4; j++) good += !is_target(W[j]) || tslot[perm[j]] >= 0;
                    if (good > best_ok) {
                        best_ok = good;
                        std::copy(perm, perm + 4, best);
                    }
                } while (best_ok < 4 && std::next_permutation(perm, perm + 4));
                for (int j = 0; j < 4; j++) {
                    const int p = W[j], i = best[j];
                    if (is_target(p) && tslot[i] >= 0) { t[tslot[i]] = p; used[p] = 1; }
                    else if (!is_target(p)) { c[cslot[i]] = p; used[p] = 1; }
                }
            } else if (!is_target(0)) {
                c[0] = 0;
                used[0] = 1;
            }
            int ti = 0, ci = 0;
            for (int p = 0; p < M; p++) {
                if (used[p]) continue;
                if (is_target(p)) {
                    while (t[ti] >= 0) ti++;
                    t[ti] = p;
                } else {
                    while (c[ci] >= 0) ci++;
                    c[ci] = p;
                }
            }
        }

        // Raw-tile and output-stage layouts: each local position p >= 4 (a run bit) gets a
        // column of the run's XOR; positions 0..3 are fixed on word bits 0..3 (the raw
        // tile cannot swizzle bit 0: a 16-byte copy keeps its two amplitudes in order).
        // The columns of the accessing lanes' run-bit positions complete their fixed
        // columns to independent ones.
        auto choose_mix = [&](const std::vector<int>& lanes, uint32_t free_bits, uint8_t* col) {
            uint32_t have = 0;
            for (int j = 0; j < 4; j++)
                if (lanes[j] < 4) have |= 1u << lanes[j];
            for (int j = 0; j < 4; j++) {
                if (lanes[j] < 4) continue;
                for (int b = 0; b < 4; b++)
                    if (((free_bits >> b) & 1) && !((have >> b) & 1)) {
                        col[lanes[j] - 4] = (uint8_t)(1u << b);
                        have |= 1u << b;
                        break;
                    }
            }
        };
        uint8_t raw_col[8] = {0}, out_col[8] = {0};
        choose_mix(C[0], 0xEu, raw_col);
        choose_mix(C[nblocks - 1], 0xFu, out_col);
        for (int r = 0; r < 256; r++) {
            uint8_t rx = 0, ox = 0;
            for (int b = 0; b < 8; b++)
                if ((r >> b) & 1) { rx ^= raw_col[b]; ox ^= out_col[b]; }
            P.raw_xor[r] = (uint8_t)(rx >> 1);      // on the chunk index (word bits 1..3)
            P.out_xor[r] = ox;                      // on the word index (bits 0..3)
        }
        auto raw_word = [&](uint32_t l) { return l ^ ((uint32_t)P.raw_xor[l >> 4] << 1); };
        auto out_word = [&](uint32_t l) { return l ^ (uint32_t)P.out_xor[l >> 4]; };

        // per-block tables; the transpose slot is linear over GF(2) in the local index
        auto slot_of = [&](int f, uint32_t l) -> uint32_t {
            uint32_t row = 0, a = 0;
            for (int i = 0; i < k; i++)
                if ((l >> T[f][i]) & 1) a |= 1u << i;
            for (size_t i = 0; i < C[f].size(); i++)
                if ((l >> C[f][i]) & 1) row |= 1u << i;
            return fused_slot(row, a, k);
        };
        std::vector<FusedBlock> fb(nblocks);
        for (int f = 0; f < nblocks; f++) {
            FusedBlock& B = fb[f];
            std::memset(&B, 0, sizeof(B));
            const bool last = (f == nblocks - 1);
            // local index bits of a target index / row bit group, and where they go next
            auto place = [&](uint32_t l, uint16_t& raw, uint16_t& next) {
                raw = (uint16_t)raw_word(l);
                next = (uint16_t)(last ? out_word(l) : slot_of(f + 1, l));
            };
            for (int a = 0; a < 64; a++) {
                uint32_t l = 0;
                for (int i = 0; i < k; i++)
                    if ((a >> i) & 1) l |= 1u << T[f][i];
                if (a < (1 << k)) place(l, B.a_sc[a], B.nxt_a[a]);
            }
            for (int j = 0; j < 32; j++) {
                uint32_t l = 0;
                for (int i = 0; i < 5 && i < (int)C[f].size(); i++)
                    if ((j >> i) & 1) l |= 1u << C[f][i];
                place(l, B.n_lo[j], B.nxt_nlo[j]);
            }
            for (int j = 0; j < 16; j++) {
                uint32_t l = 0;
                for (int i = 0; i < 4 && 5 + i < (int)C[f].size(); i++)
                    if ((j >> i) & 1) l |= 1u << C[f][5 + i];
                place(l, B.n_hi[j], B.nxt_nhi[j]);
            }
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
            // the gate operand: G_hi in rows 0..N-1 and G_lo in rows N..2N-1 of one
            // K-major operand, so one MMA of width 2N forms X_hi G_hi and X_hi G_lo and
            // one of width N (rows 0..N-1) adds X_lo G_hi
            FusedBlock& B = fb[f];
            B.gate_word = (uint32_t)plan.gates.size();
            plan.gates.resize(plan.gates.size() + 2 * (size_t)N * N);
            float* gop = plan.gates.data() + B.gate_word;
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
                    gop[kmajor_offset(mp, kk, 2 * N) / 4] = h;
                    gop[kmajor_offset(N + mp, kk, 2 * N) / 4] = tf32_hi((float)(val - (double)h));
                }
            }
            plan.blocks.push_back(B);
        }
        P.n_blocks = nblocks;
        plan.passes.push_back(P);
    }
}

namespace {

// U[r][c] (row-major, 2^|tq| square) of the ops in `idx` on the qubits tq (bit i of the
// matrix index <-> qubit tq[i]), multiplied out in FP64 column by column
void block_unitary(const std::vector<EOp>& ops, const std::vector<int>& idx, const std::vector<int>& tq,
                   std::vector<cplx>& U)
{
    int pos_of[64];
    for (int q = 0; q < 64; q++) pos_of[q] = -1;
    for (size_t i = 0; i < tq.size(); i++) pos_of[tq[i]] = (int)i;
    const int d = 1 << (int)tq.size();
    U.assign((size_t)d * d, cplx(0, 0));
    std::vector<cplx> col(d);
    for (int c = 0; c < d; c++) {
        std::fill(col.begin(), col.end(), cplx(0, 0));
        col[c] = 1.0;
        for (int i : idx) apply_small(ops[i], pos_of, col);
        for (int r = 0; r < d; r++) U[(size_t)r * d + c] = col[r];
    }
}

}  // namespace

// Fusion width 6: the op stream is cut greedily into blocks of at most 6 qubits (an op
// joins the current block when it touches no qubit of an op left out before it and the
// union stays within 6 qubits; ops on disjoint qubits commute, so later ops may be pulled
// forward past those left out).  Each block is one pass over tiles of 4,096 amplitudes:
// its 6 target qubits (padded with high qubits when it has fewer) and the 6 lowest other
// qubits as row bits, so a tile always holds qubits 0 and 1 (whole 32-byte sectors).
//
// The kernel (kernels_fused6.cu) moves amplitude x = thread + 512 i (i < 8) of a tile;
// the planner maps the 12 bits of x onto local qubits so that the 16 threads of a half
// warp hit 16 distinct bank pairs of the B-operand plane: x bits 0 and 1 are qubits 0 and
// 1 (the two lowest local qubits), and x bits 2 and 3 are chosen to complete the four
// low word-offset bits, which come from target bit 0 (+1 word) and row bits 0..2 (+2, +4,
// +8 words) of the canonical K-major layout.  When qubits 0 and 1 are both targets two
// of the half warp's words share a bank pair (a 2-way conflict).
void plan_fused6(const std::vector<EOp>& ops, int n, FusedPlan& plan)
{
    plan = FusedPlan{};
    plan.k = F6_K;
    const size_t N_ops = ops.size();
    const uint64_t all = (n >= 64) ? ~0ull : (bit(n) - 1);
    std::vector<char> done(N_ops, 0);
    size_t first = 0;
    std::vector<int> blk;
    std::vector<cplx> U;
    for (;;) {
        while (first < N_ops && done[first]) first++;
        if (first == N_ops) break;
        // the block grown from a seed set (as in plan_fused), best of the front-movable seeds
        auto grow6 = [&](uint64_t S0, std::vector<int>& b) {
            uint64_t S = S0, blocked = 0;
            b.clear();
            for (size_t i = first; i < N_ops; i++) {
                if (done[i]) continue;
                const uint64_t t = op_qubits(ops[i]);
                if ((t & blocked) || __builtin_popcountll(S | t) > F6_K) {
                    blocked |= t;
                    if (blocked == all) break;
                    continue;
                }
                S |= t;
                b.push_back((int)i);
            }
            return S;
        };
        uint64_t S = grow6(0, blk);
        {
            std::vector<int> blk2;
            uint64_t front = 0;
            size_t seen = 0;
            for (size_t i = first; i < N_ops && seen < kSeedWindow6; i++) {
                if (done[i]) continue;
                seen++;
                const uint64_t t = op_qubits(ops[i]);
                if (t & front) { front |= t; continue; }
                front |= t;
                if (seen == 1) continue;
                const uint64_t S2 = grow6(t, blk2);
                if (blk2.size() > blk.size()) {
                    blk.swap(blk2);
                    S = S2;
                }
            }
        }
        for (int i : blk) done[i] = 1;
        // targets: the block's qubits, padded from the top; rows: the 6 lowest others
        uint64_t T = S;
        for (int q = n - 1; q >= 0 && __builtin_popcountll(T) < F6_K; q--) T |= bit(q);
        uint64_t R = 0;
        for (int q = 0; q < n && __builtin_popcountll(R) < F6_TILE_BITS - F6_K; q++)
            if (!((T >> q) & 1)) R |= bit(q);
        const uint64_t L = T | R;

        Fused6Pass P;
        std::memset(&P, 0, sizeof(P));
        int nl = 0, nn = 0;
        for (int q = 0; q < n; q++) {
            if ((L >> q) & 1) P.local_q[nl++] = (uint8_t)q;
            else P.nonlocal_q[nn++] = (uint8_t)q;
        }
        P.n_nonlocal = nn;

        // roles: target bit order tq (bit i of a <-> tq[i]) and row bit order rq
        std::vector<int> tq, rq;
        const int q0 = P.local_q[0], q1 = P.local_q[1];
        const bool t0 = (T >> q0) & 1, t1 = (T >> q1) & 1;
        int xq2 = -1, xq3 = -1;            // the qubits of x bits 2 and 3
        auto first_of = [&](uint64_t set, uint64_t skip) {
            for (int i = 2; i < F6_TILE_BITS; i++) {
                const int q = P.local_q[i];
                if (((set >> q) & 1) && !((skip >> q) & 1)) return q;
            }
            return -1;
        };
        if (!t0 && !t1) {                  // rows 0, 1 <- q0, q1; x2 -> target bit 0, x3 -> row 2
            rq = {q0, q1};
            xq2 = first_of(T, 0);
            xq3 = first_of(R, 0);
            tq = {xq2};
            rq.push_back(xq3);
        } else if (t0 != t1) {             // target bit 0 and row 0 <- q0, q1; x2, x3 -> rows 1, 2
            const int qt = t0 ? q0 : q1, qr = t0 ? q1 : q0;
            tq = {qt};
            rq = {qr};
            xq2 = first_of(R, 0);
            xq3 = first_of(R, bit(xq2));
            rq.push_back(xq2);
            rq.push_back(xq3);
        } else {                           // both targets: 2-way; x2, x3 -> rows 0, 1
            tq = {q0, q1};
            xq2 = first_of(R, 0);
            xq3 = first_of(R, bit(xq2));
            rq = {xq2, xq3};
        }
        for (int i = 0; i < F6_TILE_BITS; i++) {
            const int q = P.local_q[i];
            const bool in_t = std::find(tq.begin(), tq.end(), q) != tq.end();
            const bool in_r = std::find(rq.begin(), rq.end(), q) != rq.end();
            if (in_t || in_r) continue;
            if ((T >> q) & 1) tq.push_back(q);
            else rq.push_back(q);
        }
        // x bits -> qubits: 0, 1 -> q0, q1; 2, 3 -> xq2, xq3; the rest ascending
        int xq[F6_TILE_BITS];
        xq[0] = q0;
        xq[1] = q1;
        xq[2] = xq2;
        xq[3] = xq3;
        for (int i = 2, j = 4; i < F6_TILE_BITS; i++) {
            const int q = P.local_q[i];
            if (q != xq2 && q != xq3) xq[j++] = q;
        }
        // word offset of a qubit's bit in the B-operand plane: target bit b -> 1 (b = 0)
        // or 128 << (b - 1); row bit b -> 2 << b
        auto word_of = [&](int q) -> uint32_t {
            for (int b = 0; b < F6_K; b++)
                if (tq[b] == q) return b == 0 ? 1u : (128u << (b - 1));
            for (int b = 0; b < F6_TILE_BITS - F6_K; b++)
                if (rq[b] == q) return 2u << b;
            return 0u;
        };
        for (int j = 0; j < 64; j++) {
            uint64_t glo = 0, ghi = 0;
            uint32_t slo = 0, shi = 0;
            for (int b = 0; b < 6; b++) {
                if ((j >> b) & 1) {
                    glo |= bit(xq[b]);
                    ghi |= bit(xq[6 + b]);
                    slo += word_of(xq[b]);
                    shi += word_of(xq[6 + b]);
                }
            }
            P.g_lo[j] = glo;
            P.g_hi[j] = ghi;
            P.s_lo[j] = (uint16_t)slo;
            P.s_hi[j] = (uint16_t)shi;
            uint64_t orow = 0, otgt = 0;
            for (int b = 0; b < 6; b++) {
                if ((j >> b) & 1) {
                    orow |= bit(rq[b]);
                    otgt |= bit(tq[b]);
                }
            }
            P.o_row[j] = orow;
            P.o_tgt[j] = otgt;
        }
        P.rows_paired = (P.o_row[1] == 1) ? 1 : 0;   // row bit 0 is qubit 0

        // the real form G[m'][kk] (m' = 2a' + c', kk = 2a + c) of the block's matrix,
        // row-major, hi plane then lo plane (both rounded to nearest TF32)
        block_unitary(ops, blk, tq, U);
        P.gate_word = (uint32_t)plan.gates.size();
        plan.gates.resize(plan.gates.size() + 2 * (size_t)F6_N * F6_N);
        float* gh = plan.gates.data() + P.gate_word;
        float* gl = gh + (size_t)F6_N * F6_N;
        const int d = 1 << F6_K;
        for (int mp = 0; mp < F6_N; mp++) {
            const int ar = mp >> 1, cr = mp & 1;
            for (int kk = 0; kk < F6_N; kk++) {
                const int ac = kk >> 1, cc = kk & 1;
                const cplx u = U[(size_t)ar * d + ac];
                double val;
                if (cr == 0) val = cc == 0 ? u.real() : -u.imag();
                else val = cc == 0 ? u.imag() : u.real();
                const float h = tf32_hi((float)val);
                gh[(size_t)mp * F6_N + kk] = h;
                gl[(size_t)mp * F6_N + kk] = tf32_hi((float)(val - (double)h));
            }
        }
        plan.passes6.push_back(P);
    }
}

}  // namespace svb

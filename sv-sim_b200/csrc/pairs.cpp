// Planner of the pair engine (FP64 two-qubit blocks on the FP64 tensor cores).
//
// Passes are cut exactly as for the staged engine (select_passes).  Inside a pass the
// elementary ops, in program order, are folded into two-qubit blocks:
//   * a one-qubit op (dense or diagonal) on a local qubit p is multiplied into pend[p],
//     a pending 2x2 matrix, and applied with the next block that touches p;
//   * a CX on two local qubits (c, t) closes pend[c] and pend[t] into one block,
//     CX . (pend[c] (x) pend[t]);
//   * a CX whose control is not local is an X on t for the tiles where that qubit is 1:
//     pend[t] gets a variant per value of the control (a condition qubit);
//   * a diagonal op on a non-local qubit is a phase for the tiles where that qubit is 1
//     (or 0, for the general diagonal): it is folded into a block as a scalar variant.
// Blocks on other qubits commute with a pending one-qubit matrix, so deferring it keeps
// the circuit's meaning; blocks that share a qubit keep their program order, and blocks on
// disjoint pairs are taken in the order that needs the fewest moves.  At the end of the pass
// a pending matrix without conditions on qubit q moves into the next pass that acts on q
// when q is local there (nothing in between acts on q); the others are closed in pairs.
// (n=30 depth 40: 540 blocks instead of 654, of which 285 were such closures.)  A block
// carries at most PR_MAX_COND condition qubits (4 variants); merges that would exceed it
// close the pending matrix first.
//
// Each block needs its two qubits on lane bits 0 and 1.  The layout planner follows the
// blocks: a qubit held in a register bit is swapped onto a lane with one warp shuffle
// exchange (PO_SWAP: selects around the shuffles), qubits on other lanes are brought to
// lanes 0 and 1 by one permutation of the lane bits (PO_LPERM: one indexed shuffle per
// word, no selects), and a qubit on a warp bit needs a shared-memory redistribution
// (PO_RELAYOUT) whose new layout keeps the soonest-needed qubits on lanes and registers.  A pass is loaded and
// stored with its 2 lowest local positions (qubits 0 and 1) on lanes, which makes every
// warp access whole 64-byte runs; the load puts the first block's qubits on lanes 0 and 1
// and the next-needed qubits on the free lanes, then in registers.
//
// The device form of a block variant is its real 8x8 matrix G'[r][kk] with rows
// r = 2a' + re/im of the output amplitude and columns kk = a (real part) or 4 + a
// (imaginary part) of the input amplitude, stored as 32 lanes x (G'[t>>2][t&3],
// G'[t>>2][4 + (t&3)]): the B fragments of the two k-steps of the MMA D^T = X^T G'^T.
#include <algorithm>
#include <array>
#include <complex>
#include <cstring>
#include <system_error>
#include <thread>

#include "gate_math.cuh"

namespace svb {
namespace {

using cplx = std::complex<double>;
using M2 = std::array<cplx, 4>;     // row-major 2x2
using M4 = std::array<cplx, 16>;    // row-major 4x4, index a = bit0 + 2 bit1

constexpr int NSLOT = PR_TILE_BITS;  // 0..4 lanes, 5..8 registers, 9..11 warps
constexpr int SLOT_REG = PR_LANE_BITS;
constexpr int SLOT_WARP = PR_LANE_BITS + RB;

M2 ident2() { return M2{cplx(1), cplx(0), cplx(0), cplx(1)}; }
M4 ident4()
{
    M4 m{};
    for (int i = 0; i < 4; i++) m[i * 5] = 1;
    return m;
}
M2 mul2(const M2& a, const M2& b)
{
    M2 r{};
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) r[i * 2 + j] = a[i * 2] * b[j] + a[i * 2 + 1] * b[2 + j];
    return r;
}
M4 mul4(const M4& a, const M4& b)
{
    M4 r{};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            cplx s = 0;
            for (int k = 0; k < 4; k++) s += a[i * 4 + k] * b[k * 4 + j];
            r[i * 4 + j] = s;
        }
    return r;
}
// P0 on bit 0, P1 on bit 1
M4 kron(const M2& p0, const M2& p1)
{
    M4 r{};
    for (int ap = 0; ap < 4; ap++)
        for (int a = 0; a < 4; a++)
            r[ap * 4 + a] = p0[(ap & 1) * 2 + (a & 1)] * p1[(ap >> 1) * 2 + (a >> 1)];
    return r;
}
// the same operator with the roles of bit 0 and bit 1 exchanged
M4 swap_bits(const M4& m)
{
    auto s = [](int a) { return ((a & 1) << 1) | (a >> 1); };
    M4 r{};
    for (int ap = 0; ap < 4; ap++)
        for (int a = 0; a < 4; a++) r[s(ap) * 4 + s(a)] = m[ap * 4 + a];
    return r;
}

// 2x2 matrix of an elementary op, read off the kernels' own expressions on the basis
M2 matrix_of(const EOp& e)
{
    const Coef<double> c = load_coef<double>(e.m);
    M2 u{};
    for (int col = 0; col < 2; col++) {
        double2 a0 = make_double2(col == 0 ? 1.0 : 0.0, 0.0), a1 = make_double2(col == 1 ? 1.0 : 0.0, 0.0);
        if (form_is_diag(e.form)) {
            diag_one<double>(e.form, c, a1);
            if (e.form == F_DIAG) diag_zero<double>(e.form, c, a0);
        } else {
            dense_pair<double>(e.form, c, a0, a1);
        }
        u[col] = cplx(a0.x, a0.y);
        u[2 + col] = cplx(a1.x, a1.y);
    }
    return u;
}

// condition qubits -> variants (variant index bit i = value of cond[i] in the tile)
std::vector<int> cond_union(const std::vector<int>& a, const std::vector<int>& b)
{
    std::vector<int> u = a;
    for (int q : b)
        if (std::find(u.begin(), u.end(), q) == u.end()) u.push_back(q);
    return u;
}
int sub_index(const std::vector<int>& uni, int u, const std::vector<int>& sub)
{
    int r = 0;
    for (size_t i = 0; i < sub.size(); i++) {
        const int j = (int)(std::find(uni.begin(), uni.end(), sub[i]) - uni.begin());
        r |= ((u >> j) & 1) << i;
    }
    return r;
}

struct Pend {                       // conditional 2x2 on one local position
    bool active = false;
    std::vector<int> cond;
    std::vector<M2> v{ident2()};
};
struct Scalar {                     // conditional phase of the whole tile
    bool active = false;
    std::vector<int> cond;
    std::vector<cplx> v{cplx(1)};
};
struct Block {
    int x, y;                        // local positions: bit 0 = x, bit 1 = y
    std::vector<int> cond;
    std::vector<M4> v;
};

// pend = u(cond) . pend
void pend_apply(Pend& p, const std::vector<int>& ucond, const std::vector<M2>& uv)
{
    const std::vector<int> uni = cond_union(p.cond, ucond);
    std::vector<M2> nv((size_t)1 << uni.size());
    for (size_t u = 0; u < nv.size(); u++)
        nv[u] = mul2(uv[sub_index(uni, (int)u, ucond)], p.v[sub_index(uni, (int)u, p.cond)]);
    p.cond = uni;
    p.v = nv;
    p.active = true;
}

struct PassPairs {
    std::vector<Block> blocks;
    Pend pend[NSLOT];
    Scalar ph;
    bool no_merge = false;           // set while a close must emit the pending tile phase

    // after . (pend[x] (x) pend[y]) folded into the last block when that block acts on the
    // same two positions: every op on x or y since that block is pending here (a
    // two-qubit op on either would have made a later block), so the product is that
    // block followed by this one.  A density-matrix gate and its noise channel on
    // (q, q + n), or CX . U1 . CX on one pair, become one block instead of two.
    bool merge_last(int x, int y, const M4* after)
    {
        if (blocks.empty() || no_merge) return false;
        Block& L = blocks.back();
        const bool same = L.x == x && L.y == y, swapped = L.x == y && L.y == x;
        if (!same && !swapped) return false;
        const std::vector<int> cond = cond_union(L.cond, cond_union(pend[x].cond, pend[y].cond));
        if (cond.size() > (size_t)PR_MAX_COND) return false;
        std::vector<M4> nv((size_t)1 << cond.size());
        for (size_t u = 0; u < nv.size(); u++) {
            M4 m = kron(pend[x].v[sub_index(cond, (int)u, pend[x].cond)],
                        pend[y].v[sub_index(cond, (int)u, pend[y].cond)]);
            if (after) m = mul4(*after, m);
            if (swapped) m = swap_bits(m);         // into the last block's bit order
            nv[u] = mul4(m, L.v[sub_index(cond, (int)u, L.cond)]);
        }
        L.cond = cond;
        L.v = nv;
        pend[x] = Pend{};
        pend[y] = Pend{};
        return true;
    }
    // block = after . (pend[x] (x) pend[y]), plus the pending tile phase when it fits
    void close(int x, int y, const M4* after)
    {
        if (merge_last(x, y, after)) return;
        Block b;
        b.x = x;
        b.y = y;
        b.cond = cond_union(pend[x].cond, pend[y].cond);
        const bool with_ph = ph.active && cond_union(b.cond, ph.cond).size() <= (size_t)PR_MAX_COND;
        if (with_ph) b.cond = cond_union(b.cond, ph.cond);
        b.v.resize((size_t)1 << b.cond.size());
        for (size_t u = 0; u < b.v.size(); u++) {
            M4 m = kron(pend[x].v[sub_index(b.cond, (int)u, pend[x].cond)],
                        pend[y].v[sub_index(b.cond, (int)u, pend[y].cond)]);
            if (after) m = mul4(*after, m);
            if (with_ph) {
                const cplx s = ph.v[sub_index(b.cond, (int)u, ph.cond)];
                for (auto& z : m) z *= s;
            }
            b.v[u] = m;
        }
        if (with_ph) ph = Scalar{};
        pend[x] = Pend{};
        pend[y] = Pend{};
        blocks.push_back(b);
    }
    int partner_of(int p) const { return p == 0 ? 1 : 0; }
    // closes pend[p] alone (with an idle partner)
    void flush(int p)
    {
        int q = partner_of(p);
        for (int k = 0; k < NSLOT; k++)
            if (k != p && !pend[k].active) { q = k; break; }
        if (pend[q].active && cond_union(pend[p].cond, pend[q].cond).size() > (size_t)PR_MAX_COND) {
            Pend keep = pend[q];
            pend[q] = Pend{};
            close(p, q, nullptr);
            pend[q] = keep;
        } else {
            close(p, q, nullptr);
        }
    }
    void add_1q(int p, const std::vector<int>& ucond, const std::vector<M2>& uv)
    {
        if (cond_union(pend[p].cond, ucond).size() > (size_t)PR_MAX_COND) flush(p);
        pend_apply(pend[p], ucond, uv);
    }
    void add_phase(int q, const cplx& f0, const cplx& f1)
    {
        if (ph.active && cond_union(ph.cond, {q}).size() > (size_t)PR_MAX_COND) {
            // close the tile phase on its own before it outgrows a block
            Pend a = pend[0], b = pend[1];
            pend[0] = Pend{};
            pend[1] = Pend{};
            no_merge = true;           // a block of its own, which takes the phase
            close(0, 1, nullptr);
            no_merge = false;
            pend[0] = a;
            pend[1] = b;
        }
        const std::vector<int> uni = cond_union(ph.cond, {q});
        std::vector<cplx> nv((size_t)1 << uni.size());
        for (size_t u = 0; u < nv.size(); u++) {
            const int bitq = sub_index(uni, (int)u, {q});
            nv[u] = ph.v[sub_index(uni, (int)u, ph.cond)] * (bitq ? f1 : f0);
        }
        ph.cond = uni;
        ph.v = nv;
        ph.active = true;
    }
    // a general two-qubit matrix on (a: bit 0, b: bit 1)
    void add_m4(int a, int b, const M4& m)
    {
        if (cond_union(pend[a].cond, pend[b].cond).size() > (size_t)PR_MAX_COND) flush(a);
        close(a, b, &m);
    }
    void add_cx(int c, int t)
    {
        if (cond_union(pend[c].cond, pend[t].cond).size() > (size_t)PR_MAX_COND) flush(c);
        M4 cx{};
        for (int a = 0; a < 4; a++) {
            const int ap = (a & 1) ? (a ^ 2) : a;     // bit 0 = control, bit 1 = target
            cx[ap * 4 + a] = 1;
        }
        close(c, t, &cx);
    }
    void finish()
    {
        // pair the open matrices two by two: those with the most condition qubits first,
        // each with the first partner that keeps the union within PR_MAX_COND
        std::vector<int> open;
        for (int p = 0; p < NSLOT; p++)
            if (pend[p].active) open.push_back(p);
        std::stable_sort(open.begin(), open.end(),
                         [&](int a, int b) { return pend[a].cond.size() > pend[b].cond.size(); });
        std::vector<char> used(open.size(), 0);
        for (size_t i = 0; i < open.size(); i++) {
            if (used[i]) continue;
            used[i] = 1;
            size_t j = i + 1;
            while (j < open.size() &&
                   (used[j] || cond_union(pend[open[i]].cond, pend[open[j]].cond).size() > (size_t)PR_MAX_COND))
                j++;
            if (j < open.size()) {
                used[j] = 1;
                close(open[i], open[j], nullptr);
            } else {
                flush(open[i]);
            }
        }
        if (ph.active) {               // pend[0] is idle here: a block with only the phase
            no_merge = true;
            flush(0);
            no_merge = false;
        }
    }
};

struct LayoutPlanner {
    PairPlan& plan;
    int slot_pos[NSLOT];
    int where[NSLOT];
    bool dry = false;                // only follow the layout (for trying block orders)

    DevStage stage() const
    {
        DevStage st;
        std::memset(&st, 0, sizeof(st));
        for (int i = 0; i < RB; i++) st.reg_pos[i] = (uint8_t)slot_pos[SLOT_REG + i];
        for (int b = 0; b < PR_LANE_BITS; b++) st.thr_pos[b] = (uint8_t)slot_pos[b];
        for (int w = 0; w < NSLOT - SLOT_WARP; w++) st.thr_pos[PR_LANE_BITS + w] = (uint8_t)slot_pos[SLOT_WARP + w];
        return st;
    }
    int push_layout()
    {
        plan.layouts.push_back(stage());
        return (int)plan.layouts.size() - 1;
    }
    void set(const int* sp)
    {
        for (int s = 0; s < NSLOT; s++) {
            slot_pos[s] = sp[s];
            where[sp[s]] = s;
        }
    }
    void swap_lr(int lane, int reg)
    {
        if (!dry) {
            PairOp op;
            std::memset(&op, 0, sizeof(op));
            op.kind = PO_SWAP;
            op.lane = (uint8_t)lane;
            op.reg = (uint8_t)reg;
            plan.ops.push_back(op);
            plan.n_swaps++;
        }
        const int a = slot_pos[lane], b = slot_pos[SLOT_REG + reg];
        slot_pos[lane] = b;
        slot_pos[SLOT_REG + reg] = a;
        where[b] = lane;
        where[a] = SLOT_REG + reg;
    }
    void relayout(const int* sp)
    {
        if (dry) {
            set(sp);
            return;
        }
        PairOp op;
        std::memset(&op, 0, sizeof(op));
        op.kind = PO_RELAYOUT;
        op.src = (uint16_t)push_layout();
        set(sp);
        op.layout = (uint16_t)push_layout();
        plan.ops.push_back(op);
        plan.n_relayouts++;
    }
    // one permutation of the lane bits: lane bit b receives what lane bit from[b] held
    void lane_perm(const int* from)
    {
        int old[PR_LANE_BITS];
        for (int b = 0; b < PR_LANE_BITS; b++) old[b] = slot_pos[b];
        uint32_t code = 0;
        for (int b = 0; b < PR_LANE_BITS; b++) {
            code |= (uint32_t)from[b] << (3 * b);
            slot_pos[b] = old[from[b]];
            where[slot_pos[b]] = b;
        }
        if (!dry) {
            PairOp op;
            std::memset(&op, 0, sizeof(op));
            op.kind = PO_LPERM;
            op.gate = code;
            plan.ops.push_back(op);
            plan.n_lane_perms++;
        }
    }
    // the lane (other than those holding x and y) whose qubit is needed last
    int spare_lane(int x, int y, int pref, const std::vector<int>& next_use) const
    {
        if (slot_pos[pref] != x && slot_pos[pref] != y) return pref;
        int best = -1;
        for (int l = 0; l < PR_LANE_BITS; l++) {
            if (slot_pos[l] == x || slot_pos[l] == y) continue;
            if (best < 0 || next_use[slot_pos[l]] > next_use[slot_pos[best]]) best = l;
        }
        return best;
    }
    // a layout with x, y on lanes 0, 1 and the other positions by next use
    void relayout_for(int x, int y, const std::vector<int>& next_use)
    {
        std::vector<int> rest;
        for (int p = 0; p < NSLOT; p++)
            if (p != x && p != y) rest.push_back(p);
        std::stable_sort(rest.begin(), rest.end(), [&](int a, int b) { return next_use[a] < next_use[b]; });
        int sp[NSLOT];
        sp[0] = x;
        sp[1] = y;
        // lane 2: the soonest-needed position whose residue mod 3 differs from x's and y's,
        // so the three lowest lane bits hit distinct swizzle groups (conflict-free
        // shared-memory phases); the rest by next use.  (Taking it from the latest-needed
        // end instead left a lane slot to a qubit not needed for long: n = 30, 937 ms
        // against 904 ms.)
        int l2 = -1;
        for (int i = 0; i < (int)rest.size() && l2 < 0; i++)
            if (rest[i] % 3 != x % 3 && rest[i] % 3 != y % 3) l2 = i;
        if (l2 < 0) l2 = 0;
        sp[2] = rest[l2];
        rest.erase(rest.begin() + l2);
        // soonest-needed on lanes 3..4 (one lane permutation away, both at once), then the
        // registers (one exchange each), warps last
        int k = 0;
        for (int l = 3; l < PR_LANE_BITS; l++) sp[l] = rest[k++];
        for (int r = 0; r < RB; r++) sp[SLOT_REG + r] = rest[k++];
        for (int w = SLOT_WARP; w < NSLOT; w++) sp[w] = rest[k++];
        relayout(sp);
    }
    // cost of bringing x and y to lanes 0 and 1, in units of about one lane permutation:
    // a lane/register exchange is four, a relayout fourteen
    int pair_cost(int x, int y) const
    {
        const int sx = where[x], sy = where[y];
        if ((sx == 0 && sy == 1) || (sx == 1 && sy == 0)) return 0;
        if (sx >= SLOT_WARP || sy >= SLOT_WARP) return 14;
        int c = 0;
        bool perm = false;
        for (int s : {sx, sy}) {
            if (s >= SLOT_REG) c += 4;
            else if (s > 1) perm = true;
        }
        return c + (perm ? 1 : 0);
    }
    void ensure(int x, int y, const std::vector<int>& next_use)
    {
        const int sx = where[x], sy = where[y];
        if ((sx == 0 && sy == 1) || (sx == 1 && sy == 0)) return;
        if (sx >= SLOT_WARP || sy >= SLOT_WARP) {
            relayout_for(x, y, next_use);
            return;
        }
        // qubits in registers onto lanes (lane 0 for x, lane 1 for y, where free)
        if (where[x] >= SLOT_REG) swap_lr(spare_lane(x, y, 0, next_use), where[x] - SLOT_REG);
        if (where[y] >= SLOT_REG) swap_lr(spare_lane(x, y, 1, next_use), where[y] - SLOT_REG);
        const int lx = where[x], ly = where[y];
        if ((lx == 0 && ly == 1) || (lx == 1 && ly == 0)) return;
        // then one lane permutation: a qubit already on lane 0 or 1 stays there
        int tx = 0, ty = 1;
        if (lx <= 1) { tx = lx; ty = 1 - lx; }
        else if (ly <= 1) { ty = ly; tx = 1 - ly; }
        int cur[PR_LANE_BITS];                  // cur[b]: the old lane bit now on lane bit b
        for (int b = 0; b < PR_LANE_BITS; b++) cur[b] = b;
        auto exch = [&](int a, int b) { std::swap(cur[a], cur[b]); };
        auto lane_of = [&](int old) { for (int b = 0; b < PR_LANE_BITS; b++) if (cur[b] == old) return b; return -1; };
        if (lx != tx) exch(tx, lane_of(lx));
        if (lane_of(ly) != ty) exch(ty, lane_of(ly));
        // lane 2: a qubit whose position differs mod 3 from x's and y's, when lanes 2..4
        // hold one, so that a later relayout's shared-memory phases start conflict-free
        auto clash = [&](int b) { const int r = slot_pos[cur[b]] % 3; return r == x % 3 || r == y % 3; };
        for (int b = 3; b < PR_LANE_BITS && clash(2); b++)
            if (!clash(b)) exch(2, b);
        lane_perm(cur);
    }
};

void write_block(PairPlan& plan, const Block& b, bool transposed)
{
    for (const M4& m0 : b.v) {
        const M4 m = transposed ? swap_bits(m0) : m0;
        double g[8][8];
        for (int ap = 0; ap < 4; ap++)
            for (int a = 0; a < 4; a++) {
                const cplx z = m[ap * 4 + a];
                g[2 * ap][a] = z.real();
                g[2 * ap + 1][a] = z.imag();
                g[2 * ap][4 + a] = -z.imag();
                g[2 * ap + 1][4 + a] = z.real();
            }
        for (int t = 0; t < 32; t++) {
            plan.gates.push_back(g[t >> 2][t & 3]);
            plan.gates.push_back(g[t >> 2][4 + (t & 3)]);
        }
    }
}

}  // namespace

namespace {

bool plan_pairs_cut(const std::vector<EOp>& ops, int n, PairPlan& plan, const std::vector<Mat4>* mats, int seeds)
{
    plan = PairPlan{};
    if (n < PR_TILE_BITS) return false;
    for (const EOp& e : ops) {
        if (e.form == F_SRN) return false;      // only real-linear: not a matrix
        if (e.form == F_M4 && (!mats || e.mat < 0 || (size_t)e.mat >= mats->size())) return false;
    }
    // the pass cut first (every op of a pass is placed, so nothing is handed back), then
    // the passes in order, knowing which later pass next touches each qubit
    std::vector<std::pair<uint64_t, std::vector<int>>> cuts;
    select_passes(
        ops, n, PR_TILE_BITS, PR_COAL_BITS,
        [&](uint64_t L, const std::vector<int>& taken) {
            cuts.push_back({L, taken});
            return std::vector<int>{};
        },
        seeds);
    std::vector<uint64_t> touch(cuts.size(), 0);
    for (size_t ci = 0; ci < cuts.size(); ci++)
        for (int i : cuts[ci].second) {
            const EOp& e = ops[i];
            touch[ci] |= 1ull << e.q;
            if (e.form == F_CX || e.form == F_M4) touch[ci] |= 1ull << e.c;
        }
    // A one-qubit matrix still pending on qubit q at the end of a pass is carried into
    // the next pass that touches q when q is local there (no pass in between acts on q,
    // so the deferral keeps the circuit's meaning); it then folds into that pass's next
    // block on q instead of costing a block of its own.
    std::vector<M2> carry(64);
    std::vector<char> has_carry(64, 0);
    for (size_t ci = 0; ci < cuts.size(); ci++) {
        const uint64_t L = cuts[ci].first;
        const std::vector<int>& taken = cuts[ci].second;
        PairPass P;
        std::memset(&P, 0, sizeof(P));
        int pos_of[64];
        for (int q = 0; q < 64; q++) pos_of[q] = -1;
        int nl = 0, nn = 0;
        for (int q = 0; q < n; q++) {
            if ((L >> q) & 1) { pos_of[q] = nl; P.local_q[nl++] = (uint8_t)q; }
            else P.nonlocal_q[nn++] = (uint8_t)q;
        }
        P.n_nonlocal = nn;
        // 1. blocks
        PassPairs pp;
        for (int q = 0; q < n; q++)
            if (has_carry[q] && ((touch[ci] >> q) & 1)) {
                pp.pend[pos_of[q]].active = true;
                pp.pend[pos_of[q]].v = {carry[q]};
                has_carry[q] = 0;
            }
        for (int i : taken) {
            const EOp& e = ops[i];
            if (e.form == F_M4) {                       // both qubits local (pass cut)
                const Mat4& src = (*mats)[e.mat];
                M4 m;
                for (int k = 0; k < 16; k++) m[k] = cplx(src[2 * k], src[2 * k + 1]);
                pp.add_m4(pos_of[e.q], pos_of[e.c], m);
            } else if (e.form == F_CX) {
                const int t = pos_of[e.q], c = pos_of[e.c];
                if (c >= 0) {
                    pp.add_cx(c, t);
                } else {
                    const M2 x{cplx(0), cplx(1), cplx(1), cplx(0)};
                    pp.add_1q(t, {(int)e.c}, {ident2(), x});
                }
            } else if (pos_of[e.q] >= 0) {
                pp.add_1q(pos_of[e.q], {}, {matrix_of(e)});
            } else {
                const M2 d = matrix_of(e);             // diagonal op on a tile qubit
                pp.add_phase((int)e.q, d[0], d[3]);
            }
        }
        for (int pos = 0; pos < NSLOT; pos++) {
            Pend& pd = pp.pend[pos];
            if (!pd.active || !pd.cond.empty()) continue;
            const int q = P.local_q[pos];
            size_t nj = ci + 1;
            while (nj < cuts.size() && !((touch[nj] >> q) & 1)) nj++;
            if (nj < cuts.size() && ((cuts[nj].first >> q) & 1)) {
                carry[q] = pd.v[0];
                has_carry[q] = 1;
                pd = Pend{};
            }
        }
        pp.finish();
        // 2. layouts: next use of every position after each block
        const size_t nb = pp.blocks.size();
        const int INF = 1 << 30;
        std::vector<std::vector<int>> next(nb + 1, std::vector<int>(NSLOT, INF));
        for (size_t i = nb; i-- > 0;) {
            next[i] = next[i + 1];
            next[i][pp.blocks[i].x] = (int)i;
            next[i][pp.blocks[i].y] = (int)i;
        }
        LayoutPlanner lp{plan, {}, {}};
        int sp[NSLOT];
        {
            // lanes 0 and 1: the first block's qubits (where the low positions leave room);
            // the low positions (qubits 0 and 1) on lanes; then the soonest-needed
            // positions on the free lanes, the next in registers, the latest on the warp bits
            std::vector<int> lanes;
            auto on_lanes = [&](int p) { return std::find(lanes.begin(), lanes.end(), p) != lanes.end(); };
            if (nb > 0) {
                const int x = pp.blocks[0].x, y = pp.blocks[0].y;
                const int room = PR_LANE_BITS - PR_COAL_BITS + (x < PR_COAL_BITS) + (y < PR_COAL_BITS);
                if (room >= 2) { lanes.push_back(x); lanes.push_back(y); }
            }
            for (int p = 0; p < PR_COAL_BITS; p++)
                if (!on_lanes(p)) lanes.push_back(p);
            std::vector<int> rest;
            for (int p = 0; p < NSLOT; p++)
                if (std::find(lanes.begin(), lanes.end(), p) == lanes.end()) rest.push_back(p);
            std::stable_sort(rest.begin(), rest.end(), [&](int a, int b) { return next[0][a] < next[0][b]; });
            size_t k = 0;
            while ((int)lanes.size() < PR_LANE_BITS) lanes.push_back(rest[k++]);
            for (int r = 0; r < RB; r++) sp[SLOT_REG + r] = rest[k++];
            for (int l = 0; l < PR_LANE_BITS; l++) sp[l] = lanes[l];
            for (int w = SLOT_WARP; w < NSLOT; w++) sp[w] = rest[k++];
        }
        lp.set(sp);
        P.load_layout = lp.push_layout();
        P.op_begin = (int32_t)plan.ops.size();
        P.gate_begin = (int32_t)(plan.gates.size() / 64);
        // blocks on disjoint pairs commute: take them in an order that needs few moves.
        // Block j may go once every earlier block sharing a qubit with it has gone.
        std::vector<int> order;
        {
            std::vector<char> done(nb, 0);
            LayoutPlanner probe = lp;
            probe.dry = true;
            size_t first = 0;
            for (size_t step = 0; step < nb; step++) {
                while (first < nb && done[first]) first++;
                int best = -1, best_cost = 1 << 30;
                uint32_t busy = 0;            // qubits of skipped blocks (to keep order)
                for (size_t j = first; j < nb && j < first + 48; j++) {
                    if (done[j]) continue;
                    const uint32_t m = (1u << pp.blocks[j].x) | (1u << pp.blocks[j].y);
                    if (m & busy) { busy |= m; continue; }
                    const int c = probe.pair_cost(pp.blocks[j].x, pp.blocks[j].y);
                    if (c < best_cost) { best_cost = c; best = (int)j; }
                    busy |= m;
                    if (c == 0) break;
                }
                if (best < 0) best = (int)first;     // the first open block is always ready
                done[best] = 1;
                order.push_back(best);
                // advance the probe layout as the real planner will (next use in
                // program order is a close stand-in for the final order's)
                probe.ensure(pp.blocks[best].x, pp.blocks[best].y, next[best]);
            }
        }
        // next use in the chosen order
        std::vector<std::vector<int>> nxt(nb + 1, std::vector<int>(NSLOT, INF));
        for (size_t i = nb; i-- > 0;) {
            nxt[i] = nxt[i + 1];
            nxt[i][pp.blocks[order[i]].x] = (int)i;
            nxt[i][pp.blocks[order[i]].y] = (int)i;
        }
        for (size_t oi = 0; oi < nb; oi++) {
            const Block& b = pp.blocks[order[oi]];
            lp.ensure(b.x, b.y, nxt[oi]);
            PairOp op;
            std::memset(&op, 0, sizeof(op));
            op.kind = PO_BLOCK;
            op.ncond = (uint8_t)b.cond.size();
            for (size_t c = 0; c < b.cond.size(); c++) op.cond_q[c] = (uint8_t)b.cond[c];
            op.gate = (uint32_t)(plan.gates.size() / 64);
            write_block(plan, b, lp.slot_pos[0] != b.x);
            plan.ops.push_back(op);
            plan.n_blocks++;
        }
        // 3. back to a storable layout: positions 0..PR_COAL_BITS-1 on lanes
        bool warp_low = false;
        for (int p = 0; p < PR_COAL_BITS; p++)
            if (lp.where[p] >= SLOT_WARP) warp_low = true;
        if (warp_low) {
            lp.relayout(sp);                   // the load layout is storable
        } else {
            for (int p = 0; p < PR_COAL_BITS; p++) {
                const int s = lp.where[p];
                if (s < SLOT_REG) continue;    // on a lane already
                for (int l = 0; l < PR_LANE_BITS; l++)
                    if (lp.slot_pos[l] >= PR_COAL_BITS) {
                        lp.swap_lr(l, s - SLOT_REG);
                        break;
                    }
            }
        }
        P.store_layout = lp.push_layout();
        P.op_end = (int32_t)plan.ops.size();
        P.gate_count = (int32_t)(plan.gates.size() / 64) - P.gate_begin;
        // what the kernel copies into shared memory beside the tile
        const size_t tile = sizeof(double) * 2 << PR_TILE_BITS;
        const size_t fixed = pair_stage_bytes(P.op_end - P.op_begin, P.store_layout - P.load_layout + 1, 0);
        const size_t with_gates = pair_stage_bytes(P.op_end - P.op_begin, P.store_layout - P.load_layout + 1,
                                                   P.gate_count);
        P.stage_gates = tile + with_gates <= PR_SMEM_CAP ? 1 : 0;
        plan.stage_bytes = std::max(plan.stage_bytes, P.stage_gates ? with_gates : fixed);
        plan.passes.push_back(P);
    }
    return true;
}


// Cost of a plan in units of one block, from the kernel's measured shares (n = 30: a
// lane/register exchange 0.49, a lane permutation 0.36, a relayout 2.05, a pass's tile
// load and store about 0.6).
double plan_cost(const PairPlan& p)
{
    return (double)p.n_blocks + 0.49 * (double)p.n_swaps + 0.36 * (double)p.n_lane_perms +
           2.05 * (double)p.n_relayouts + 0.6 * (double)p.passes.size();
}

}  // namespace

// The pass cut in program order and the one whose first local qubits are also seeded
// (select_passes with 32 seeds) give different plans; the cheaper by the cost model is
// kept (n = 30: 48 passes and 529 blocks, 936 ms, against 50, 539 and 952 ms; at n = 26
// the program-order cut is the cheaper).
bool plan_pairs(const std::vector<EOp>& ops, int n, PairPlan& plan, const std::vector<Mat4>* mats, bool both_cuts)
{
    if (!both_cuts) return plan_pairs_cut(ops, n, plan, mats, 1);
    // the two cuts are independent: a long circuit plans the seeded one on a second host
    // thread (n = 30, 1,800 gates: about 2.5 ms each)
    PairPlan alt;
    bool ok_alt = false;
    std::thread helper;
    if (ops.size() >= 512) {
        try {
            helper = std::thread([&] { ok_alt = plan_pairs_cut(ops, n, alt, mats, 32); });
        } catch (const std::system_error&) {
        }
    }
    const bool ok = plan_pairs_cut(ops, n, plan, mats, 1);
    if (helper.joinable()) helper.join();
    else ok_alt = ok && plan_pairs_cut(ops, n, alt, mats, 32);
    if (!ok) return false;
    if (ok_alt && plan_cost(alt) < plan_cost(plan)) plan = std::move(alt);
    return true;
}
}  // namespace svb

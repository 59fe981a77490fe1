// Pass planner of the staged engine.
//
// The reference sweeps the whole state once per elementary gate and separates the
// sweeps with grid.sync() (svsim/src/svsim_nvgpu_sin.cuh:614-651).  Here the
// elementary-op stream is cut into passes; in one pass every CTA loads one tile of
// 2^M amplitudes (the pass's M local qubits), applies all of the pass's ops to it and
// writes it back, so a pass costs one read and one write of the state however many
// gates it holds.
//
// Legality.  An op may join a pass when
//   * its dense target (or CX target) is one of the pass's local qubits, and
//   * it does not touch a qubit that an op skipped earlier in the scan touches.
// Diagonal ops (Z, S, SDG, T, TDG, R, U1) and CX controls need no locality: their
// qubit only selects which amplitudes change, and a non-local qubit has one fixed
// value per tile.  The skip rule keeps every pair of non-commuting ops in program
// order, because complex-linear ops on disjoint qubits commute (SRN, which is not
// complex-linear, is treated as touching every qubit).
//
// Within a pass the ops are grouped into stages by which 4 local qubits each thread
// holds in registers; between stages the tile is re-distributed through shared memory.
#include <algorithm>
#include <cstring>
#include <functional>

#include "svb_internal.h"

namespace svb {
namespace {

inline uint64_t bit(int q) { return 1ull << q; }

struct OpInfo {
    uint64_t touch;
    int need;      // qubit that must be local (and in registers), or -1
    int need2;     // a second qubit that must be local (F_M4), or -1
};

OpInfo info_of(const EOp& e, uint64_t all)
{
    OpInfo r;
    r.need2 = -1;
    if (e.form == F_M4) {
        r.touch = bit(e.q) | bit(e.c);
        r.need = (int)e.q;
        r.need2 = (int)e.c;
    } else if (e.form == F_SRN) {
        // SRN_GATE (:894-907) as coded maps a to 0.5 (a0 + conj(a1), conj(a0) + a1):
        // it is only real-linear, so it does not commute with a complex gate on any
        // other qubit.  It is ordered against every op of the circuit.
        r.touch = all;
        r.need = (int)e.q;
    } else if (e.form == F_CX) {
        r.touch = bit(e.q) | bit(e.c);
        r.need = (int)e.q;
    } else if (form_is_diag(e.form)) {
        r.touch = bit(e.q);
        r.need = -1;
    } else {
        r.touch = bit(e.q);
        r.need = (int)e.q;
    }
    return r;
}

struct PassBuilder {
    const std::vector<EOp>& ops;
    const std::vector<OpInfo>& inf;
    int n, M, G, TB;
    StagedPlan& plan;

    // order the thread bits of a layout whose register positions are `regs`
    void fill_threads(const std::vector<int>& regs, DevStage& st, bool force_low_lanes) const {
        std::vector<int> comp;
        for (int p = 0; p < M; p++)
            if (std::find(regs.begin(), regs.end(), p) == regs.end()) comp.push_back(p);
        std::vector<int> lanes;
        bool low_free = true;
        for (int p = 0; p < G; p++)
            if (std::find(comp.begin(), comp.end(), p) == comp.end()) low_free = false;
        if (low_free || force_low_lanes) {
            for (int p = 0; p < G; p++) lanes.push_back(p);
        } else {
            // one position per residue class mod G keeps shared-memory phases conflict-free
            for (int r = 0; r < G; r++) {
                for (int p : comp) {
                    if (p % G == r && std::find(lanes.begin(), lanes.end(), p) == lanes.end()) {
                        lanes.push_back(p);
                        break;
                    }
                }
            }
            for (int p : comp) {
                if ((int)lanes.size() >= G) break;
                if (std::find(lanes.begin(), lanes.end(), p) == lanes.end()) lanes.push_back(p);
            }
        }
        std::vector<int> order = lanes;
        for (int p : comp)
            if (std::find(order.begin(), order.end(), p) == order.end()) order.push_back(p);
        std::memset(st.thr_pos, 0, sizeof(st.thr_pos));
        for (int b = 0; b < TB; b++) st.thr_pos[b] = (uint8_t)order[b];
        for (int i = 0; i < RB; i++) st.reg_pos[i] = (uint8_t)regs[i];
    }

    // Builds one pass from `taken` (program order).  Returns the ops that did not fit
    // in MAX_PASS_STAGES stages; they are left for later passes.
    std::vector<int> build(uint64_t L, const std::vector<int>& taken) {
        DevPass P;
        std::memset(&P, 0, sizeof(P));
        int pos_of[64];
        for (int q = 0; q < 64; q++) pos_of[q] = -1;
        int nl = 0, nn = 0;
        for (int q = 0; q < n; q++) {
            if ((L >> q) & 1) { pos_of[q] = nl; P.local_q[nl++] = (uint8_t)q; }
            else P.nonlocal_q[nn++] = (uint8_t)q;
        }
        P.n_nonlocal = nn;
        P.stage_begin = (int32_t)plan.stages.size();

        std::vector<int> remaining = taken, rest, stage_ops;
        bool first = true;
        DevStage last{};
        int n_stages = 0;
        do {
            if (n_stages == MAX_PASS_STAGES) break;
            n_stages++;
            // register positions: first distinct target positions in program order
            std::vector<int> regs;
            for (int i : remaining) {
                if (inf[i].need < 0) continue;
                const int p = pos_of[inf[i].need];
                if (first && p < G) continue;   // low positions are lanes in the load layout
                if (std::find(regs.begin(), regs.end(), p) == regs.end()) regs.push_back(p);
                if ((int)regs.size() == RB) break;
            }
            for (int p = M - 1; (int)regs.size() < RB && p >= (first ? G : 0); p--)
                if (std::find(regs.begin(), regs.end(), p) == regs.end()) regs.push_back(p);
            DevStage st;
            std::memset(&st, 0, sizeof(st));
            fill_threads(regs, st, first);

            uint64_t blocked = 0;
            rest.clear();
            stage_ops.clear();
            for (int i : remaining) {
                const uint64_t t = inf[i].touch;
                if (t & blocked) { blocked |= t; rest.push_back(i); continue; }
                if (inf[i].need >= 0) {
                    const int p = pos_of[inf[i].need];
                    if (std::find(regs.begin(), regs.end(), p) == regs.end()) {
                        blocked |= t;
                        rest.push_back(i);
                        continue;
                    }
                }
                stage_ops.push_back(i);
            }
            st.op_begin = (int32_t)plan.ops.size();
            for (int i : stage_ops) plan.ops.push_back(convert(ops[i], regs, st, pos_of));
            st.op_end = (int32_t)plan.ops.size();
            plan.stages.push_back(st);
            last = st;
            remaining.swap(rest);
            first = false;
        } while (!remaining.empty());

        P.stage_end = (int32_t)plan.stages.size();
        bool store_ok = true;
        for (int b = 0; b < G; b++)
            if (last.thr_pos[b] != b) store_ok = false;
        P.final_relayout = store_ok ? 0 : 1;
        if (!store_ok) {
            std::vector<int> regs;
            for (int p = M - 1; (int)regs.size() < RB; p--) regs.push_back(p);
            std::memset(&P.store_layout, 0, sizeof(P.store_layout));
            fill_threads(regs, P.store_layout, true);
        }
        plan.passes.push_back(P);
        return remaining;
    }

    void locate(uint32_t q, const std::vector<int>& regs, const DevStage& st, const int* pos_of,
                DevOp& d) const {
        const int p = pos_of[q];
        if (p < 0) {
            d.loc_kind = LOC_TILE;
            d.tile_qubit = q;
            return;
        }
        for (int i = 0; i < RB; i++)
            if (regs[i] == p) { d.loc_kind = LOC_REG; d.loc_bit = (uint8_t)i; return; }
        for (int b = 0; b < TB; b++)
            if (st.thr_pos[b] == p) { d.loc_kind = LOC_THR; d.loc_bit = (uint8_t)b; return; }
    }

    DevOp convert(const EOp& e, const std::vector<int>& regs, const DevStage& st,
                  const int* pos_of) const {
        DevOp d;
        std::memset(&d, 0, sizeof(d));
        d.form = e.form;
        std::memcpy(d.m, e.m, sizeof(d.m));
        d.loc_kind = LOC_NONE;
        if (e.form == F_CX || !form_is_diag(e.form)) {
            const int p = pos_of[e.q];
            for (int i = 0; i < RB; i++)
                if (regs[i] == p) d.tgt = (uint8_t)i;
        }
        if (e.form == F_CX) locate(e.c, regs, st, pos_of, d);
        else if (form_is_diag(e.form)) locate(e.q, regs, st, pos_of, d);
        return d;
    }
};

}  // namespace

void select_passes(const std::vector<EOp>& ops, int n, int M, int G,
                   const std::function<std::vector<int>(uint64_t, const std::vector<int>&)>& build,
                   int seeds)
{
    const size_t N = ops.size();
    const uint64_t all = (n >= 64) ? ~0ull : (bit(n) - 1);
    std::vector<OpInfo> inf(N);
    for (size_t i = 0; i < N; i++) inf[i] = info_of(ops[i], all);
    const uint64_t low = bit(G) - 1;
    std::vector<char> done(N, 0);
    size_t first = 0;
    struct Cut {
        uint64_t L = 0;
        int nL = 0;
        std::vector<int> taken, entries;   // entries: taken ops that made qubits local
    };
    // one greedy scan from `first` in program order; op `banned` is treated as blocked;
    // op `seed` (if any) makes its qubits local first
    auto scan = [&](long banned, Cut& c, long seed = -1) {
        c.L = (n == M) ? all : low;
        c.nL = (n == M) ? n : G;
        if (seed >= 0) {
            const int q = inf[seed].need, q2 = inf[seed].need2;
            if (q >= 0 && !((c.L >> q) & 1)) { c.L |= bit(q); c.nL++; }
            if (q2 >= 0 && !((c.L >> q2) & 1)) { c.L |= bit(q2); c.nL++; }
        }
        c.taken.clear();
        c.entries.clear();
        uint64_t blocked = 0;
        for (size_t i = first; i < N; i++) {
            if (done[i]) continue;
            const uint64_t t = inf[i].touch;
            if ((t & blocked) || (long)i == banned) {
                blocked |= t;
                if (blocked == all) break;
                continue;
            }
            const int q = inf[i].need, q2 = inf[i].need2;
            const int extra = (q >= 0 && !((c.L >> q) & 1)) + (q2 >= 0 && !((c.L >> q2) & 1));
            if (extra > 0) {
                if (c.nL + extra <= M) {
                    if (q >= 0) c.L |= bit(q);
                    if (q2 >= 0) c.L |= bit(q2);
                    c.nL += extra;
                    c.entries.push_back((int)i);
                } else {
                    blocked |= t;
                    if (blocked == all) break;
                    continue;
                }
            }
            c.taken.push_back((int)i);
            if ((int)c.taken.size() == MAX_PASS_OPS) break;
        }
    };
    Cut best, alt;
    for (;;) {
        while (first < N && done[first]) first++;
        if (first == N) break;
        scan(-1, best);
        uint64_t front = 0;
        int seen = 0;
        for (size_t i = first; i < N && seen < seeds; i++) {
            if (done[i]) continue;
            seen++;
            const uint64_t t = inf[i].touch;
            if (t & front) { front |= t; continue; }
            front |= t;
            if (seen == 1) continue;
            scan(-1, alt, (long)i);
            if (alt.taken.size() > best.taken.size()) std::swap(best, alt);
        }
        // one step of local search: leaving out one of the ops that chose the local
        // qubits (the first op excepted, so that every pass makes progress) may let the
        // pass take more ops
        const std::vector<int> entries = best.entries;
        for (int e : entries) {
            if (e == (int)first) continue;
            scan(e, alt);
            if (alt.taken.size() > best.taken.size()) std::swap(best, alt);
        }
        for (int i : best.taken) done[i] = 1;
        uint64_t L = best.L;
        int nL = best.nL;
        for (int q = 0; nL < M && q < n; q++)
            if (!((L >> q) & 1)) { L |= bit(q); nL++; }
        for (int i : build(L, best.taken)) done[i] = 0;
    }
}

void plan_staged(const std::vector<EOp>& ops, int n, int M, int G, StagedPlan& plan)
{
    plan.passes.clear();
    plan.stages.clear();
    plan.ops.clear();
    plan.M = M;
    plan.G = G;
    const size_t N = ops.size();
    const uint64_t all = (n >= 64) ? ~0ull : (bit(n) - 1);
    std::vector<OpInfo> inf(N);
    for (size_t i = 0; i < N; i++) inf[i] = info_of(ops[i], all);
    PassBuilder pb{ops, inf, n, M, G, M - RB, plan};
    select_passes(ops, n, M, G, [&](uint64_t L, const std::vector<int>& taken) { return pb.build(L, taken); });
}

}  // namespace svb

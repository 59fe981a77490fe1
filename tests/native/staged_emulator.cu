// TEST INFRASTRUCTURE: runs a staged plan on the CPU.
//
// The planner (sv-sim_b200/csrc/plan.cpp) decides which qubits are local to each pass,
// how each pass is cut into register layouts and where every op's qubits live.  This
// file executes such a plan on host memory with the same per-thread helpers the tile
// kernel uses (staged_core.cuh: swizzle, layout decoding, op application), thread by
// thread and barrier by barrier, and checks on the way that every shared-memory slot is
// written exactly once per re-distribution.  Comparing its output with the oracle
// validates the plan and the kernel's index arithmetic without a GPU.
#include <cstdio>
#include <cstring>
#include <vector>

#include "staged_core.cuh"

using namespace svb;

namespace {

template <typename T, int M>
int run_plan(uint32_t n, const StagedPlan& plan, std::vector<typename VecOf<T>::type>& sv)
{
    using V = typename VecOf<T>::type;
    constexpr int TBITS = M - RB;
    constexpr int NT = 1 << TBITS;
    constexpr int NR = 1 << RB;
    std::vector<V> sm(1u << M);
    std::vector<int> written(1u << M);
    std::vector<V> regs((size_t)NT * NR);
    std::vector<Slots> cur(NT);
    const uint64_t tiles = 1ull << (n - M);

    auto relayout = [&](const DevStage& to) -> int {
        std::fill(written.begin(), written.end(), 0);
        for (int t = 0; t < NT; t++)
            for (int k = 0; k < NR; k++) {
                const uint32_t sl = slot_of(cur[t], k);
                if (sl >= (1u << M) || written[sl]++) return -2;   // not a bijection
                sm[sl] = regs[(size_t)t * NR + k];
            }
        for (int t = 0; t < NT; t++) {
            Slots nx;
            make_slots<T, TBITS>(to, t, nx);
            for (int k = 0; k < NR; k++) regs[(size_t)t * NR + k] = sm[slot_of(nx, k)];
            cur[t] = nx;
        }
        return 0;
    };

    for (size_t p = 0; p < plan.passes.size(); p++) {
        const DevPass& P = plan.passes[p];
        for (uint64_t tile = 0; tile < tiles; tile++) {
            uint64_t base = 0;
            for (int j = 0; j < P.n_nonlocal; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];
            const DevStage* last = &plan.stages[P.stage_begin];
            for (int t = 0; t < NT; t++) {
                GOffs g;
                make_goffs<TBITS>(*last, P, t, g);
                for (int k = 0; k < NR; k++) regs[(size_t)t * NR + k] = sv[base | goff_of(g, k)];
                make_slots<T, TBITS>(*last, t, cur[t]);
            }
            for (int s = P.stage_begin; s < P.stage_end; s++) {
                const DevStage& S = plan.stages[s];
                if (s != P.stage_begin) {
                    if (relayout(S)) return -2;
                    last = &S;
                }
                for (int t = 0; t < NT; t++)
                    for (int o = S.op_begin; o < S.op_end; o++)
                        apply_devop<T>(&plan.ops[o], &regs[(size_t)t * NR], t, base);
            }
            if (P.final_relayout) {
                if (relayout(P.store_layout)) return -2;
                last = &P.store_layout;
            }
            // stores must cover the tile exactly once as well
            for (int t = 0; t < NT; t++) {
                GOffs g;
                make_goffs<TBITS>(*last, P, t, g);
                for (int k = 0; k < NR; k++) sv[base | goff_of(g, k)] = regs[(size_t)t * NR + k];
            }
        }
    }
    return 0;
}

template <typename T>
int run_typed(uint32_t n, const StagedPlan& plan, double* re, double* im)
{
    using V = typename VecOf<T>::type;
    const uint64_t dim = 1ull << n;
    std::vector<V> sv(dim);
    for (uint64_t i = 0; i < dim; i++) { sv[i].x = (T)re[i]; sv[i].y = (T)im[i]; }
    int rc;
    switch (plan.M) {
    case 10: rc = run_plan<T, 10>(n, plan, sv); break;
    case 11: rc = run_plan<T, 11>(n, plan, sv); break;
    case 12: rc = run_plan<T, 12>(n, plan, sv); break;
    case 13: rc = run_plan<T, 13>(n, plan, sv); break;
    default: return -1;
    }
    for (uint64_t i = 0; i < dim; i++) { re[i] = (double)sv[i].x; im[i] = (double)sv[i].y; }
    return rc;
}

}  // namespace

extern "C" {

// Applies `gates` to the SoA state (re, im) in place through the staged plan with tile
// bits M.  precision: 0 = FP64, 1 = FP32.  Returns 0, -1 for bad arguments, -2 if a
// re-distribution is not a bijection on the tile.
int emu_staged_run(uint32_t n, const svb_gate* gates, size_t n_gates, int M, int precision,
                   double* re, double* im, uint64_t* n_passes, uint64_t* n_stages)
{
    if (M < 10 || M > 13 || (int)n < M) return -1;
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    StagedPlan plan;
    plan_staged(eops, (int)n, M, precision == 0 ? 3 : 4, plan);
    if (n_passes) *n_passes = plan.passes.size();
    if (n_stages) *n_stages = plan.stages.size();
    return precision == 0 ? run_typed<double>(n, plan, re, im) : run_typed<float>(n, plan, re, im);
}

// Pass / stage / relayout counts of the plan without executing it.
int emu_plan_stats(uint32_t n, const svb_gate* gates, size_t n_gates, int M, int precision,
                   uint64_t* n_passes, uint64_t* n_stages, uint64_t* n_final_relayouts,
                   uint64_t* n_elementary)
{
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    StagedPlan plan;
    plan_staged(eops, (int)n, M, precision == 0 ? 3 : 4, plan);
    *n_passes = plan.passes.size();
    *n_stages = plan.stages.size();
    uint64_t f = 0;
    for (const DevPass& P : plan.passes) f += P.final_relayout;
    *n_final_relayouts = f;
    *n_elementary = eops.size();
    return 0;
}

}  // extern "C"

extern "C" int emu_plan_dump(uint32_t n, const svb_gate* gates, size_t n_gates, int M, int precision)
{
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    StagedPlan plan;
    plan_staged(eops, (int)n, M, precision == 0 ? 3 : 4, plan);
    const int TB = M - RB;
    for (size_t p = 0; p < plan.passes.size(); p++) {
        const DevPass& P = plan.passes[p];
        printf("pass %zu local:", p);
        for (int j = 0; j < M; j++) printf(" %d", P.local_q[j]);
        printf(" final_relayout=%d\n", P.final_relayout);
        for (int s = P.stage_begin; s < P.stage_end; s++) {
            const DevStage& S = plan.stages[s];
            printf("  stage %d regs(pos):", s);
            for (int i = 0; i < RB; i++) printf(" %d", S.reg_pos[i]);
            printf(" thr(pos):");
            for (int b = 0; b < TB; b++) printf(" %d", S.thr_pos[b]);
            printf("\n");
            for (int o = S.op_begin; o < S.op_end; o++) {
                const DevOp& d = plan.ops[o];
                printf("    form=%d tgt=%d loc=%d bit=%d tq=%u\n", d.form, d.tgt, d.loc_kind, d.loc_bit, d.tile_qubit);
            }
        }
    }
    fflush(stdout);
    return 0;
}

// ---- fused tensor-core plans ---------------------------------------------------------
// Executes a fused plan on the CPU with the kernel's data flow: block 0's rows gathered
// from the raw tile (raw_xor layout) through the a/n tables; D[n][m'] =
// sum_kk X[n][kk] (G_hi + G_lo)[m'][kk] with G_hi and G_lo read from rows m' and N + m'
// of the 2N-row canonical K-major gate operand; each D row scattered through the
// XOR-combined next tables into the transpose buffer (every slot written once) and the
// next block's rows read back from it at fused_slot(n, a); the last block's rows
// scattered into the output stage (out_xor layout).  The MMA is evaluated in FP64
// here; only the layout and table logic are under test.
static uint32_t emu_kmajor(uint32_t row, uint32_t kk, uint32_t rows)
{
    return ((kk >> 2) * (rows * 16u) + (row >> 3) * 128u + (row & 7u) * 16u + (kk & 3u) * 4u) / 4u;
}

extern "C" int emu_fused_run(uint32_t n, const svb_gate* gates, size_t n_gates, int k,
                             double* re, double* im, uint64_t* n_passes, uint64_t* n_blocks)
{
    if ((int)n < FT_TILE_BITS || k < FT_MIN_K || k >= F6_K) return -1;
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    if (!fusable(eops)) return -3;
    FusedPlan plan;
    plan_fused(eops, (int)n, k, plan);
    if (n_passes) *n_passes = plan.passes.size();
    if (n_blocks) *n_blocks = plan.blocks.size();
    const int N = 1 << (k + 1), ROWS = 1 << (FT_TILE_BITS - k), A = 1 << k;
    const uint64_t tiles = 1ull << (n - FT_TILE_BITS);
    std::vector<double> X((size_t)ROWS * N), T(4096 * 2), O(4096 * 2);
    std::vector<double> raw(4096 * 2);
    for (const FusedPass& P : plan.passes) {
        if (P.n_blocks < 1 || P.n_blocks > fused_max_blocks(k)) return -5;
        for (uint64_t t = 0; t < tiles; t++) {
            uint64_t base = 0;
            for (int j = 0; j < P.n_nonlocal; j++) base |= ((t >> j) & 1ull) << P.nonlocal_q[j];
            // the raw tile: 256 runs of 16 local positions (local index 16 r + i)
            for (uint32_t r = 0; r < 256; r++) {
                for (uint32_t i = 0; i < 16; i++) {
                    const uint64_t g = base + P.g_lo[((r & 3) << 4) | i] + P.g_hi[r >> 2];
                    const uint32_t w = (16 * r + i) ^ ((uint32_t)P.raw_xor[r] << 1);
                    raw[2 * w] = re[g];
                    raw[2 * w + 1] = im[g];
                }
            }
            const FusedBlock& B0 = plan.blocks[P.block_begin];
            for (int nr = 0; nr < ROWS; nr++) {
                const uint32_t rl = (uint32_t)B0.n_lo[nr & 31] ^ (uint32_t)B0.n_hi[nr >> 5];
                for (int a = 0; a < A; a++) {
                    const uint32_t l = rl ^ B0.a_sc[a];   // raw-tile word
                    X[(size_t)nr * N + 2 * a] = raw[2 * l];
                    X[(size_t)nr * N + 2 * a + 1] = raw[2 * l + 1];
                }
            }
            for (int b = 0; b < P.n_blocks; b++) {
                const FusedBlock& B = plan.blocks[P.block_begin + b];
                const float* gop = plan.gates.data() + B.gate_word;
                const bool last = (b + 1 == P.n_blocks);
                std::vector<int> seen(4096, 0);
                for (int nr = 0; nr < ROWS; nr++) {
                    std::vector<double> d(N, 0.0);
                    for (int mp = 0; mp < N; mp++) {
                        double s = 0;
                        for (int kk = 0; kk < N; kk++) {
                            const double g = (double)gop[emu_kmajor(mp, kk, 2 * N)] +
                                             (double)gop[emu_kmajor(N + mp, kk, 2 * N)];
                            s += X[(size_t)nr * N + kk] * g;
                        }
                        d[mp] = s;
                    }
                    const uint32_t wn = (uint32_t)B.nxt_nlo[nr & 31] ^ (uint32_t)B.nxt_nhi[nr >> 5];
                    for (int a = 0; a < A; a++) {
                        const uint32_t w = wn ^ B.nxt_a[a];
                        if (w >= 4096 || seen[w]++) return -2;
                        std::vector<double>& dst = last ? O : T;
                        dst[2 * w] = d[2 * a];
                        dst[2 * w + 1] = d[2 * a + 1];
                    }
                }
                if (!last) {
                    // rows of the next block, read back at their transpose slots
                    for (int nr = 0; nr < ROWS; nr++)
                        for (int a = 0; a < A; a++) {
                            const uint32_t w = fused_slot((uint32_t)nr, (uint32_t)a, k);
                            X[(size_t)nr * N + 2 * a] = T[2 * w];
                            X[(size_t)nr * N + 2 * a + 1] = T[2 * w + 1];
                        }
                }
            }
            for (uint32_t r = 0; r < 256; r++) {
                for (uint32_t i = 0; i < 16; i++) {
                    const uint64_t g = base + P.g_lo[((r & 3) << 4) | i] + P.g_hi[r >> 2];
                    const uint32_t w = (16 * r + i) ^ (uint32_t)P.out_xor[r];
                    re[g] = O[2 * w];
                    im[g] = O[2 * w + 1];
                }
            }
        }
    }
    return 0;
}

// Fusion width 6 (plan_fused6, kernels_fused6.cu): amplitude x = thread + 512 i of a tile
// is copied to word s_lo[x & 63] + s_hi[x >> 6] of the B-operand plane (each word once);
// the MMA reads X[n][kk] at the canonical K-major position of (row n, kk) among 64 rows;
// D^T[m'][n] = sum_kk (G_hi + G_lo)[m'][kk] X[n][kk]; amplitude (n, a') of the output goes
// to o_row[n] | o_tgt[a'] (each once), and pairs of rows share one 16-byte store when
// rows_paired is set.  The arithmetic is FP64; only the layouts and tables are under test.
extern "C" int emu_fused6_run(uint32_t n, const svb_gate* gates, size_t n_gates, double* re, double* im,
                              uint64_t* n_passes)
{
    if ((int)n < F6_TILE_BITS) return -1;
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    if (!fusable(eops)) return -3;
    FusedPlan plan;
    plan_fused6(eops, (int)n, plan);
    if (n_passes) *n_passes = plan.passes6.size();
    const uint64_t tiles = 1ull << (n - F6_TILE_BITS);
    std::vector<double> plane(4096 * 2), D((size_t)F6_N * F6_ROWS);
    for (const Fused6Pass& P : plan.passes6) {
        if (P.n_nonlocal != (int)n - F6_TILE_BITS) return -5;
        if (P.rows_paired)
            for (int r = 0; r < F6_ROWS; r += 2)
                if (P.o_row[r + 1] != P.o_row[r] + 1) return -6;
        const float* gh = plan.gates.data() + P.gate_word;
        const float* gl = gh + (size_t)F6_N * F6_N;
        for (uint64_t t = 0; t < tiles; t++) {
            uint64_t base = 0;
            for (int j = 0; j < P.n_nonlocal; j++) base |= ((t >> j) & 1ull) << P.nonlocal_q[j];
            std::vector<int> seen(4096, 0);
            for (uint32_t x = 0; x < 4096; x++) {
                const uint64_t g = base + (P.g_lo[x & 63] | P.g_hi[x >> 6]);
                const uint32_t w = (uint32_t)P.s_lo[x & 63] + (uint32_t)P.s_hi[x >> 6];
                if (w >= 4096 || seen[w]++) return -2;
                plane[2 * w] = re[g];
                plane[2 * w + 1] = im[g];
            }
            for (int nr = 0; nr < F6_ROWS; nr++)
                for (int mp = 0; mp < F6_N; mp++) {
                    double s = 0;
                    for (int kk = 0; kk < F6_N; kk++)
                        s += ((double)gh[(size_t)mp * F6_N + kk] + (double)gl[(size_t)mp * F6_N + kk]) *
                             plane[emu_kmajor((uint32_t)nr, (uint32_t)kk, F6_ROWS)];
                    D[(size_t)mp * F6_ROWS + nr] = s;
                }
            std::vector<int> out(4096, 0);
            for (int nr = 0; nr < F6_ROWS; nr++)
                for (int a = 0; a < (1 << F6_K); a++) {
                    const uint64_t off = P.o_row[nr] | P.o_tgt[a];
                    if (off >= (1ull << n) || (off & ~(P.g_lo[63] | P.g_hi[63])) != 0) return -4;
                    re[base + off] = D[(size_t)(2 * a) * F6_ROWS + nr];
                    im[base + off] = D[(size_t)(2 * a + 1) * F6_ROWS + nr];
                }
        }
    }
    return 0;
}

// passes and blocks of a fused plan, without running it
extern "C" int emu_fused_stats(uint32_t n, const svb_gate* gates, size_t n_gates, int k, uint64_t* n_passes,
                               uint64_t* n_blocks)
{
    if ((int)n < FT_TILE_BITS || k < FT_MIN_K || k > FT_MAX_K) return -1;
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    if (!fusable(eops)) return -3;
    FusedPlan plan;
    if (k == F6_K) plan_fused6(eops, (int)n, plan);
    else plan_fused(eops, (int)n, k, plan);
    *n_passes = plan.n_passes();
    *n_blocks = k == F6_K ? plan.passes6.size() : plan.blocks.size();
    return 0;
}

// ---- pair engine ---------------------------------------------------------------------
// Executes a pair plan (pairs.cpp) thread by thread with the kernel's data movement:
// PO_SWAP as the warp-shuffle exchange, PO_RELAYOUT through the swizzled shared tile
// (every slot written once), PO_BLOCK as the mma.sync m8n8k4 fragment rules (thread t
// holds A[t>>2][t&3] and B[t&3][t>>2], receives D[t>>2][2(t&3)], D[t>>2][2(t&3)+1]).
static int pairs_run(uint32_t n, const svb_gate* gates, size_t n_gates, double* re, double* im,
                     uint64_t* stats, bool from_input)
{
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    PairPlan plan;
    if (!plan_pairs(eops, (int)n, plan)) return -6;
    constexpr int NT = 256, NR = 16, TB = 8;
    std::vector<double2> sv(1ull << n);
    for (auto& a : sv) a = make_double2(0, 0);
    sv[0] = make_double2(1, 0);
    if (from_input)
        for (uint64_t i = 0; i < sv.size(); i++) sv[i] = make_double2(re[i], im[i]);
    std::vector<double2> regs((size_t)NT * NR), sm(4096);
    std::vector<int> written(4096);
    const uint64_t tiles = 1ull << (n - PR_TILE_BITS);
    for (const PairPass& P : plan.passes) {
        auto goff = [&](const DevStage& S, int t, int k) {
            uint64_t g = 0;
            for (int b = 0; b < TB; b++)
                if ((t >> b) & 1) g |= 1ull << P.local_q[S.thr_pos[b]];
            for (int i = 0; i < RB; i++)
                if ((k >> i) & 1) g |= 1ull << P.local_q[S.reg_pos[i]];
            return g;
        };
        const DevStage& Ld = plan.layouts[P.load_layout];
        const DevStage& St = plan.layouts[P.store_layout];
        for (int p = 0; p < PR_COAL_BITS; p++) {              // the low positions on lanes at load and store
            bool ld = false, st = false;
            for (int l = 0; l < PR_LANE_BITS; l++) {
                ld |= Ld.thr_pos[l] == p;
                st |= St.thr_pos[l] == p;
            }
            if (!ld || !st) return -5;
        }
        for (uint64_t tile = 0; tile < tiles; tile++) {
            uint64_t base = 0;
            for (int j = 0; j < P.n_nonlocal; j++) base |= ((tile >> j) & 1ull) << P.nonlocal_q[j];
            for (int t = 0; t < NT; t++)
                for (int k = 0; k < NR; k++) regs[(size_t)t * NR + k] = sv[base | goff(Ld, t, k)];
            // the layout the planner believes in, tracked through the swaps
            int slot_pos[PR_TILE_BITS];
            for (int l = 0; l < PR_LANE_BITS; l++) slot_pos[l] = Ld.thr_pos[l];
            for (int r = 0; r < RB; r++) slot_pos[PR_LANE_BITS + r] = Ld.reg_pos[r];
            for (int w = 0; w < 3; w++) slot_pos[PR_LANE_BITS + RB + w] = Ld.thr_pos[PR_LANE_BITS + w];
            for (int o = P.op_begin; o < P.op_end; o++) {
                const PairOp& op = plan.ops[o];
                if (op.kind == PO_SWAP) {
                    const int L = op.lane, R = op.reg;
                    std::vector<double2> send((size_t)NT * NR);
                    for (int t = 0; t < NT; t++) {
                        const bool hi = (t >> L) & 1;
                        for (int k = 0; k < NR; k++) {
                            if (k & (1 << R)) continue;
                            const int k1 = k | (1 << R);
                            send[(size_t)t * NR + k] = hi ? regs[(size_t)t * NR + k] : regs[(size_t)t * NR + k1];
                        }
                    }
                    for (int t = 0; t < NT; t++) {
                        const bool hi = (t >> L) & 1;
                        const int u = t ^ (1 << L);
                        for (int k = 0; k < NR; k++) {
                            if (k & (1 << R)) continue;
                            const int k1 = k | (1 << R);
                            const double2 recv = send[(size_t)u * NR + k];
                            if (hi) regs[(size_t)t * NR + k] = recv;
                            else regs[(size_t)t * NR + k1] = recv;
                        }
                    }
                    std::swap(slot_pos[L], slot_pos[PR_LANE_BITS + R]);
                } else if (op.kind == PO_LPERM) {
                    // lane bit b takes the element of lane bit from[b]
                    int from[PR_LANE_BITS];
                    for (int b = 0; b < PR_LANE_BITS; b++) from[b] = (int)((op.gate >> (3 * b)) & 7u);
                    std::vector<double2> old(regs);
                    for (int t = 0; t < NT; t++) {
                        const int lane = t & 31;
                        int src = 0;
                        for (int b = 0; b < PR_LANE_BITS; b++) src |= ((lane >> b) & 1) << from[b];
                        if (src > 31) return -7;
                        for (int k = 0; k < NR; k++) regs[(size_t)t * NR + k] = old[(size_t)((t & ~31) | src) * NR + k];
                    }
                    int sp[PR_LANE_BITS];
                    for (int b = 0; b < PR_LANE_BITS; b++) sp[b] = slot_pos[from[b]];
                    for (int b = 0; b < PR_LANE_BITS; b++) slot_pos[b] = sp[b];
                } else if (op.kind == PO_RELAYOUT) {
                    const DevStage& A = plan.layouts[op.src];
                    const DevStage& B = plan.layouts[op.layout];
                    for (int l = 0; l < PR_LANE_BITS; l++)
                        if (A.thr_pos[l] != slot_pos[l]) return -2;
                    for (int r = 0; r < RB; r++)
                        if (A.reg_pos[r] != slot_pos[PR_LANE_BITS + r]) return -2;
                    std::fill(written.begin(), written.end(), 0);
                    for (int t = 0; t < NT; t++) {
                        Slots s;
                        make_slots<double, TB>(A, t, s);
                        for (int k = 0; k < NR; k++) {
                            const uint32_t sl = slot_of(s, k);
                            if (sl >= 4096 || written[sl]++) return -3;
                            sm[sl] = regs[(size_t)t * NR + k];
                        }
                    }
                    for (int t = 0; t < NT; t++) {
                        Slots s;
                        make_slots<double, TB>(B, t, s);
                        for (int k = 0; k < NR; k++) regs[(size_t)t * NR + k] = sm[slot_of(s, k)];
                    }
                    for (int l = 0; l < PR_LANE_BITS; l++) slot_pos[l] = B.thr_pos[l];
                    for (int r = 0; r < RB; r++) slot_pos[PR_LANE_BITS + r] = B.reg_pos[r];
                    for (int w = 0; w < 3; w++) slot_pos[PR_LANE_BITS + RB + w] = B.thr_pos[PR_LANE_BITS + w];
                } else {
                    int var = 0;
                    for (int c = 0; c < op.ncond; c++) var |= (int)((base >> op.cond_q[c]) & 1ull) << c;
                    const double* g = plan.gates.data() + (size_t)(op.gate + var) * 64;
                    for (int w = 0; w < NT / 32; w++)
                        for (int k = 0; k < NR; k++) {
                            double D[8][8] = {{0}};
                            for (int step = 0; step < 2; step++) {
                                double A[8][4], Bm[4][8];
                                for (int t = 0; t < 32; t++) {
                                    const double2 x = regs[(size_t)(w * 32 + t) * NR + k];
                                    A[t >> 2][t & 3] = step ? x.y : x.x;
                                    Bm[t & 3][t >> 2] = g[2 * t + step];
                                }
                                for (int r = 0; r < 8; r++)
                                    for (int c = 0; c < 8; c++) {
                                        double acc = D[r][c];
                                        for (int kk = 0; kk < 4; kk++) acc += A[r][kk] * Bm[kk][c];
                                        D[r][c] = acc;
                                    }
                            }
                            for (int t = 0; t < 32; t++)
                                regs[(size_t)(w * 32 + t) * NR + k] =
                                    make_double2(D[t >> 2][2 * (t & 3)], D[t >> 2][2 * (t & 3) + 1]);
                        }
                }
            }
            for (int l = 0; l < PR_LANE_BITS; l++)
                if (St.thr_pos[l] != slot_pos[l]) return -4;
            for (int r = 0; r < RB; r++)
                if (St.reg_pos[r] != slot_pos[PR_LANE_BITS + r]) return -4;
            for (int t = 0; t < NT; t++)
                for (int k = 0; k < NR; k++) sv[base | goff(St, t, k)] = regs[(size_t)t * NR + k];
        }
    }
    for (size_t i = 0; i < sv.size(); i++) {
        re[i] = sv[i].x;
        im[i] = sv[i].y;
    }
    if (stats) {
        stats[0] = plan.passes.size();
        stats[1] = plan.n_blocks;
        stats[2] = plan.n_swaps;
        stats[3] = plan.n_relayouts;
    }
    return 0;
}

// Plan statistics of the pair engine (no execution): passes, blocks, swaps, relayouts.

// A pair plan run thread by thread from |0..0> (re, im out).
extern "C" int emu_pairs_run(uint32_t n, const svb_gate* gates, size_t n_gates, double* re, double* im,
                             uint64_t* stats)
{
    return pairs_run(n, gates, n_gates, re, im, stats, false);
}

// The same from the state in re, im (in and out): a plan must be right on any input state.
extern "C" int emu_pairs_run_from(uint32_t n, const svb_gate* gates, size_t n_gates, double* re, double* im,
                                  uint64_t* stats)
{
    return pairs_run(n, gates, n_gates, re, im, stats, true);
}

static int pairs_stats(uint32_t n, const svb_gate* gates, size_t n_gates, uint64_t* stats, bool both_cuts)
{
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    PairPlan plan;
    if (!plan_pairs(eops, (int)n, plan, nullptr, both_cuts)) return -6;
    stats[0] = plan.passes.size();
    stats[1] = plan.n_blocks;
    stats[2] = plan.n_swaps;
    stats[3] = plan.n_relayouts;
    // passes whose gate fragments stay in global memory (too many for shared memory), and
    // the largest per-pass copy into shared memory
    uint64_t unstaged = 0;
    for (const PairPass& P : plan.passes) unstaged += P.stage_gates ? 0 : 1;
    stats[4] = unstaged;
    stats[5] = plan.stage_bytes;
    stats[6] = plan.n_lane_perms;
    return 0;
}

extern "C" int emu_pairs_stats(uint32_t n, const svb_gate* gates, size_t n_gates, uint64_t* stats)
{
    return pairs_stats(n, gates, n_gates, stats, true);
}

// The same for the program-order pass cut alone.
extern "C" int emu_pairs_stats_one_cut(uint32_t n, const svb_gate* gates, size_t n_gates, uint64_t* stats)
{
    return pairs_stats(n, gates, n_gates, stats, false);
}

// ---- shared-memory bank model of the fused kernel's accesses ---------------------------
// Wavefronts of one warp access: 8-byte accesses go in two phases of 16 lanes (16 bank
// pairs of 8 bytes), 16-byte accesses in four phases of 8 lanes (8 groups of 16 bytes);
// within a phase, distinct words on the same bank unit serialise.
static int emu_wavefronts(const uint32_t* word, int bytes)
{
    const int lanes = bytes == 8 ? 16 : 8, units = bytes == 8 ? 16 : 8;
    int wf = 0;
    for (int p = 0; p < 32 / lanes; p++) {
        int worst = 0;
        for (int u = 0; u < units; u++) {
            uint32_t seen[32];
            int cnt = 0;
            for (int l = p * lanes; l < (p + 1) * lanes; l++) {
                if ((int)(word[l] % (uint32_t)units) != u) continue;
                bool dup = false;
                for (int i = 0; i < cnt; i++) dup |= seen[i] == word[l];
                if (!dup) seen[cnt++] = word[l];
            }
            if (cnt > worst) worst = cnt;
        }
        wf += worst;
    }
    return wf;
}

// Average wavefronts per warp instruction of the fused kernel's shared-memory accesses for
// the plan of a circuit: out[0] block-0 gather from the raw tile (8-byte loads, ideal 2),
// out[1] D rows into the transpose buffer (8-byte stores, ideal 2), out[2] rows read back
// (16-byte loads, ideal 4), out[3] last block into the output stage (8-byte stores, ideal 2).
extern "C" int emu_fused_conflicts(uint32_t n, const svb_gate* gates, size_t n_gates, int k, double* out)
{
    if ((int)n < FT_TILE_BITS || k < FT_MIN_K || k > FT_MAX_K) return -1;
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++)
        if (!lower_gate(gates[i], (int32_t)i, eops)) return -1;
    if (!fusable(eops)) return -3;
    FusedPlan plan;
    plan_fused(eops, (int)n, k, plan);
    const int PARTS = FT_EPI_WARPS / 4;
    const int MBLK = (1 << (FT_TILE_BITS - k)) / 128, CW = (2 << k) / PARTS, CA = CW / 2;
    double wf[4] = {0, 0, 0, 0}, ins[4] = {0, 0, 0, 0};
    uint32_t word[32];
    for (const FusedPass& P : plan.passes) {
        for (int b = 0; b < P.n_blocks; b++) {
            const FusedBlock& B = plan.blocks[P.block_begin + b];
            const bool last = b + 1 == P.n_blocks;
            for (int warp = 0; warp < FT_EPI_WARPS; warp++) {
                const int quad = warp & 3, part = warp >> 2;
                for (int mb = 0; mb < MBLK; mb++)
                    for (int a2 = 0; a2 < CA; a2++) {
                        const int a = part * CA + a2;
                        if (b == 0) {
                            for (int lane = 0; lane < 32; lane++) {
                                const uint32_t nr = (uint32_t)(128 * mb + 32 * quad + lane);
                                word[lane] = (uint32_t)B.n_lo[nr & 31] ^ B.n_hi[nr >> 5] ^ B.a_sc[a];
                            }
                            wf[0] += emu_wavefronts(word, 8);
                            ins[0] += 1;
                        }
                        for (int lane = 0; lane < 32; lane++) {
                            const uint32_t nr = (uint32_t)(128 * mb + 32 * quad + lane);
                            word[lane] = (uint32_t)B.nxt_nlo[nr & 31] ^ B.nxt_nhi[nr >> 5] ^ B.nxt_a[a];
                        }
                        wf[last ? 3 : 1] += emu_wavefronts(word, 8);
                        ins[last ? 3 : 1] += 1;
                    }
                if (!last)
                    for (int mb = 0; mb < MBLK; mb++)
                        for (int c2 = 0; c2 < CA / 2; c2++) {
                            const uint32_t c = (uint32_t)(part * (CA / 2) + c2);
                            for (int lane = 0; lane < 32; lane++) {
                                const uint32_t nr = (uint32_t)(128 * mb + 32 * quad + lane);
                                word[lane] = fused_slot(nr, 2 * c, k) >> 1;
                            }
                            wf[2] += emu_wavefronts(word, 16);
                            ins[2] += 1;
                        }
            }
        }
    }
    for (int i = 0; i < 4; i++) out[i] = ins[i] > 0 ? wf[i] / ins[i] : 0.0;
    return 0;
}

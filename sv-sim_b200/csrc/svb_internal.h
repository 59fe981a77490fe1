// Internal declarations of libsvsim_b200: elementary ops, the pass planner's output,
// the device-side descriptors and the handle.
#pragma once

#include <array>
#include <cstdint>
#include <cstddef>
#include <string>
#include <functional>
#include <vector>

#include <cuda_runtime.h>

#include "svsim_b200.h"

namespace svb {

// ---------------------------------------------------------------------------------
// Elementary ops.  The reference applies every gate as a sequence of these
// (svsim_nvgpu_sin.cuh:654-1454); each form keeps the reference's arithmetic.
// ---------------------------------------------------------------------------------
enum Form : uint8_t {
    F_C1 = 0,   // C1_GATE :654      general 2x2: m = e0r e0i e1r e1i e2r e2i e3r e3i
    F_X,        // X_GATE :818
    F_Y,        // Y_GATE :837
    F_H,        // H_GATE :873
    F_SRN,      // SRN_GATE :894
    F_W,        // W_GATE :1428
    F_RX,       // RX_GATE :1085     m[0] = cos(t/2), m[1] = -sin(t/2)
    F_RY,       // RY_GATE :1104     m[0..3] = e0r e1r e2r e3r
    // forms that only change the |1> amplitude of the pair (diagonal): the qubit
    // need not be local to a tile
    F_Z,        // Z_GATE :857
    F_S,        // S_GATE :940
    F_SDG,      // SDG_GATE :955
    F_T,        // T_GATE :970
    F_TDG,      // TDG_GATE :985
    F_R,        // R_GATE :924       m[0] = phase
    F_U1,       // U1_GATE :1022     m[0] = cos(l), m[1] = sin(l)
    F_DIAG,     // diag(d0, d1), m = d0r d0i d1r d1i (adjoint inverses only)
    // two-qubit
    F_CX,       // CX_GATE :779      swap (c=1,t=0) <-> (c=1,t=1)
    F_M4,       // general 4x4 complex matrix on (q: bit 0, c: bit 1), entries in a side
                // table (EOp::mat); density-matrix superoperators; pair and per-gate only
    F_COUNT
};

__host__ __device__ inline bool form_is_diag(int f) { return f >= F_Z && f <= F_DIAG; }

struct EOp {
    uint8_t form = F_C1;
    uint32_t q = 0;        // target (dense, CX) or the qubit of a diagonal op
    uint32_t c = 0;        // control (CX); second qubit (F_M4)
    int32_t mat = -1;      // F_M4: index of its 4x4 matrix in the circuit's matrix table
    double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // --- adjoint bookkeeping ---
    int32_t gate = -1;     // index of the source gate
    uint8_t kind = 0;      // elementary kind for derivatives: see lower.cpp (EK_*)
    double ang[3] = {0, 0, 0};    // the elementary op's own angles
    double jac[3][3] = {{0}};     // d ang[i] / d gate-field[f]  (theta, phi, lambda)
};

// Expands one reference gate into elementary ops (the composite sequences of
// svsim_nvgpu_sin.cuh:1134-1454).  Returns false for an unknown op.
bool lower_gate(const svb_gate& g, int32_t gate_index, std::vector<EOp>& out);

// Number of elementary ops and of per-gate-model sweeps (half sweeps count 1/2)
// the reference spends on one op.
double reference_sweeps(uint32_t op);

// ---------------------------------------------------------------------------------
// Staged engine: passes and stages.
//
// A pass streams the state once through tiles of 2^M amplitudes.  The M "local"
// qubits of a pass always include the G lowest qubits (so every tile is made of
// contiguous 2^G-amplitude runs) plus M-G qubits chosen by the planner.  Inside a
// tile each of the 2^(M-RB) threads holds 2^RB amplitudes in registers; a stage is a
// run of ops whose dense targets are among the RB register qubits of the stage's
// layout.  Between stages the tile is re-distributed through shared memory.
// ---------------------------------------------------------------------------------
constexpr int RB = 4;            // register bits per thread (16 amplitudes)
constexpr int MAX_PASS_OPS = 256;     // ops of one pass, staged in shared memory
constexpr int MAX_PASS_STAGES = 64;   // stages of one pass
constexpr int MAX_TB = 9;        // thread bits (512 threads)
constexpr int MAX_M = RB + MAX_TB;

enum LocKind : uint8_t { LOC_REG = 0, LOC_THR = 1, LOC_TILE = 2, LOC_NONE = 3 };

struct DevOp {                   // 80 bytes, read by every thread of a tile
    double m[8];                 // coefficients first: 16-byte aligned for vector loads
    uint8_t form;
    uint8_t tgt;                 // register bit of the dense/CX target
    uint8_t loc_kind;            // where the diagonal qubit / CX control lives
    uint8_t loc_bit;             // its register or thread bit
    uint32_t tile_qubit;         // its global qubit when loc_kind == LOC_TILE
    uint64_t pad;
};
static_assert(sizeof(DevOp) == 80, "DevOp layout");

struct DevStage {
    uint8_t reg_pos[RB];         // local positions held in registers (bit i of k)
    uint8_t thr_pos[MAX_TB];     // local positions of thread-index bits
    uint8_t pad[3];
    int32_t op_begin, op_end;    // range in the DevOp array
};
static_assert(sizeof(DevStage) == 24, "DevStage layout");

struct DevPass {
    uint8_t local_q[MAX_M];      // global qubit of each local position (ascending)
    uint8_t nonlocal_q[64 - MAX_M];  // global qubits of tile-index bits (ascending)
    int32_t n_nonlocal;
    int32_t stage_begin, stage_end;
    int32_t final_relayout;      // 1: re-distribute to a store layout before writing
    DevStage store_layout;       // used when final_relayout
};

struct StagedPlan {
    int M = 0;                   // tile bits
    int G = 0;                   // always-local low qubits (swizzle group)
    std::vector<DevPass> passes;
    std::vector<DevStage> stages;
    std::vector<DevOp> ops;
};

// Builds the staged plan for `ops` on n qubits with tile bits M and low-group G.
void plan_staged(const std::vector<EOp>& ops, int n, int M, int G, StagedPlan& plan);

// ---- pair engine (FP64 two-qubit blocks on the FP64 tensor cores) ----------------
//
// A pass holds PR_TILE_BITS = 12 local qubits.  Each of the 256 threads keeps 16
// amplitudes; the 12 local positions sit on 5 lane bits, 4 register bits and 3 warp
// bits, described by a DevStage (thr_pos[0..4] = lane bits, thr_pos[5..7] = warp bits,
// reg_pos = register bits).  A block is a 4x4 complex matrix on the two qubits held by
// lane bits 0 and 1 (amplitude index a = lane bits 0 + 2 lane bit 1), applied with
// mma.sync m8n8k4 f64 to every register slot.  Between blocks, a lane bit and a register
// bit are exchanged with warp shuffles (PO_SWAP), the lane bits are permuted by one
// indexed shuffle of every register (PO_LPERM), or the tile is redistributed through
// shared memory (PO_RELAYOUT).
constexpr int PR_TILE_BITS = 12;
constexpr int PR_LANE_BITS = 5;
// qubits 0 and 1 are local in every pass (positions 0 and 1) and sit on lane bits when a
// tile is loaded and stored, so that every warp access is made of whole 64-byte runs (two
// full 32-byte sectors).  Forcing qubit 2 as well (128-byte runs) costs more passes and
// moves than it saves in DRAM efficiency; qubit 0 alone (32-byte runs) costs more DRAM time.
constexpr int PR_COAL_BITS = 2;
constexpr int PR_MAX_COND = 2;          // tile-selected variants: at most 2 non-local qubits
enum PairOpKind : uint8_t { PO_SWAP = 0, PO_RELAYOUT = 1, PO_BLOCK = 2, PO_LPERM = 3 };

struct PairOp {                          // 16 bytes
    uint8_t kind;
    uint8_t lane;                        // PO_SWAP: lane bit
    uint8_t reg;                         // PO_SWAP: register bit
    uint8_t ncond;                       // PO_BLOCK: number of condition qubits
    uint8_t cond_q[PR_MAX_COND];         // PO_BLOCK: global qubits selecting the variant
    uint16_t layout;                     // PO_RELAYOUT: target layout
    uint32_t gate;                       // PO_BLOCK: first variant (units of 32 double2);
                                         // PO_LPERM: 3 bits per lane bit b, the lane bit
                                         // whose element moves to lane bit b
    uint16_t src;                        // PO_RELAYOUT: current layout
    uint16_t pad;
};

static_assert(sizeof(PairOp) == 16, "PairOp layout");

struct PairPass {
    uint8_t local_q[PR_TILE_BITS];
    uint8_t nonlocal_q[64 - PR_TILE_BITS];
    int32_t n_nonlocal;
    int32_t op_begin, op_end;
    int32_t load_layout, store_layout;   // the pass's layouts are load_layout..store_layout
    int32_t gate_begin, gate_count;      // its blocks' gate fragments (32 lanes x 16 bytes)
    int32_t stage_gates;                 // whether they are copied into shared memory too
};
static_assert(sizeof(PairPass) % 16 == 0, "PairPass layout");
// Shared memory of a pair CTA: the 64 KiB tile, then the pass's ops, layouts and (when
// they fit) gate fragments, all within what two CTAs per SM can hold.
constexpr size_t PR_SMEM_CAP = 112 * 1024;
// bytes of a pass's ops, layouts and gate fragments in shared memory (16-byte aligned parts)
inline size_t pair_stage_bytes(int n_ops, int n_layouts, int n_gates)
{
    return 16 * (size_t)n_ops + ((24 * (size_t)n_layouts + 15) / 16) * 16 + 512 * (size_t)n_gates;
}

struct PairPlan {
    std::vector<PairPass> passes;
    std::vector<PairOp> ops;
    std::vector<DevStage> layouts;
    std::vector<double> gates;           // per variant: 32 lanes x (B0, B1)
    size_t n_blocks = 0, n_swaps = 0, n_relayouts = 0, n_lane_perms = 0;
    size_t stage_bytes = 0;              // largest per-pass copy into shared memory
};

// 4x4 complex matrix of an F_M4 op, row-major, re/im interleaved (index a = bit0 + 2 bit1)
using Mat4 = std::array<double, 32>;

// Builds the pair plan; false if an op cannot be written as a matrix (SRN).  `mats` holds
// the matrices of F_M4 ops.  With both_cuts, the seeded pass cut is planned as well and the
// cheaper plan kept (about twice the planning time; callers that plan on every call of a
// short circuit, such as the adjoint's forward segments, plan the program-order cut only).
bool plan_pairs(const std::vector<EOp>& ops, int n, PairPlan& plan, const std::vector<Mat4>* mats = nullptr,
                bool both_cuts = true);

struct DevPairBuffers {
    PairPass* passes = nullptr;
    PairOp* ops = nullptr;
    DevStage* layouts = nullptr;
    double* gates = nullptr;
    size_t stage_bytes = 0;
};
cudaError_t launch_pair_pass(void* state, int n, int pass_index, const DevPairBuffers& b, cudaStream_t s);

// The pass cut shared by the staged, pair and adjoint planners: ops in program order are
// taken into a pass of M local qubits (always including the G lowest) while their dense
// or CX target can be made local and they touch no qubit of an op skipped earlier; of the
// cuts that leave out one of the ops that brought new qubits in, the one taking the most
// ops is kept.  With seeds > 1, each of the first `seeds` open ops that could move to the
// front (no earlier open op shares a qubit) is also tried as the one that brings the first
// new qubits in.  `build` receives each pass's local-qubit mask and ops and returns the ops
// it could not place.
void select_passes(const std::vector<EOp>& ops, int n, int M, int G,
                   const std::function<std::vector<int>(uint64_t, const std::vector<int>&)>& build,
                   int seeds = 1);

// ---------------------------------------------------------------------------------
// Fused tensor-core engine (FP32 states): passes of up to FT_MAX_BLOCKS fused k-qubit
// blocks over tiles of 2^FT_TILE_BITS amplitudes (fuse.cpp, kernels_fused.cu)
// ---------------------------------------------------------------------------------
constexpr int FT_TILE_BITS = 12;     // 4096 FP32 amplitudes per tile (32 KiB)
// the 3 lowest qubits are always local: tiles move in whole 64-byte runs (8 amplitudes,
// two 32-byte sectors); forcing a fourth (128-byte runs) costs more passes than it saves
constexpr int FT_LOW_BITS = 3;
constexpr int FT_MAX_BLOCKS = 8;     // upper bound of fused blocks per pass
// Shared memory of a fused CTA: a transpose buffer, an output stage and the raw-tile
// prefetch buffers (32 KiB each), then the pass's gate operands (hi + lo planes,
// 2 (2^(k+1))^2 floats per block).  k = 5 keeps one prefetch buffer and 3 blocks; k <= 4
// two buffers and 5 (k = 4) or 8 (k = 3) blocks, all inside the 227 KiB of one CTA.
__host__ __device__ constexpr int fused_max_blocks(int k) { return k >= 5 ? 3 : (k == 4 ? 5 : 8); }
__host__ __device__ constexpr int fused_raw_buffers(int k) { return k >= 5 ? 1 : 2; }
constexpr int FT_EPI_WARPS = 16;     // warps that move tiles and operands: four per TMEM lane quadrant
constexpr int FT_THREADS = 32 * (FT_EPI_WARPS + 1);   // plus one warp that issues the MMAs
constexpr int FT_MAX_NONLOCAL = 24;  // tile-index bits of a pass (n <= 36)
constexpr int FT_MIN_K = 3, FT_MAX_K = 6;   // 6: one block per pass (kernels_fused6.cu)
constexpr int FT_DEFAULT_K = 5;          // the fastest width on the random circuits measured

// Shared-memory layouts of the fused kernel.  All are linear over GF(2) in the bits they
// index, so tables of them combine by XOR.
//
// Raw tile (a prefetched tile) and output stage (a finished tile): the amplitude of local
// index l sits at word (8-byte slot) l ^ raw_xor[l >> 4] << 1, resp. l ^ out_xor[l >> 4]:
// per 128-byte run (16 amplitudes, local index bits 0..3 = qubits 0..3) an XOR on the
// run's chunk index, resp. on its word index (which may swap the two amplitudes of a
// 16-byte chunk).  The planner picks both per pass (FusedPass) so that the 16 threads of
// a half warp that gather block 0's rows from the raw tile, or scatter the last block's
// rows into the output stage, hit 16 distinct bank pairs.
//
// Transpose buffer: amplitude (row n, target index a) of a k-qubit block at word
// fused_slot(n, a, k): rows of 2^k amplitudes; the 16-byte chunks of a row XOR-swizzled by
// row bits so that the 8 threads of a quarter warp reading one chunk of 8 consecutive rows
// hit 8 bank groups, and the two amplitudes of a chunk swapped by row bit 3.  The bank
// pair of a word (its bits 0..3) takes image 0 from target bit 0 or row bit 3, and images
// 1..3 from target bits 1..3 or row bits 0..2 (k >= 4); for k = 3 from target bits 1, 2 or
// row bits 1, 2, and image 3 from row bit 0.
__host__ __device__ constexpr uint32_t fused_chunk_swizzle(uint32_t n, int k)
{
    return k >= 4 ? (n & 7u) : ((n >> 1) & 3u);
}
__host__ __device__ constexpr uint32_t fused_slot(uint32_t n, uint32_t a, int k)
{
    return (n << k) | ((((a >> 1) ^ fused_chunk_swizzle(n, k)) << 1)) | ((a ^ (n >> 3)) & 1u);
}

struct FusedBlock {                  // 464 bytes
    // where this block's input amplitudes sit in the raw tile (their word there; used for
    // a pass's first block), XOR-combined over the target index and row bits 0-4 and 5-8
    uint16_t a_sc[64];               // target index a
    uint16_t n_lo[32];               // row bits 0-4
    uint16_t n_hi[16];               // row bits 5-8
    // where the amplitudes of this block's output rows go: their slot in the next
    // block's transpose layout (fused_slot of the next block's (row, target index)), or,
    // after the last block, their word in the output stage; XOR-combined over the target
    // index and row bits 0-4 and 5-8
    uint16_t nxt_a[64];              // target index a
    uint16_t nxt_nlo[32];            // row bits 0-4
    uint16_t nxt_nhi[16];            // row bits 5-8
    uint32_t gate_word;              // word offset of the gate operand (hi plane, then lo)
    uint32_t pad[3];
};
static_assert(sizeof(FusedBlock) % 16 == 0, "FusedBlock layout");

struct FusedPass {
    uint8_t local_q[FT_TILE_BITS];
    uint8_t nonlocal_q[64 - FT_TILE_BITS];
    uint64_t g_lo[64];               // local index bits 0-5 -> global amplitude offset
    uint64_t g_hi[64];               // local index bits 6-11 -> global amplitude offset
    uint8_t raw_xor[256];            // per run (local index >> 4): XOR on its chunk index in a raw tile
    uint8_t out_xor[256];            // per run: XOR on its word index in the output stage
    int32_t n_nonlocal, block_begin, n_blocks, pad;
};
static_assert(sizeof(FusedPass) % 16 == 0, "FusedPass layout");

// Fusion width 6 (kernels_fused6.cu): one 6-qubit block per pass, applied in the
// transposed form D^T = G X^T.  The block's real form G (128 x 128: M = 128 rows, the full
// width of one tcgen05.mma) is the A operand and stays in tensor memory for the whole
// launch; the state tile (4,096 amplitudes: the 6 target qubits and the 6 lowest other
// qubits) is the B operand in shared memory, where the loaded FP32 values themselves are
// the hi plane.  A pass is one block: two 6-qubit blocks' hi + lo operands (256 KiB) do
// not fit on one SM.
constexpr int F6_K = 6;
constexpr int F6_TILE_BITS = 12;     // 6 target + 6 row bits: 64 rows of 64 amplitudes
constexpr int F6_ROWS = 64;          // N of the MMA: rows of the tile
constexpr int F6_N = 128;            // real dimension 2^(k+1): M and K of the MMA
constexpr int F6_SLOTS = 3;          // tiles in flight (shared memory: hi + lo plane each)

struct Fused6Pass {                  // one 6-qubit block = one pass
    uint8_t local_q[F6_TILE_BITS];   // the tile's qubits, ascending
    uint8_t nonlocal_q[64 - F6_TILE_BITS];   // tile index bit j <-> nonlocal_q[j]
    // The kernel moves amplitude x = thread + 512 i of a tile (12 bits, mapped onto the
    // local qubits by the planner): its global offset g_lo[x & 63] | g_hi[x >> 6] and its
    // word (8-byte) offset s_lo[x & 63] + s_hi[x >> 6] in a B-operand plane (canonical
    // K-major layout without swizzle, 64 rows: target bit 0 -> 1 word, target bit b > 0
    // -> 128 << (b - 1), row bit b -> 2 << b)
    uint64_t g_lo[64];
    uint64_t g_hi[64];
    uint16_t s_lo[64];
    uint16_t s_hi[64];
    uint64_t o_row[64];              // row index n -> global amplitude offset of its bits
    uint64_t o_tgt[64];              // target index a -> global amplitude offset of its bits
    uint32_t gate_word;              // float offset of G_hi (row-major 128 x 128), G_lo after it
    int32_t n_nonlocal;
    int32_t rows_paired;             // 1 when row bit 0 is qubit 0 (rows 2r, 2r+1 adjacent)
    int32_t pad;
};
static_assert(sizeof(Fused6Pass) % 16 == 0, "Fused6Pass layout");

struct FusedPlan {
    int k = 0;
    std::vector<FusedPass> passes;
    std::vector<FusedBlock> blocks;
    std::vector<Fused6Pass> passes6; // fusion width 6: one block per pass
    std::vector<float> gates;        // per block: hi plane then lo plane, canonical layout
    size_t n_passes() const { return k == F6_K ? passes6.size() : passes.size(); }
};

bool fusable(const std::vector<EOp>& ops);
void plan_fused(const std::vector<EOp>& ops, int n, int k, FusedPlan& plan);
void plan_fused6(const std::vector<EOp>& ops, int n, FusedPlan& plan);

struct DevFusedBuffers {
    FusedPass* passes = nullptr;
    FusedBlock* blocks = nullptr;
    Fused6Pass* passes6 = nullptr;
    float* gates = nullptr;
    int* err = nullptr;
    double* norm_partial = nullptr;      // REDUCE_BLOCKS FP64 partial sums of |a|^2
};
cudaError_t launch_fused_pass(void* state, int n, int k, int pass_index, int n_blocks,
                              int gate_words_per_block, const DevFusedBuffers& b, cudaStream_t s);
cudaError_t launch_fused6_pass(void* state, int n, int pass_index, const DevFusedBuffers& b, cudaStream_t s);

// Self-test of the bounded device waits (selftest.cu, batch.cu): the grid barrier of the
// batched kernels on a target never reached (sets bar[1]); the mbarrier wait of the fused
// kernels on a barrier nothing arrives at (writes 1 to *flag when it gives up).
cudaError_t launch_grid_barrier_probe(unsigned* bar, cudaStream_t s);
cudaError_t launch_mbarrier_probe(int* flag, cudaStream_t s);
// Rescales the FP32 state to unit norm (norm summed in FP64) after a fused run.
cudaError_t launch_fused_renorm(void* state, int n, const DevFusedBuffers& b, cudaStream_t s);

// ---------------------------------------------------------------------------------
// Kernel launchers (kernels_apply.cu)
// ---------------------------------------------------------------------------------
struct DevPlanBuffers {
    DevPass* passes = nullptr;
    DevStage* stages = nullptr;
    DevOp* ops = nullptr;
};

// one elementary op, one sweep (per-gate engine)
template <typename T>
cudaError_t launch_eop(void* state, int n, const EOp& op, cudaStream_t s);
// one staged pass
template <typename T>
cudaError_t launch_staged_pass(void* state, int n, int M, int pass_index,
                               const DevPlanBuffers& b, cudaStream_t s);
template <typename T>
cudaError_t launch_reset(void* state, int n, cudaStream_t s);
template <typename T>
cudaError_t launch_soa_split(const void* state, uint64_t first, uint64_t count,
                             double* re, double* im, cudaStream_t s);
template <typename T>
cudaError_t launch_soa_merge(void* state, uint64_t first, uint64_t count,
                             const double* re, const double* im, cudaStream_t s);

// ---------------------------------------------------------------------------------
// Reductions and measurement (measure.cu)
// ---------------------------------------------------------------------------------
struct MeasureScratch {
    double* cdf = nullptr;          // measurement workspace, measure_layout(n).doubles doubles
    double* uniforms = nullptr;
    uint64_t* samples = nullptr;
    double* partial = nullptr;      // reduction partials
    size_t cap_doubles = 0, cap_shots = 0, cap_partial = 0;
};
constexpr int MEAS_BLOCK_BITS = 12;   // 4096 amplitudes per block
constexpr int MEAS_SUPER_BITS = 6;    // 64 blocks per superblock

// Offsets (in doubles) of the measurement workspace's arrays for a 2^n state.
struct MeasureLayout {
    uint64_t nblocks = 0, nsuper = 0;
    uint64_t off_entry = 0, off_start = 0, off_sentry = 0, off_sstart = 0, off_desc = 0;
    uint64_t doubles = 0;
};
constexpr MeasureLayout measure_layout(int n)
{
    MeasureLayout L;
    const uint64_t dim = 1ull << n;
    L.nblocks = (dim + (1ull << MEAS_BLOCK_BITS) - 1) >> MEAS_BLOCK_BITS;
    L.nsuper = (L.nblocks + (1ull << MEAS_SUPER_BITS) - 1) >> MEAS_SUPER_BITS;
    // block entries | block starts (+ total) | superblock entries |
    // superblock starts (+ total) | descent flags (two 32-bit flags per double)
    L.off_entry = 0;
    L.off_start = L.off_entry + L.nblocks;
    L.off_sentry = L.off_start + L.nblocks + 1;
    L.off_sstart = L.off_sentry + L.nsuper;
    L.off_desc = L.off_sstart + L.nsuper + 1;
    L.doubles = L.off_desc + (L.nsuper + 1) / 2;
    return L;
}

// Samples with the reference's rule on its sequential FP64 prefix, bit for bit
// (measure.cu).  Fails with cudaErrorInvalidValue if scr.cdf holds fewer than
// measure_layout(n).doubles doubles.
template <typename T>
cudaError_t measure_device(const void* state, int n, const double* d_uniforms, uint32_t shots,
                           uint64_t* d_samples, double* d_total, MeasureScratch& scr,
                           cudaStream_t s);
size_t measure_scratch_doubles(int n);
// sum |a|^2 in FP64, summed hierarchically (4096-amplitude blocks, then their scan): the
// accurate norm, not the reference's sequential total (which measure_device reports)
template <typename T>
cudaError_t norm2_device(const void* state, int n, double* d_total, MeasureScratch& scr, cudaStream_t s);
template <typename T>
cudaError_t expectation_device(const void* state, int n, const svb_pauli_term* d_terms,
                               int n_terms, double* d_out, double* d_partial, cudaStream_t s);
constexpr int REDUCE_BLOCKS = 592;   // 4 x 148 SMs
template <typename TA, typename TB>
cudaError_t compare_device(const void* a, const void* b, int n, double* d_out5, double* d_partial5,
                           cudaStream_t s);

// ---------------------------------------------------------------------------------
// Adjoint (adjoint.cu)
// ---------------------------------------------------------------------------------
// A device buffer kept by the handle and reallocated only when a call needs more.
struct GrowBuf {
    void* p = nullptr;
    size_t cap = 0;
};
cudaError_t grow(GrowBuf& b, size_t bytes);
void release(GrowBuf& b);
cudaError_t grow_host(GrowBuf& b, size_t bytes);   // pinned host memory (cudaMallocHost)
void release_host(GrowBuf& b);

// Scratch of svb_adjoint, reused across calls on the same handle.
struct AdjScratch {
    GrowBuf lam, partial, results, terms, final_state;
    GrowBuf host_stage;                             // pinned host staging of plans and results
    int ck_count = -1;                              // checkpoints chosen for ck_bytes-sized states
    size_t ck_bytes = 0;
    GrowBuf plan_passes, plan_stages, plan_ops;     // forward segments' staged plans
    GrowBuf pair_passes, pair_ops, pair_layouts, pair_gates;   // or their pair plans
    GrowBuf rev_passes, rev_ops, rev_slots;         // the tiled reverse sweep's plan
    GrowBuf rev_stages, rev_sops;                   // its register stages (tiles of 10 qubits)
    std::vector<GrowBuf> ckpts;
};

// Runs elementary ops on an FP64 device state, queued on `st`: the pair engine for
// n >= PR_TILE_BITS, the staged engine for 10 <= n < 12 (or when an op has no matrix),
// per-gate sweeps below.  The plan is uploaded into `cache`'s buffers.
svb_status run_eops_fp64(int n, void* state, const std::vector<EOp>& ops, cudaStream_t st,
                         AdjScratch& cache);
void free_adjoint_scratch(AdjScratch& a);
struct Sim;
// Validates gate records against the handle and lowers them to elementary ops (the
// first half of svb_set_circuit, without planning).
svb_status validate_and_lower(Sim* s, const svb_gate* gates, size_t n_gates, std::vector<EOp>& eops,
                              double* sweeps);

// ---------------------------------------------------------------------------------
// The handle
// ---------------------------------------------------------------------------------
struct Sim {
    uint32_t n = 0;
    int device = 0;
    int precision = SVB_FP64;
    void* state = nullptr;         // 2^n interleaved complex amplitudes
    size_t amp_bytes = 16;
    // circuit and plan
    std::vector<svb_gate> gates;
    std::vector<EOp> eops;
    int engine_req = SVB_ENGINE_AUTO, tile_bits_req = 0, fusion_req = 0;
    int engine = SVB_ENGINE_PER_GATE;
    StagedPlan staged;
    DevPlanBuffers dplan;
    FusedPlan fused;
    DevFusedBuffers dfused;
    PairPlan pairs;
    DevPairBuffers dpairs;
    bool have_circuit = false;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t capture_stream = nullptr;
    svb_plan_info info{};
    // scratch
    MeasureScratch mscr;
    double* d_small = nullptr;     // a few doubles for reduction results
    AdjScratch adj;
    std::vector<Mat4> mats;        // matrices of F_M4 ops of the current circuit
    uint32_t dm_qubits = 0;        // density-matrix handle: qubits of rho (state has 2x)
};

void set_error(const std::string& msg);

// Plans and uploads an already lowered circuit on the handle (svb_set_circuit after its
// validation and lowering; the density-matrix entry point with its superoperator blocks).
svb_status set_circuit_lowered(Sim* s, std::vector<EOp>& eops, const svb_gate* gates, size_t n_gates,
                               double sweeps);
// qubit slots a reference op uses (0 for an unknown op)
int gate_qubit_slots(uint32_t op);
// one general 4x4 block (F_M4) as a per-gate sweep
template <typename T>
cudaError_t launch_m4(void* state, int n, int q0, int q1, const Mat4& m, cudaStream_t s);

}  // namespace svb

struct svb_sim : public svb::Sim {};

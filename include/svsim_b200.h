/*
 * svsim_b200.h — C ABI of the B200 state-vector engine (libsvsim_b200.so).
 *
 * This is the boundary that the reference's single-GPU backend
 * (svsim/src/svsim_nvgpu_sin.cuh) crosses into hand-written sm_100a kernels.  The
 * reference's C++ API (class Simulation / class Gate, and the pybind11 module built
 * from svsim/src/py_wrapper.cpp) is kept as a header-only drop-in under
 * include/svsim_dropin/, which calls these functions.  Every entry point below names
 * the reference code it replaces.
 *
 * Conventions
 *   - Plain C types only: host pointers, sizes, and an opaque `void* stream` that is a
 *     cudaStream_t (NULL = the legacy default stream).
 *   - Every function returns an svb_status; SVB_OK is 0.  On failure the reason is
 *     available from svb_last_error() on the calling thread.  Nothing in the library
 *     calls exit() or assert(): invalid gates, qubit indices and sizes are rejected
 *     on the host before any kernel runs.
 *   - Qubit q is bit q of the basis-state index (little-endian), as in the reference.
 *   - A handle owns its device memory and is used from one host thread at a time.
 */
#ifndef SVSIM_B200_H
#define SVSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum svb_status {
    SVB_OK = 0,
    SVB_ERR_INVALID = 1,      /* bad argument, gate, qubit index or size */
    SVB_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    SVB_ERR_OOM = 3,          /* device or host allocation failed */
    SVB_ERR_UNSUPPORTED = 4,  /* valid request this build does not support */
    SVB_ERR_STATE = 5         /* call out of order (e.g. run before a circuit is set) */
} svb_status;

typedef enum svb_precision {
    SVB_FP64 = 0,  /* complex<double> amplitudes: the reference's ValType (config.hpp:42) */
    SVB_FP32 = 1   /* complex<float> amplitudes: fused tensor-core and batched forms */
} svb_precision;

typedef enum svb_engine {
    SVB_ENGINE_AUTO = 0,      /* n >= 12 without SRN: pairs (FP64) or fused (FP32); else
                                 staged for n >= 10 (FP32: 11), per-gate below */
    SVB_ENGINE_PER_GATE = 1,  /* one HBM sweep per elementary gate, as the reference */
    SVB_ENGINE_STAGED = 2,    /* many gates per HBM sweep through a shared-memory tile */
    SVB_ENGINE_FUSED = 3,     /* gates fused into dense k-qubit blocks (FP32 only) */
    SVB_ENGINE_PAIRS = 4      /* FP64 two-qubit blocks on the FP64 tensor cores (FP64, n >= 12,
                                 no SRN) */
} svb_engine;

/* One gate: the fields of the reference's class Gate (svsim_nvgpu_sin.cuh:99-188)
 * without its device function pointer.  `op` is the reference's enum OP value
 * (:42-48, U3 = 0 ... RYY = 37).  48 bytes. */
typedef struct svb_gate {
    uint32_t op;
    uint32_t qb[5];
    double theta, phi, lambda;
} svb_gate;

/* Parameter binding of one gate for the adjoint: for each angle field
 * (0 = theta, 1 = phi, 2 = lambda) the index of the circuit parameter it depends on
 * (-1 = constant) and d(angle)/d(parameter).  40 bytes. */
typedef struct svb_param_binding {
    int32_t idx[3];
    int32_t reserved;
    double coef[3];
} svb_param_binding;

/* One Pauli string of an observable: coef * prod_q sigma_q, where qubit q carries
 * X if only x_mask has bit q, Z if only z_mask has it, Y if both do. */
typedef struct svb_pauli_term {
    double coef;
    uint64_t x_mask;
    uint64_t z_mask;
} svb_pauli_term;

/* Execution statistics of the current plan. */
typedef struct svb_plan_info {
    uint64_t n_gates;          /* gates as given */
    uint64_t n_elementary;     /* elementary ops after expanding composites */
    uint64_t n_passes;         /* kernel launches per run */
    uint64_t n_sweeps_model;   /* per-gate sweep count of the reference (half sweeps x2) */
    double   state_bytes;      /* bytes of the state vector */
    double   model_bytes;      /* per-gate-model algorithmic bytes of one run */
    double   moved_bytes;      /* bytes the plan reads+writes in HBM per run */
    uint64_t plan_bytes;       /* bytes of plan descriptors uploaded by svb_set_circuit */
    int      engine;           /* engine the plan was built for */
    int      tile_bits;        /* local qubits per tile (staged engine) */
    uint64_t n_blocks;         /* tensor-core blocks per run: two-qubit blocks of the pair
                                  engine, fused blocks of the fused engine; 0 otherwise */
} svb_plan_info;

typedef struct svb_sim svb_sim;

/* ---- lifetime ------------------------------------------------------------------- */

/* Replaces Simulation::Simulation (svsim_nvgpu_sin.cuh:193-225): selects `device`,
 * allocates the 2^n-amplitude state on it and sets |0..0>.  Unlike the reference no
 * host copy of the state is kept.  n_qubits in [1, 36]. */
svb_status svb_create(uint32_t n_qubits, int device, int precision, svb_sim** out);

/* Replaces Simulation::~Simulation (:227-237). NULL is accepted. */
svb_status svb_destroy(svb_sim* sim);

/* Replaces Simulation::reset_sv (:243-255): state <- |0..0>, on the device. */
svb_status svb_reset_state(svb_sim* sim);

/* ---- circuit -------------------------------------------------------------------- */

/* Replaces Simulation::append + Simulation::upload (:257-294): validates the gate list
 * on the host (op in range, qubits < n, distinct qubits within a gate), expands the
 * composites into the reference's elementary sequences (:1134-1454), plans the
 * kernel passes and uploads the plan.  Replaces any previous circuit. */
svb_status svb_set_circuit(svb_sim* sim, const svb_gate* gates, size_t n_gates);

/* Replaces Simulation::clear_circuit (:341-358). The state is kept. */
svb_status svb_clear_circuit(svb_sim* sim);

/* Chooses the execution engine (svb_engine) for the next svb_set_circuit; tile_bits
 * (0 = automatic) and fusion_width (0 = automatic: 5; else 3..6, where 6 runs one block
 * per pass) tune the staged and fused engines. */
svb_status svb_set_engine(svb_sim* sim, int engine, int tile_bits, int fusion_width);

/* Result of svb_autotune. */
typedef struct svb_tune_result {
    int engine;               /* svb_engine chosen */
    int tile_bits;            /* staged engine: local qubits per tile (0 otherwise) */
    int fusion_width;         /* fused engine: qubits per fused block (0 otherwise) */
    int candidates;           /* configurations timed */
    double best_ms;           /* time of the chosen configuration on the timed gates */
    double default_ms;        /* time of the static AUTO choice on the same gates (-1 if it failed) */
    uint64_t timed_gates;     /* gates timed: the circuit's first min(n_gates, 360) */
} svb_tune_result;

/* Autotuner (no reference counterpart; the reference fixes its launch shape,
 * svsim_nvgpu_sin.cuh:309-316, config.hpp:48): times every engine configuration that can
 * run the circuit on this handle (per-gate for n <= 26; staged at each tile size; the pair
 * engine for FP64 or the fused engine at k = 3..6 for FP32, when the circuit has no SRN)
 * on its first min(n_gates, 360) gates, one warm-up and one timed run each, and keeps the
 * fastest for this circuit structure (qubit count, precision, and the ops and qubits of
 * every elementary op; angles ignored): from then on svb_set_circuit with
 * SVB_ENGINE_AUTO picks it for any circuit of that structure on this device.  The handle
 * ends with `gates` set as its circuit and the state at |0..0>.  `out` may be NULL. */
svb_status svb_autotune(svb_sim* sim, const svb_gate* gates, size_t n_gates, svb_tune_result* out);

/* Statistics of the current plan. */
svb_status svb_get_plan_info(const svb_sim* sim, svb_plan_info* out);

/* ---- execution ------------------------------------------------------------------ */

/* Replaces Simulation::sim (:306-339) minus its full-state device-to-host copy:
 * applies the current circuit to the device state, asynchronously on `stream`. */
svb_status svb_run(svb_sim* sim, void* stream);

/* Blocks until all work of this handle's device is done; reports kernel errors. */
svb_status svb_synchronize(svb_sim* sim);

/* ---- state access --------------------------------------------------------------- */

/* The device-to-host copy at the end of Simulation::sim (:328-329): writes the state
 * as the reference's SoA host arrays sv_real_cpu / sv_imag_cpu (2^n doubles each;
 * FP32 states are widened).  Either pointer may be NULL. */
svb_status svb_get_state_soa(svb_sim* sim, double* re, double* im);

/* Loads an SoA host state (for tests and restarts; no reference counterpart). */
svb_status svb_set_state_soa(svb_sim* sim, const double* re, const double* im);

/* Device address of the interleaved (re, im) amplitude array and its precision. */
svb_status svb_state_device_ptr(svb_sim* sim, void** dptr, int* precision);

/* ---- measurement ---------------------------------------------------------------- */

/* Replaces Simulation::measure (:359-383) with the uniforms supplied by the caller
 * instead of rand(): shot s returns the j with S_j <= uniforms[s] < S_{j+1}, and 0 if
 * there is no such j — the reference's rule, including its default of 0.  S is the
 * reference's own prefix, bit for bit: S_0 = 0, S_{i+1} = fl(S_i + fl(fl(re_i^2) +
 * fl(im_i^2))) summed in index order in FP64 (:362-365).  The GPU computes those
 * sequential values exactly without a sequential pass (integer grid deltas inside a
 * binade, IEEE adds one by one at ties and binade crossings) and without a 2^n scan
 * array, so any uniform, including one equal to some S_j or next to it, gives the
 * reference's sample for the same state.  prob_total (may be NULL) receives S_{2^n}. */
svb_status svb_measure(svb_sim* sim, const double* uniforms, uint32_t shots,
                       uint64_t* out, double* prob_total);

/* Simulation::measure (:359-383) itself, with a seed in place of its time(0): seeds the
 * C library generator with srand(seed) and draws shot s as rand() / RAND_MAX, in shot
 * order, as the reference does after srand(time(0)); then samples as svb_measure.  The
 * same seed gives the reference's samples for the same state.  Like the reference, it
 * reseeds the process-wide rand() sequence (not thread-safe). */
svb_status svb_measure_seeded(svb_sim* sim, uint32_t seed, uint32_t shots, uint64_t* out,
                              double* prob_total);

/* Self-test of the bounded waits the persistent kernels rely on (no reference counterpart:
 * the reference's grid.sync() in simulation_kernel, svsim_nvgpu_sin.cuh:614-621, waits
 * without limit).  One kernel waits on an mbarrier nothing arrives at, with the fused
 * engines' tensor-core completion wait (it gives up after 2 s); one waits at a grid
 * barrier whose arrival count is never reached, with the batched engines' barrier (it
 * gives up after more than 1 s).  Each must give up and report it, and the context must
 * stay usable: *mbar_timed_out and *grid_timed_out receive 1 when the wait gave up. */
svb_status svb_selftest_waits(int device, int* mbar_timed_out, int* grid_timed_out);

/* Largest state size svb_measure_noalloc accepts. */
#define SVB_NOALLOC_MAX_QUBITS 30

/* Measurement that allocates nothing (no counterpart in the reference).  Same sampling
 * rule and results as svb_measure, for callers that cannot allocate device memory: an
 * application whose device memory is fully reserved by its own pool, or one that owns
 * the state buffer and wants no hidden cudaMalloc/cudaFree.  Every pointer is a device
 * pointer on the current device: `state` (2^n_qubits interleaved amplitudes of
 * `precision`), `uniforms` and `samples` (`shots` entries each) and `prob_total` (one
 * double, may be NULL).  Work is queued on `stream`; results are valid once it completes.
 * The FP64 scratch lives in a fixed array of about 4.1 MiB in the library's device image,
 * sized for n_qubits <= SVB_NOALLOC_MAX_QUBITS; larger states are rejected with
 * SVB_ERR_INVALID.  The first call on a device looks the array's address up
 * (cudaGetSymbolAddress), so make that first call before any stream capture.  Modules
 * load lazily by default (CUDA 12.2+): the first call also loads the module that holds
 * the array and commits its memory, so a caller that later reserves the whole device
 * should make one call first (shots = 0 is enough) or set CUDA_MODULE_LOADING=EAGER.
 * All calls on a device share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  Nothing needs clearing between calls (the kernels
 * overwrite what they read). */
svb_status svb_measure_noalloc(const void* state, uint32_t n_qubits, int precision,
                               const double* uniforms, uint32_t shots, uint64_t* samples,
                               double* prob_total, void* stream);

/* Squared norm sum |a|^2 in FP64, summed hierarchically (blocks of 4,096 amplitudes, then
 * their prefix): accurate to a few ulps.  The reference's own check against 1 (:379) uses
 * its sequential prefix total, which svb_measure returns as prob_total and which can lose
 * ~1e-10 at 2^31 amplitudes when many probabilities are below half an ulp of the sum. */
svb_status svb_norm2(svb_sim* sim, double* out);

/* Re <psi| sum_t coef_t P_t |psi> in FP64 for a Pauli-sum observable. */
svb_status svb_expectation(svb_sim* sim, const svb_pauli_term* terms, size_t n_terms,
                           double* out);

/* Compares the states of two handles of equal size and device, either precision:
 * fidelity = |<a|b>|^2 / (<a|a><b|b>) and max_i |a_i - b_i|, both in FP64 (the
 * accuracy report of the FP32 engines against FP64; no reference counterpart). */
svb_status svb_compare_states(svb_sim* a, svb_sim* b, double* fidelity, double* max_abs_diff);

/* ---- immediate-mode operations of the Q#/QIR variant ---------------------------- */

/* Replaces the masked multi-controlled gates of svsim_qsharp/svsim_nvgpu_sin.cuh
 * (ControlledX ... ControlledAdjointT, OP_HEAD_MASK :680-690): applies the 2x2 complex
 * matrix m (row-major, re/im interleaved: m00r m00i m01r m01i m10r m10i m11r m11i) to
 * `target` on the amplitudes whose control_mask bits are all 1, at once on `stream`
 * (not part of the circuit).  The target may not be in the mask. */
svb_status svb_apply_controlled(svb_sim* sim, uint32_t target, uint64_t control_mask, const double* m,
                                void* stream);

/* Replaces Measure_GATE of the Q# variant (:1486-1600): measures `qubit` in the Pauli
 * basis `pauli` (0 = Z, 1 = X, 2 = Y) and collapses the state on the GPU.  The outcome is
 * 1 when the caller's uniform r < P(1) (P(1) summed in FP64); the other half is zeroed
 * and the kept half scaled by 1/sqrt(P(outcome)).  Writes the outcome and P(1). */
svb_status svb_measure_qubit(svb_sim* sim, uint32_t qubit, int pauli, double r, int* outcome,
                             double* prob_one);

/* ---- density matrices with noise (the reference's svsim_qsharp_noise variant) ----- */

/* A density-matrix handle for rho of n_qubits qubits (1..17): an FP64 state of 2 n_qubits
 * qubits holding rho[i][j] at index i + 2^n j (the noise variant's layout, dim 2^(2n) at
 * svsim_qsharp_noise/svsim_nvgpu_sin.cuh:527-529), set to |0..0><0..0|.  svb_run,
 * svb_reset_state and svb_destroy apply to it; svb_norm2 gives Tr(rho^2). */
svb_status svb_dm_create(uint32_t n_qubits, int device, svb_sim** out);

/* The circuit of a density-matrix handle: every gate U becomes rho -> U rho U^dagger, and
 * when n_kraus > 0 the one-qubit channel with Kraus operators noise_kraus (n_kraus 2x2
 * complex matrices, row-major, re/im interleaved: 8 doubles each) is applied after every
 * gate to each qubit the gate touches (the variant's noisy gates, a superoperator per
 * gate).  SRN has no superoperator and is rejected. */
svb_status svb_dm_set_circuit(svb_sim* sim, const svb_gate* gates, size_t n_gates,
                              const double* noise_kraus, uint32_t n_kraus);

/* The superoperator of a one-qubit op in a density-matrix circuit, as the noise
 * variant bakes noise into its gates (svsim_qsharp_noise/noise_gate_*.cuh tables, applied
 * by C2_GATE, svsim_qsharp_noise/svsim_nvgpu_sin.cuh:1727-1800): `op` is the enum OP value
 * of a one-qubit gate and m the 4x4 complex matrix e_rc, row-major, re/im interleaved,
 * acting as out[r] = sum_c e_rc in[c] on the local index r = 2 i + j of rho[i][j] for the
 * gate's qubit (C2_GATE's pos0..pos3 on the pair (qubit, qubit + n_qubits)).  280 bytes. */
typedef struct svb_superop {
    uint32_t op;
    uint32_t reserved;
    double m[32];
} svb_superop;

/* svb_dm_set_circuit with per-op superoperators: every gate whose op has an entry in
 * `superops` is applied as that superoperator alone (it replaces rho -> U rho U^dagger and
 * the Kraus noise after the gate, as the reference's noisy gates do); the other gates as
 * in svb_dm_set_circuit. */
svb_status svb_dm_set_circuit_superops(svb_sim* sim, const svb_gate* gates, size_t n_gates,
                                       const double* noise_kraus, uint32_t n_kraus,
                                       const svb_superop* superops, size_t n_superops);

/* The diagonal of rho (the outcome probabilities), 2^n_qubits doubles, to the host. */
svb_status svb_dm_probabilities(svb_sim* sim, double* out);

/* ---- differentiation (no reference counterpart) --------------------------------- */

/* Adjoint differentiation of E(p) = <psi(p)| H |psi(p)>, psi(p) = U(p)|0..0>:
 * runs the circuit forward from |0..0>, forms lambda = H psi, then walks the
 * elementary ops backwards applying U^dagger to psi and lambda while accumulating
 * grad[binding.idx] += 2 Re <lambda| dU/dp |psi_prev> * binding.coef in FP64.
 * `gates` carry the angle values at the current parameters; `bindings` (one per gate)
 * say which angles depend on which of the n_params parameters.  Writes energy (may
 * be NULL) and grad[n_params].  The handle's state is left holding psi(p); its circuit
 * and plan (svb_set_circuit) are not changed. */
svb_status svb_adjoint(svb_sim* sim, const svb_gate* gates, const svb_param_binding* bindings,
                       size_t n_gates, uint32_t n_params, const svb_pauli_term* terms,
                       size_t n_terms, double* energy, double* grad);

/* ---- batched QAOA (no reference counterpart) ------------------------------------ */

/* A batch of weighted MaxCut QAOA instances evaluated together: for each instance the
 * cost expectation E = <psi|C|psi> and its gradient with respect to the 2p angles.
 * Instance i has n_qubits[i] qubits and the edges edge_offsets[i] .. edge_offsets[i+1]-1
 * of `edges` (pairs a, b) with `weights`.  Its circuit is what the reference builds from
 * H on every qubit, then per layer l RZZ(-gamma_l w_e) on every edge (:1288-1294) and
 * RX(2 beta_l) on every qubit (:1085-1100); C(z) = sum_e w_e [z_a != z_b]. */
typedef struct svb_qaoa_batch svb_qaoa_batch;

typedef struct {
    uint32_t n_instances;
    uint32_t p;
    uint32_t tile_bits;          /* log2 amplitudes per tile of the batched kernel */
    uint32_t graphed;            /* 1 if svb_qaoa_run replays a CUDA graph */
    uint64_t total_amplitudes;   /* sum over instances of 2^n */
    uint64_t tiles_per_pass;
    double moved_bytes;          /* state and cost-table bytes one evaluation reads and writes */
    uint32_t grid;               /* resident blocks of the persistent launch */
    uint32_t reserved;
} svb_qaoa_stats;

/* Builds the batch on `device`: uploads the graphs, computes every instance's cost
 * table and captures one evaluation (parameters in, one cooperative launch, results
 * out) as a CUDA graph.  Each instance has 2 <= n <= 24 qubits (FP64) or 26 (FP32) and at
 * most 512 edges; edge_offsets has n_instances + 1 entries starting at 0. */
svb_status svb_qaoa_create(int device, int precision, uint32_t n_instances, const uint32_t* n_qubits,
                           const uint32_t* edge_offsets, const uint32_t* edges, const double* weights,
                           uint32_t p, svb_qaoa_batch** out);

/* One evaluation at gammas[i*p + l], betas[i*p + l] (host arrays).  Writes energies[i]
 * and grads[i*2p + l] = dE_i/dgamma_l, grads[i*2p + p + l] = dE_i/dbeta_l (either may be
 * NULL).  Blocks until the results are on the host. */
svb_status svb_qaoa_run(svb_qaoa_batch* batch, const double* gammas, const double* betas,
                        double* energies, double* grads);

/* Queues the evaluation kernel alone on `stream`, with the parameters of the last
 * svb_qaoa_run and results left on the device (for timing the kernel by itself). */
svb_status svb_qaoa_launch(svb_qaoa_batch* batch, void* stream);

svb_status svb_qaoa_info(const svb_qaoa_batch* batch, svb_qaoa_stats* info);

svb_status svb_qaoa_destroy(svb_qaoa_batch* batch);

/* ---- batched circuits (no reference counterpart) ----------------------------------- */

/* Many independent circuits, each on its own state of n_qubits[i] qubits (1..24, sizes
 * mixed freely), run from |0..0> together by one persistent cooperative launch replayed
 * from a CUDA graph; replaces one Simulation and one sim() per circuit
 * (svsim_nvgpu_sin.cuh:193-339) with its fixed launch shape (:309-316, config.hpp:48).
 * Circuit i's gates are gates[gate_offsets[i] .. gate_offsets[i+1]); its observable (may be
 * empty) terms[term_offsets[i] .. term_offsets[i+1]) (term_offsets may be NULL: no
 * energies).  tile_bits: the local qubits of a shared-memory sweep tile (6..12 FP64, 6..13
 * FP32), every op one sweep of the tile; SVB_CBATCH_PAIRS = the pair engine (FP64
 * two-qubit blocks on the tensor cores, 4,096-amplitude tiles) for every FP64 circuit of
 * 12 or more qubits it can run (no SRN), 12-qubit sweep tiles for the others; 0 = chosen by
 * the autotuner: these candidates (three tile sizes and two block sizes of the sweep, and
 * the pair engine) are timed on the batch itself and the fastest kept; the choice is cached
 * per batch shape (precision, device, qubit and gate counts) for later batches of that
 * shape. */
#define SVB_CBATCH_PAIRS (-1)

typedef struct svb_circuit_batch svb_circuit_batch;

typedef struct {
    uint32_t n_circuits;
    uint32_t n_phases;            /* grid-wide phases of one launch */
    uint32_t tile_bits;           /* local qubits of a work tile */
    uint32_t threads;             /* threads per CTA */
    uint64_t pool_amplitudes;     /* sum over circuits of 2^n */
    uint64_t items;               /* (circuit, pass, tile) work items of one run */
    uint32_t grid;                /* resident CTAs of the persistent launch */
    uint32_t graphed;             /* 1 if a run replays a CUDA graph */
    double moved_bytes;           /* state bytes one run reads and writes (passes x 2 x state) */
    uint32_t tuned;               /* 1 if the autotuner chose tile_bits and threads */
    uint32_t n_passes;            /* sweep passes of all circuits */
    uint32_t pair_circuits;       /* circuits run by the pair engine */
    uint32_t pair_passes;         /* their passes */
    uint32_t pair_phases;         /* phases of the pair launch */
    uint32_t pair_grid;           /* resident CTAs of the pair launch */
} svb_cbatch_stats;

svb_status svb_cbatch_create(int device, int precision, uint32_t n_circuits, const uint32_t* n_qubits,
                             const uint64_t* gate_offsets, const svb_gate* gates,
                             const uint64_t* term_offsets, const svb_pauli_term* terms,
                             int tile_bits, svb_circuit_batch** out);

/* Runs every circuit from |0..0> and writes energies[i] = Re <psi_i| H_i |psi_i> (0 for a
 * circuit without terms; energies may be NULL).  `gates` NULL runs the gates given at
 * creation; otherwise the same gate structure (ops and qubits) with new angles, e.g.
 * another set of parameters.  Blocks until the energies are on the host. */
svb_status svb_cbatch_run(svb_circuit_batch* batch, const svb_gate* gates, double* energies);

/* The final state of one circuit of the last run, as SoA host arrays (2^n doubles each). */
svb_status svb_cbatch_get_state(svb_circuit_batch* batch, uint32_t circuit, double* re, double* im);

svb_status svb_cbatch_info(const svb_circuit_batch* batch, svb_cbatch_stats* out);

svb_status svb_cbatch_destroy(svb_circuit_batch* batch);

/* ---- diagnostics ---------------------------------------------------------------- */

/* Message of the last failed call on this thread ("" if none). */
const char* svb_last_error(void);

/* Library version string. */
const char* svb_version(void);

/* No reference counterpart (a measurement helper): times a register-only loop of FP64
 * tensor-core MMAs (mma.sync m8n8k4 f64, 8 independent chains per warp) on `device` for a
 * few milliseconds and writes the rate in TFLOP/s: the bound of the pair engine's blocks. */
svb_status svb_fp64_mma_peak(int device, double* tflops);

/* No reference counterpart (a measurement helper): the L2 copy bandwidth of `device` in
 * GB/s (read + write bytes), from a copy between two 16 MiB buffers repeated inside one
 * launch: the bound of states small enough to stay in L2. */
svb_status svb_l2_copy_peak(int device, double* gbs);

#ifdef __cplusplus
}
#endif

#endif /* SVSIM_B200_H */

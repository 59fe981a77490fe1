// C ABI of libsvsim_b200 (declared in include/svsim_b200.h).
//
// Host-side runtime of the engine: argument validation (the reference asserts or
// exits instead, svsim_nvgpu_sin.cuh:259-264, util_nvgpu.cuh:29-65), lowering and
// planning of the circuit, plan upload, launch sequencing (optionally replayed from a
// CUDA graph), state transfer and measurement.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <string>

#include "svb_internal.h"

namespace svb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

namespace {

svb_status cuda_fail(cudaError_t e, const char* what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    set_error(m);
    (void)cudaGetLastError();   // clear a sticky launch error where possible
    return e == cudaErrorMemoryAllocation ? SVB_ERR_OOM : SVB_ERR_CUDA;
}

#define SVB_CUDA(call, what)                                   \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, what);     \
    } while (0)

svb_status invalid(const std::string& msg)
{
    set_error(msg);
    return SVB_ERR_INVALID;
}

template <typename F>
cudaError_t dispatch_prec(int precision, F&& f)
{
    if (precision == SVB_FP64) return f(double(0));
    return f(float(0));
}

int n_qubit_slots(uint32_t op)
{
    static const int slots[38] = {
        1, 1, 1, 2, 1, 1, 1, 1, 1, 1,
        1, 1, 1, 1, 1, 1, 2, 2, 2, 2,
        3, 3, 2, 2, 2, 2, 2, 2, 2, 3,
        4, 4, 4, 5, 1, 1, 1, 2};
    return op < 38 ? slots[op] : 0;
}

void free_plan(Sim* s)
{
    if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
    cudaFree(s->dplan.passes);
    cudaFree(s->dplan.stages);
    cudaFree(s->dplan.ops);
    s->dplan = DevPlanBuffers{};
    s->staged = StagedPlan{};
    cudaFree(s->dfused.passes);
    cudaFree(s->dfused.blocks);
    cudaFree(s->dfused.passes6);
    cudaFree(s->dfused.gates);
    cudaFree(s->dfused.err);
    cudaFree(s->dfused.norm_partial);
    s->dfused = DevFusedBuffers{};
    cudaFree(s->dpairs.passes);
    cudaFree(s->dpairs.ops);
    cudaFree(s->dpairs.layouts);
    cudaFree(s->dpairs.gates);
    s->dpairs = DevPairBuffers{};
    s->pairs = PairPlan{};
    s->fused = FusedPlan{};
    s->eops.clear();
    s->gates.clear();
    s->have_circuit = false;
    std::memset(&s->info, 0, sizeof(s->info));
}

void free_scratch(Sim* s)
{
    free_adjoint_scratch(s->adj);
    cudaFree(s->mscr.cdf);
    cudaFree(s->mscr.uniforms);
    cudaFree(s->mscr.samples);
    cudaFree(s->mscr.partial);
    s->mscr = MeasureScratch{};
}

svb_status ensure_scratch(Sim* s, size_t shots)
{
    const size_t nb = measure_scratch_doubles((int)s->n);
    if (s->mscr.cap_doubles < nb) {
        cudaFree(s->mscr.cdf);
        s->mscr.cdf = nullptr;
        s->mscr.cap_doubles = 0;
        SVB_CUDA(cudaMalloc(&s->mscr.cdf, nb * sizeof(double)), "cudaMalloc(measurement workspace)");
        s->mscr.cap_doubles = nb;
    }
    if (s->mscr.cap_shots < shots) {
        cudaFree(s->mscr.uniforms);
        cudaFree(s->mscr.samples);
        s->mscr.uniforms = nullptr;
        s->mscr.samples = nullptr;
        s->mscr.cap_shots = 0;
        SVB_CUDA(cudaMalloc(&s->mscr.uniforms, shots * sizeof(double)), "cudaMalloc(uniforms)");
        SVB_CUDA(cudaMalloc(&s->mscr.samples, shots * sizeof(uint64_t)), "cudaMalloc(samples)");
        s->mscr.cap_shots = shots;
    }
    if (s->mscr.cap_partial < (size_t)REDUCE_BLOCKS) {
        SVB_CUDA(cudaMalloc(&s->mscr.partial, REDUCE_BLOCKS * sizeof(double)), "cudaMalloc(partials)");
        s->mscr.cap_partial = REDUCE_BLOCKS;
    }
    return SVB_OK;
}

int pick_tile_bits(const Sim* s)
{
    const int n = (int)s->n;
    if (s->tile_bits_req > 0) return s->tile_bits_req;
    if (s->precision == SVB_FP64) {
        if (n >= 20) return 12;
        if (n >= 12) return 10;
        return n;                 // 10 or 11: a single tile
    }
    if (n >= 20) return 13;
    if (n >= 13) return 11;
    return n;
}

bool staged_supported(int precision, int M)
{
    if (precision == SVB_FP64) return M >= 10 && M <= 12;
    return M >= 11 && M <= 13;
}

svb_status launch_all(Sim* s, cudaStream_t st)
{
    const int n = (int)s->n;
    if (s->engine == SVB_ENGINE_FUSED) {
        const FusedPlan& F = s->fused;
        if (F.k == F6_K) {
            for (size_t p = 0; p < F.passes6.size(); p++) {
                cudaError_t e = launch_fused6_pass(s->state, n, (int)p, s->dfused, st);
                if (e != cudaSuccess) return cuda_fail(e, "fused pass launch");
            }
        } else {
            for (size_t p = 0; p < F.passes.size(); p++) {
                cudaError_t e = launch_fused_pass(s->state, n, F.k, (int)p, F.passes[p].n_blocks, 0,
                                                  s->dfused, st);
                if (e != cudaSuccess) return cuda_fail(e, "fused pass launch");
            }
        }
        if (F.n_passes() > 0) {
            cudaError_t e = launch_fused_renorm(s->state, n, s->dfused, st);
            if (e != cudaSuccess) return cuda_fail(e, "fused renormalisation");
        }
        return SVB_OK;
    }
    if (s->engine == SVB_ENGINE_PAIRS) {
        for (size_t p = 0; p < s->pairs.passes.size(); p++) {
            cudaError_t e = launch_pair_pass(s->state, n, (int)p, s->dpairs, st);
            if (e != cudaSuccess) return cuda_fail(e, "pair pass launch");
        }
        return SVB_OK;
    }
    if (s->engine == SVB_ENGINE_STAGED) {
        for (size_t p = 0; p < s->staged.passes.size(); p++) {
            cudaError_t e = dispatch_prec(s->precision, [&](auto t) {
                using T = decltype(t);
                return launch_staged_pass<T>(s->state, n, s->staged.M, (int)p, s->dplan, st);
            });
            if (e != cudaSuccess) return cuda_fail(e, "staged pass launch");
        }
    } else {
        for (const EOp& op : s->eops) {
            cudaError_t e = dispatch_prec(s->precision, [&](auto t) {
                using T = decltype(t);
                if (op.form == F_M4) return launch_m4<T>(s->state, n, (int)op.q, (int)op.c, s->mats[op.mat], st);
                return launch_eop<T>(s->state, n, op, st);
            });
            if (e != cudaSuccess) return cuda_fail(e, "gate launch");
        }
    }
    return SVB_OK;
}

bool use_graph(const Sim* s)
{
    static const bool disabled = std::getenv("SVB_NO_GRAPH") != nullptr;
    if (disabled) return false;
    return s->info.n_passes >= 4;
}

}  // namespace

int gate_qubit_slots(uint32_t op) { return n_qubit_slots(op); }

cudaError_t grow(GrowBuf& b, size_t bytes)
{
    if (b.cap >= bytes && b.p) return cudaSuccess;
    cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    const cudaError_t e = cudaMalloc(&b.p, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) b.cap = std::max<size_t>(bytes, 16);
    else b.p = nullptr;
    return e;
}

void release(GrowBuf& b)
{
    cudaFree(b.p);
    b = GrowBuf{};
}

cudaError_t grow_host(GrowBuf& b, size_t bytes)
{
    if (b.cap >= bytes && b.p) return cudaSuccess;
    cudaFreeHost(b.p);
    b.p = nullptr;
    b.cap = 0;
    const size_t want = std::max<size_t>(bytes, 4096);
    const cudaError_t e = cudaMallocHost(&b.p, want);
    if (e == cudaSuccess) b.cap = want;
    else b.p = nullptr;
    return e;
}

void release_host(GrowBuf& b)
{
    cudaFreeHost(b.p);
    b = GrowBuf{};
}

void free_adjoint_scratch(AdjScratch& a)
{
    release(a.lam);
    release(a.partial);
    release(a.results);
    release(a.terms);
    release(a.final_state);
    release(a.plan_passes);
    release(a.plan_stages);
    release(a.plan_ops);
    release(a.pair_passes);
    release(a.pair_ops);
    release(a.pair_layouts);
    release(a.pair_gates);
    release(a.rev_passes);
    release(a.rev_ops);
    release(a.rev_slots);
    release(a.rev_stages);
    release(a.rev_sops);
    release_host(a.host_stage);
    for (GrowBuf& b : a.ckpts) release(b);
    a.ckpts.clear();
    a.ck_count = -1;
    a.ck_bytes = 0;
}

svb_status run_eops_fp64(int n, void* state, const std::vector<EOp>& ops, cudaStream_t st, AdjScratch& cache)
{
    PairPlan R;
    if (n >= PR_TILE_BITS && plan_pairs(ops, n, R)) {
        if (R.passes.empty()) return SVB_OK;
        // the previous segment's kernels may still read the plan buffers: wait before reuse
        cudaError_t e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = grow(cache.pair_passes, R.passes.size() * sizeof(PairPass));
        if (e == cudaSuccess) e = grow(cache.pair_ops, std::max<size_t>(1, R.ops.size()) * sizeof(PairOp));
        if (e == cudaSuccess) e = grow(cache.pair_layouts, std::max<size_t>(1, R.layouts.size()) * sizeof(DevStage));
        if (e == cudaSuccess) e = grow(cache.pair_gates, std::max<size_t>(2, R.gates.size()) * sizeof(double));
        DevPairBuffers b;
        b.passes = static_cast<PairPass*>(cache.pair_passes.p);
        b.ops = static_cast<PairOp*>(cache.pair_ops.p);
        b.layouts = static_cast<DevStage*>(cache.pair_layouts.p);
        b.gates = static_cast<double*>(cache.pair_gates.p);
        b.stage_bytes = R.stage_bytes;
        if (e == cudaSuccess)
            e = cudaMemcpy(b.passes, R.passes.data(), R.passes.size() * sizeof(PairPass), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !R.ops.empty())
            e = cudaMemcpy(b.ops, R.ops.data(), R.ops.size() * sizeof(PairOp), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !R.layouts.empty())
            e = cudaMemcpy(b.layouts, R.layouts.data(), R.layouts.size() * sizeof(DevStage), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !R.gates.empty())
            e = cudaMemcpy(b.gates, R.gates.data(), R.gates.size() * sizeof(double), cudaMemcpyHostToDevice);
        for (size_t p = 0; e == cudaSuccess && p < R.passes.size(); p++)
            e = launch_pair_pass(state, n, (int)p, b, st);
        if (e != cudaSuccess) return cuda_fail(e, "pair run");
        return SVB_OK;
    }
    const int M = n >= 20 ? 12 : (n >= 12 ? 10 : n);
    if (M < 10) {
        for (const EOp& op : ops) {
            cudaError_t e = launch_eop<double>(state, n, op, st);
            if (e != cudaSuccess) return cuda_fail(e, "gate launch");
        }
        return SVB_OK;
    }
    StagedPlan P;
    plan_staged(ops, n, M, 3, P);
    if (P.passes.empty()) return SVB_OK;
    // the previous segment's kernels may still read the plan buffers: wait before reuse
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = grow(cache.plan_passes, P.passes.size() * sizeof(DevPass));
    if (e == cudaSuccess) e = grow(cache.plan_stages, std::max<size_t>(1, P.stages.size()) * sizeof(DevStage));
    if (e == cudaSuccess) e = grow(cache.plan_ops, std::max<size_t>(1, P.ops.size()) * sizeof(DevOp));
    DevPlanBuffers b;
    b.passes = static_cast<DevPass*>(cache.plan_passes.p);
    b.stages = static_cast<DevStage*>(cache.plan_stages.p);
    b.ops = static_cast<DevOp*>(cache.plan_ops.p);
    if (e == cudaSuccess)
        e = cudaMemcpy(b.passes, P.passes.data(), P.passes.size() * sizeof(DevPass), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !P.stages.empty())
        e = cudaMemcpy(b.stages, P.stages.data(), P.stages.size() * sizeof(DevStage), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !P.ops.empty())
        e = cudaMemcpy(b.ops, P.ops.data(), P.ops.size() * sizeof(DevOp), cudaMemcpyHostToDevice);
    for (size_t p = 0; e == cudaSuccess && p < P.passes.size(); p++)
        e = launch_staged_pass<double>(state, n, M, (int)p, b, st);
    if (e != cudaSuccess) return cuda_fail(e, "staged run");
    return SVB_OK;
}

}  // namespace svb

using namespace svb;

namespace svb {

// Checks every gate record against the handle (op known, qubits < n, no repeats; the
// reference asserts qb0..qb4 < n_qubits for every gate, :259-264) and lowers the
// circuit to elementary ops; `sweeps` gets the reference's per-gate sweep count.
svb_status validate_and_lower(Sim* s, const svb_gate* gates, size_t n_gates, std::vector<EOp>& eops,
                              double* sweeps)
{
    if (n_gates > 0 && !gates) return invalid("svb_set_circuit: gates is NULL");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    for (size_t i = 0; i < n_gates; i++) {
        const svb_gate& g = gates[i];
        const int k = n_qubit_slots(g.op);
        if (k == 0) return invalid("gate " + std::to_string(i) + ": unknown op " + std::to_string(g.op));
        for (int j = 0; j < 5; j++)
            if (g.qb[j] >= s->n)
                return invalid("gate " + std::to_string(i) + ": qubit index " +
                               std::to_string(g.qb[j]) + " >= n_qubits");
        for (int a = 0; a < k; a++)
            for (int b = a + 1; b < k; b++)
                if (g.qb[a] == g.qb[b])
                    return invalid("gate " + std::to_string(i) + ": repeated qubit " +
                                   std::to_string(g.qb[a]));
    }
    eops.clear();
    eops.reserve(n_gates * 2);
    double sw = 0;
    for (size_t i = 0; i < n_gates; i++) {
        lower_gate(gates[i], (int32_t)i, eops);
        sw += reference_sweeps(gates[i].op);
    }
    if (sweeps) *sweeps = sw;
    return SVB_OK;
}

}  // namespace svb

extern "C" {

const char* svb_last_error(void) { return g_last_error.c_str(); }

const char* svb_version(void) { return "svsim_b200 0.1 (sm_100a)"; }

svb_status svb_create(uint32_t n_qubits, int device, int precision, svb_sim** out)
{
    if (!out) return invalid("svb_create: out is NULL");
    *out = nullptr;
    if (n_qubits < 1 || n_qubits > 36) return invalid("svb_create: n_qubits must be in [1, 36]");
    if (precision != SVB_FP64 && precision != SVB_FP32)
        return invalid("svb_create: precision must be SVB_FP64 or SVB_FP32");
    int count = 0;
    SVB_CUDA(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (device < 0 || device >= count) return invalid("svb_create: no such CUDA device");
    SVB_CUDA(cudaSetDevice(device), "cudaSetDevice");
    svb_sim* s = new svb_sim();
    s->n = n_qubits;
    s->device = device;
    s->precision = precision;
    s->amp_bytes = precision == SVB_FP64 ? 16 : 8;
    const size_t bytes = s->amp_bytes << n_qubits;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if (bytes > free_b) {
        delete s;
        set_error("svb_create: state of " + std::to_string(bytes) + " bytes exceeds free device memory");
        return SVB_ERR_OOM;
    }
    cudaError_t e = cudaMalloc(&s->state, bytes);
    if (e != cudaSuccess) { delete s; return cuda_fail(e, "cudaMalloc(state)"); }
    e = cudaMalloc(&s->d_small, 64 * sizeof(double));
    if (e != cudaSuccess) { cudaFree(s->state); delete s; return cuda_fail(e, "cudaMalloc"); }
    e = dispatch_prec(precision, [&](auto t) {
        using T = decltype(t);
        return launch_reset<T>(s->state, (int)n_qubits, nullptr);
    });
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(s->state); cudaFree(s->d_small); delete s;
        return cuda_fail(e, "reset");
    }
    *out = s;
    return SVB_OK;
}

svb_status svb_destroy(svb_sim* s)
{
    if (!s) return SVB_OK;
    cudaSetDevice(s->device);
    free_plan(s);
    free_scratch(s);
    cudaFree(s->state);
    cudaFree(s->d_small);
    if (s->capture_stream) cudaStreamDestroy(s->capture_stream);
    delete s;
    return SVB_OK;
}

svb_status svb_reset_state(svb_sim* s)
{
    if (!s) return invalid("svb_reset_state: NULL handle");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    cudaError_t e = dispatch_prec(s->precision, [&](auto t) {
        using T = decltype(t);
        return launch_reset<T>(s->state, (int)s->n, nullptr);
    });
    if (e != cudaSuccess) return cuda_fail(e, "reset");
    return SVB_OK;
}

svb_status svb_set_engine(svb_sim* s, int engine, int tile_bits, int fusion_width)
{
    if (!s) return invalid("svb_set_engine: NULL handle");
    if (engine < SVB_ENGINE_AUTO || engine > SVB_ENGINE_PAIRS)
        return invalid("svb_set_engine: unknown engine");
    if (engine == SVB_ENGINE_FUSED && s->precision != SVB_FP32)
        return invalid("svb_set_engine: the fused engine runs FP32 states");
    if (engine == SVB_ENGINE_PAIRS && s->precision != SVB_FP64)
        return invalid("svb_set_engine: the pair engine runs FP64 states");
    if (tile_bits != 0 && !staged_supported(s->precision, tile_bits))
        return invalid("svb_set_engine: tile_bits must be 10..12 (FP64) or 11..13 (FP32)");
    if (fusion_width != 0 && (fusion_width < FT_MIN_K || fusion_width > FT_MAX_K))
        return invalid("svb_set_engine: fusion_width must be 3..6");
    s->engine_req = engine;
    s->tile_bits_req = tile_bits;
    s->fusion_req = fusion_width;
    return SVB_OK;
}

svb_status svb_set_circuit(svb_sim* s, const svb_gate* gates, size_t n_gates)
{
    if (!s) return invalid("svb_set_circuit: NULL handle");
    std::vector<EOp> eops;
    double sweeps = 0;
    const svb_status st = validate_and_lower(s, gates, n_gates, eops, &sweeps);
    if (st != SVB_OK) return st;
    s->mats.clear();
    return set_circuit_lowered(s, eops, gates, n_gates, sweeps);
}

}  // extern "C"

namespace svb {

// ---- the autotuner's choices, per circuit structure --------------------------------
// Key: device, qubit count, precision and an FNV-1a hash of the elementary ops' forms and
// qubits (angles left out, so a variational loop reuses one choice).
struct TuneChoice {
    int engine = SVB_ENGINE_AUTO, tile_bits = 0, fusion_width = 0;
};
std::mutex g_tune_mutex;
std::map<std::array<uint64_t, 4>, TuneChoice> g_tuned;

std::array<uint64_t, 4> structure_key(const Sim* s, const std::vector<EOp>& eops)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
    for (const EOp& e : eops) {
        mix(e.form);
        mix(e.q);
        mix(e.c);
    }
    return {(uint64_t)s->device, (uint64_t)s->n | ((uint64_t)s->precision << 32), (uint64_t)eops.size(), h};
}

svb_status set_circuit_lowered(Sim* s, std::vector<EOp>& eops, const svb_gate* gates, size_t n_gates, double sweeps)
{
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    bool has_m4 = false;
    for (const EOp& e : eops) has_m4 |= e.form == F_M4;
    std::vector<Mat4> mats;
    mats.swap(s->mats);                    // free_plan leaves them alone; keep them with the plan
    free_plan(s);
    s->mats.swap(mats);
    if (gates) s->gates.assign(gates, gates + n_gates);
    s->eops.swap(eops);

    int engine = s->engine_req;
    const int n = (int)s->n;
    int M = pick_tile_bits(s);
    int fusion = s->fusion_req;
    if (engine == SVB_ENGINE_AUTO && !has_m4 && !s->dm_qubits) {
        // a choice of svb_autotune for this circuit structure, if there is one
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tuned.find(structure_key(s, s->eops));
        if (it != g_tuned.end()) {
            engine = it->second.engine;
            if (it->second.tile_bits) M = it->second.tile_bits;
            if (it->second.fusion_width) fusion = it->second.fusion_width;
        }
    }
    if (has_m4) {
        // general 4x4 blocks: the pair engine, or per-gate sweeps below its tile
        if (engine == SVB_ENGINE_AUTO)
            engine = (s->precision == SVB_FP64 && n >= PR_TILE_BITS) ? SVB_ENGINE_PAIRS : SVB_ENGINE_PER_GATE;
        if (engine != SVB_ENGINE_PAIRS && engine != SVB_ENGINE_PER_GATE) {
            set_error("svb_set_circuit: two-qubit matrix blocks run on the pair or the per-gate engine");
            return SVB_ERR_UNSUPPORTED;
        }
    }
    if (engine == SVB_ENGINE_AUTO) {
        // Circuits of >= 12 qubits without SRN (which has no matrix) go to the tensor cores:
        // FP64 to the pair engine, FP32 to the fused engine (2x the staged engine at n = 24
        // and 30); otherwise the staged engine, per-gate below its tile
        if (n >= PR_TILE_BITS && fusable(s->eops))
            engine = s->precision == SVB_FP64 ? SVB_ENGINE_PAIRS : SVB_ENGINE_FUSED;
        else engine = (staged_supported(s->precision, M) && n >= M) ? SVB_ENGINE_STAGED : SVB_ENGINE_PER_GATE;
    }
    if (engine == SVB_ENGINE_FUSED) {
        if (s->precision != SVB_FP32 || n < FT_TILE_BITS) {
            set_error("svb_set_circuit: the fused engine needs an FP32 state of >= 12 qubits");
            return SVB_ERR_UNSUPPORTED;
        }
        if (!fusable(s->eops)) {
            set_error("svb_set_circuit: SRN is not complex-linear and cannot be fused");
            return SVB_ERR_UNSUPPORTED;
        }
    }
    if (engine == SVB_ENGINE_PAIRS) {
        if (s->precision != SVB_FP64 || n < PR_TILE_BITS) {
            set_error("svb_set_circuit: the pair engine needs an FP64 state of >= 12 qubits");
            return SVB_ERR_UNSUPPORTED;
        }
        if (!fusable(s->eops)) {
            set_error("svb_set_circuit: SRN is not complex-linear and has no matrix for the pair engine");
            return SVB_ERR_UNSUPPORTED;
        }
    }
    if (engine == SVB_ENGINE_STAGED && !(staged_supported(s->precision, M) && n >= M)) {
        set_error("svb_set_circuit: the staged engine needs n_qubits >= tile bits (10 FP64, 11 FP32)");
        return SVB_ERR_UNSUPPORTED;
    }
    s->engine = engine;

    const double sb = (double)s->amp_bytes * (double)(1ull << n);
    s->info.n_gates = n_gates;
    s->info.n_elementary = s->eops.size();
    s->info.n_sweeps_model = (uint64_t)(sweeps * 2 + 0.5) / 2;
    s->info.state_bytes = sb;
    s->info.model_bytes = 2.0 * sb * sweeps;
    s->info.engine = engine;
    if (engine == SVB_ENGINE_FUSED) {
        const int k = fusion ? fusion : FT_DEFAULT_K;
        if (k == F6_K) plan_fused6(s->eops, n, s->fused);
        else plan_fused(s->eops, n, k, s->fused);
        const FusedPlan& F = s->fused;
        SVB_CUDA(cudaMalloc(&s->dfused.passes, std::max<size_t>(1, F.passes.size()) * sizeof(FusedPass)),
                 "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dfused.blocks, std::max<size_t>(1, F.blocks.size()) * sizeof(FusedBlock)),
                 "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dfused.gates, std::max<size_t>(4, F.gates.size()) * sizeof(float)),
                 "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dfused.err, sizeof(int)), "cudaMalloc(flag)");
        SVB_CUDA(cudaMemset(s->dfused.err, 0, sizeof(int)), "cudaMemset");
        SVB_CUDA(cudaMalloc(&s->dfused.norm_partial, REDUCE_BLOCKS * sizeof(double)), "cudaMalloc(norm)");
        if (!F.passes.empty())
            SVB_CUDA(cudaMemcpy(s->dfused.passes, F.passes.data(), F.passes.size() * sizeof(FusedPass),
                                cudaMemcpyHostToDevice), "plan upload");
        if (!F.blocks.empty())
            SVB_CUDA(cudaMemcpy(s->dfused.blocks, F.blocks.data(), F.blocks.size() * sizeof(FusedBlock),
                                cudaMemcpyHostToDevice), "plan upload");
        if (!F.gates.empty())
            SVB_CUDA(cudaMemcpy(s->dfused.gates, F.gates.data(), F.gates.size() * sizeof(float),
                                cudaMemcpyHostToDevice), "plan upload");
        if (!F.passes6.empty()) {
            SVB_CUDA(cudaMalloc(&s->dfused.passes6, F.passes6.size() * sizeof(Fused6Pass)), "cudaMalloc(plan)");
            SVB_CUDA(cudaMemcpy(s->dfused.passes6, F.passes6.data(), F.passes6.size() * sizeof(Fused6Pass),
                                cudaMemcpyHostToDevice), "plan upload");
        }
        const size_t np = F.n_passes();
        s->info.n_passes = np;
        s->info.tile_bits = k == F6_K ? F6_TILE_BITS : FT_TILE_BITS;
        s->info.n_blocks = k == F6_K ? F.passes6.size() : F.blocks.size();
        s->info.plan_bytes = F.passes.size() * sizeof(FusedPass) + F.blocks.size() * sizeof(FusedBlock) +
                             F.passes6.size() * sizeof(Fused6Pass) + F.gates.size() * sizeof(float);
        // one read + write per pass, then the renormalisation (two reads, one write)
        s->info.moved_bytes = 2.0 * sb * (double)np + (np == 0 ? 0.0 : 3.0 * sb);
    } else if (engine == SVB_ENGINE_PAIRS) {
        if (!plan_pairs(s->eops, n, s->pairs, &s->mats)) {
            set_error("svb_set_circuit: the pair planner rejected the circuit");
            return SVB_ERR_UNSUPPORTED;
        }
        const PairPlan& R = s->pairs;
        SVB_CUDA(cudaMalloc(&s->dpairs.passes, std::max<size_t>(1, R.passes.size()) * sizeof(PairPass)),
                 "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dpairs.ops, std::max<size_t>(1, R.ops.size()) * sizeof(PairOp)), "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dpairs.layouts, std::max<size_t>(1, R.layouts.size()) * sizeof(DevStage)),
                 "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dpairs.gates, std::max<size_t>(2, R.gates.size()) * sizeof(double)),
                 "cudaMalloc(plan)");
        if (!R.passes.empty())
            SVB_CUDA(cudaMemcpy(s->dpairs.passes, R.passes.data(), R.passes.size() * sizeof(PairPass),
                                cudaMemcpyHostToDevice), "plan upload");
        if (!R.ops.empty())
            SVB_CUDA(cudaMemcpy(s->dpairs.ops, R.ops.data(), R.ops.size() * sizeof(PairOp), cudaMemcpyHostToDevice),
                     "plan upload");
        if (!R.layouts.empty())
            SVB_CUDA(cudaMemcpy(s->dpairs.layouts, R.layouts.data(), R.layouts.size() * sizeof(DevStage),
                                cudaMemcpyHostToDevice), "plan upload");
        if (!R.gates.empty())
            SVB_CUDA(cudaMemcpy(s->dpairs.gates, R.gates.data(), R.gates.size() * sizeof(double),
                                cudaMemcpyHostToDevice), "plan upload");
        s->dpairs.stage_bytes = R.stage_bytes;
        s->info.n_passes = R.passes.size();
        s->info.tile_bits = PR_TILE_BITS;
        s->info.n_blocks = R.n_blocks;
        s->info.plan_bytes = R.passes.size() * sizeof(PairPass) + R.ops.size() * sizeof(PairOp) +
                             R.layouts.size() * sizeof(DevStage) + R.gates.size() * sizeof(double);
        s->info.moved_bytes = 2.0 * sb * (double)R.passes.size();
    } else if (engine == SVB_ENGINE_STAGED) {
        const int G = s->precision == SVB_FP64 ? 3 : 4;
        plan_staged(s->eops, n, M, G, s->staged);
        const StagedPlan& P = s->staged;
        SVB_CUDA(cudaMalloc(&s->dplan.passes, std::max<size_t>(1, P.passes.size()) * sizeof(DevPass)),
                 "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dplan.stages, std::max<size_t>(1, P.stages.size()) * sizeof(DevStage)),
                 "cudaMalloc(plan)");
        SVB_CUDA(cudaMalloc(&s->dplan.ops, std::max<size_t>(1, P.ops.size()) * sizeof(DevOp)),
                 "cudaMalloc(plan)");
        if (!P.passes.empty())
            SVB_CUDA(cudaMemcpy(s->dplan.passes, P.passes.data(), P.passes.size() * sizeof(DevPass),
                                cudaMemcpyHostToDevice), "plan upload");
        if (!P.stages.empty())
            SVB_CUDA(cudaMemcpy(s->dplan.stages, P.stages.data(), P.stages.size() * sizeof(DevStage),
                                cudaMemcpyHostToDevice), "plan upload");
        if (!P.ops.empty())
            SVB_CUDA(cudaMemcpy(s->dplan.ops, P.ops.data(), P.ops.size() * sizeof(DevOp),
                                cudaMemcpyHostToDevice), "plan upload");
        s->info.n_passes = P.passes.size();
        s->info.tile_bits = M;
        s->info.plan_bytes = P.passes.size() * sizeof(DevPass) + P.stages.size() * sizeof(DevStage) +
                             P.ops.size() * sizeof(DevOp);
        s->info.moved_bytes = 2.0 * sb * (double)P.passes.size();
    } else {
        s->info.n_passes = s->eops.size();
        s->info.tile_bits = 0;
        double moved = 0;
        // dense forms read and write every amplitude (2 sb); diagonal forms other than
        // DIAG and CX read and write one half of the state (its |1> half, resp. its
        // control = 1 half: sb).  F_M4 blocks count as dense.
        for (const EOp& e : s->eops)
            moved += (e.form == F_CX || (form_is_diag(e.form) && e.form != F_DIAG)) ? sb : 2.0 * sb;
        s->info.moved_bytes = moved;
    }
    s->have_circuit = true;
    return SVB_OK;
}

}  // namespace svb

extern "C" {

svb_status svb_clear_circuit(svb_sim* s)
{
    if (!s) return invalid("svb_clear_circuit: NULL handle");
    cudaSetDevice(s->device);
    free_plan(s);
    return SVB_OK;
}

svb_status svb_get_plan_info(const svb_sim* s, svb_plan_info* out)
{
    if (!s || !out) return invalid("svb_get_plan_info: NULL argument");
    *out = s->info;
    return SVB_OK;
}

svb_status svb_run(svb_sim* s, void* stream)
{
    if (!s) return invalid("svb_run: NULL handle");
    if (!s->have_circuit) {
        set_error("svb_run: no circuit set");
        return SVB_ERR_STATE;
    }
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (s->info.n_passes == 0) return SVB_OK;
    if (use_graph(s)) {
        if (!s->graph) {
            if (!s->capture_stream)
                SVB_CUDA(cudaStreamCreateWithFlags(&s->capture_stream, cudaStreamNonBlocking),
                         "cudaStreamCreate");
            SVB_CUDA(cudaStreamBeginCapture(s->capture_stream, cudaStreamCaptureModeThreadLocal),
                     "cudaStreamBeginCapture");
            svb_status rc = launch_all(s, s->capture_stream);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(s->capture_stream, &g);
            if (rc != SVB_OK) { if (g) cudaGraphDestroy(g); return rc; }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&s->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) { s->graph = nullptr; return cuda_fail(e, "cudaGraphInstantiate"); }
        }
        SVB_CUDA(cudaGraphLaunch(s->graph, st), "cudaGraphLaunch");
        return SVB_OK;
    }
    return launch_all(s, st);
}

svb_status svb_synchronize(svb_sim* s)
{
    if (!s) return invalid("svb_synchronize: NULL handle");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    SVB_CUDA(cudaDeviceSynchronize(), "kernel execution");
    if (s->engine == SVB_ENGINE_FUSED && s->dfused.err) {
        int flag = 0;
        SVB_CUDA(cudaMemcpy(&flag, s->dfused.err, sizeof(int), cudaMemcpyDeviceToHost), "flag read");
        if (flag) {
            cudaMemset(s->dfused.err, 0, sizeof(int));
            set_error("fused kernel: a tensor-core completion wait timed out");
            return SVB_ERR_CUDA;
        }
    }
    return SVB_OK;
}

svb_status svb_get_state_soa(svb_sim* s, double* re, double* im)
{
    if (!s) return invalid("svb_get_state_soa: NULL handle");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    const uint64_t dim = 1ull << s->n;
    const uint64_t chunk = std::min<uint64_t>(dim, 1ull << 24);
    double *dre = nullptr, *dim_ = nullptr;
    SVB_CUDA(cudaMalloc(&dre, chunk * sizeof(double)), "cudaMalloc(staging)");
    cudaError_t e = cudaMalloc(&dim_, chunk * sizeof(double));
    if (e != cudaSuccess) { cudaFree(dre); return cuda_fail(e, "cudaMalloc(staging)"); }
    for (uint64_t f = 0; f < dim && e == cudaSuccess; f += chunk) {
        const uint64_t c = std::min(chunk, dim - f);
        e = dispatch_prec(s->precision, [&](auto t) {
            using T = decltype(t);
            return launch_soa_split<T>(s->state, f, c, re ? dre : nullptr, im ? dim_ : nullptr, nullptr);
        });
        if (e == cudaSuccess && re) e = cudaMemcpy(re + f, dre, c * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && im) e = cudaMemcpy(im + f, dim_, c * sizeof(double), cudaMemcpyDeviceToHost);
    }
    cudaFree(dre);
    cudaFree(dim_);
    if (e != cudaSuccess) return cuda_fail(e, "svb_get_state_soa");
    return SVB_OK;
}

svb_status svb_set_state_soa(svb_sim* s, const double* re, const double* im)
{
    if (!s || !re || !im) return invalid("svb_set_state_soa: NULL argument");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    const uint64_t dim = 1ull << s->n;
    const uint64_t chunk = std::min<uint64_t>(dim, 1ull << 24);
    double *dre = nullptr, *dim_ = nullptr;
    SVB_CUDA(cudaMalloc(&dre, chunk * sizeof(double)), "cudaMalloc(staging)");
    cudaError_t e = cudaMalloc(&dim_, chunk * sizeof(double));
    if (e != cudaSuccess) { cudaFree(dre); return cuda_fail(e, "cudaMalloc(staging)"); }
    for (uint64_t f = 0; f < dim && e == cudaSuccess; f += chunk) {
        const uint64_t c = std::min(chunk, dim - f);
        e = cudaMemcpy(dre, re + f, c * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dim_, im + f, c * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = dispatch_prec(s->precision, [&](auto t) {
                using T = decltype(t);
                return launch_soa_merge<T>(s->state, f, c, dre, dim_, nullptr);
            });
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    cudaFree(dre);
    cudaFree(dim_);
    if (e != cudaSuccess) return cuda_fail(e, "svb_set_state_soa");
    return SVB_OK;
}

svb_status svb_state_device_ptr(svb_sim* s, void** dptr, int* precision)
{
    if (!s || !dptr) return invalid("svb_state_device_ptr: NULL argument");
    *dptr = s->state;
    if (precision) *precision = s->precision;
    return SVB_OK;
}

svb_status svb_measure(svb_sim* s, const double* uniforms, uint32_t shots, uint64_t* out,
                       double* prob_total)
{
    if (!s) return invalid("svb_measure: NULL handle");
    if (shots > 0 && (!uniforms || !out)) return invalid("svb_measure: NULL uniforms or output");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    svb_status rc = ensure_scratch(s, std::max<uint32_t>(shots, 1));
    if (rc != SVB_OK) return rc;
    if (shots > 0)
        SVB_CUDA(cudaMemcpy(s->mscr.uniforms, uniforms, shots * sizeof(double), cudaMemcpyHostToDevice),
                 "uniforms upload");
    cudaError_t e = dispatch_prec(s->precision, [&](auto t) {
        using T = decltype(t);
        return measure_device<T>(s->state, (int)s->n, s->mscr.uniforms, shots, s->mscr.samples,
                                 s->d_small, s->mscr, nullptr);
    });
    if (e != cudaSuccess) return cuda_fail(e, "measure");
    if (shots > 0)
        SVB_CUDA(cudaMemcpy(out, s->mscr.samples, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost),
                 "samples download");
    double total = 0;
    SVB_CUDA(cudaMemcpy(&total, s->d_small, sizeof(double), cudaMemcpyDeviceToHost), "total download");
    if (prob_total) *prob_total = total;
    return SVB_OK;
}

svb_status svb_measure_seeded(svb_sim* s, uint32_t seed, uint32_t shots, uint64_t* out, double* prob_total)
{
    if (!s) return invalid("svb_measure_seeded: NULL handle");
    if (shots > 0 && !out) return invalid("svb_measure_seeded: NULL output");
    // the reference's draws (svsim_nvgpu_sin.cuh:367-371) with the caller's seed
    std::vector<double> u(shots);
    srand(seed);
    for (uint32_t i = 0; i < shots; i++) u[i] = (double)rand() / (double)RAND_MAX;
    return svb_measure(s, u.data(), shots, out, prob_total);
}

svb_status svb_norm2(svb_sim* s, double* out)
{
    if (!s || !out) return invalid("svb_norm2: NULL argument");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    svb_status rc = ensure_scratch(s, 1);
    if (rc != SVB_OK) return rc;
    cudaError_t e = dispatch_prec(s->precision, [&](auto t) {
        using T = decltype(t);
        return norm2_device<T>(s->state, (int)s->n, s->d_small, s->mscr, nullptr);
    });
    if (e != cudaSuccess) return cuda_fail(e, "norm2");
    SVB_CUDA(cudaMemcpy(out, s->d_small, sizeof(double), cudaMemcpyDeviceToHost), "norm download");
    return SVB_OK;
}

svb_status svb_compare_states(svb_sim* a, svb_sim* b, double* fidelity, double* max_abs_diff)
{
    if (!a || !b) return invalid("svb_compare_states: NULL handle");
    if (a->n != b->n || a->device != b->device)
        return invalid("svb_compare_states: states differ in size or device");
    SVB_CUDA(cudaSetDevice(a->device), "cudaSetDevice");
    double* buf = nullptr;
    SVB_CUDA(cudaMalloc(&buf, (5 + 5 * REDUCE_BLOCKS) * sizeof(double)), "cudaMalloc(compare)");
    cudaError_t e;
    const int n = (int)a->n;
    if (a->precision == SVB_FP64 && b->precision == SVB_FP64)
        e = compare_device<double, double>(a->state, b->state, n, buf, buf + 5, nullptr);
    else if (a->precision == SVB_FP64)
        e = compare_device<double, float>(a->state, b->state, n, buf, buf + 5, nullptr);
    else if (b->precision == SVB_FP64)
        e = compare_device<float, double>(a->state, b->state, n, buf, buf + 5, nullptr);
    else
        e = compare_device<float, float>(a->state, b->state, n, buf, buf + 5, nullptr);
    double v[5] = {0, 0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(v, buf, sizeof(v), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(e, "svb_compare_states");
    if (fidelity) *fidelity = (v[2] > 0 && v[3] > 0) ? (v[0] * v[0] + v[1] * v[1]) / (v[2] * v[3]) : 0.0;
    if (max_abs_diff) *max_abs_diff = v[4];
    return SVB_OK;
}

svb_status svb_expectation(svb_sim* s, const svb_pauli_term* terms, size_t n_terms, double* out)
{
    if (!s || !out || (n_terms > 0 && !terms)) return invalid("svb_expectation: NULL argument");
    if (n_terms > 4096) return invalid("svb_expectation: at most 4096 terms");
    for (size_t t = 0; t < n_terms; t++)
        if ((terms[t].x_mask | terms[t].z_mask) >> s->n)
            return invalid("svb_expectation: term acts on a qubit >= n_qubits");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    if (n_terms == 0) { *out = 0; return SVB_OK; }
    svb_status rc = ensure_scratch(s, 1);
    if (rc != SVB_OK) return rc;
    svb_pauli_term* dterms = nullptr;
    SVB_CUDA(cudaMalloc(&dterms, n_terms * sizeof(svb_pauli_term)), "cudaMalloc(terms)");
    cudaError_t e = cudaMemcpy(dterms, terms, n_terms * sizeof(svb_pauli_term), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = dispatch_prec(s->precision, [&](auto t) {
            using T = decltype(t);
            return expectation_device<T>(s->state, (int)s->n, dterms, (int)n_terms, s->d_small,
                                         s->mscr.partial, nullptr);
        });
    if (e == cudaSuccess) e = cudaMemcpy(out, s->d_small, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dterms);
    if (e != cudaSuccess) return cuda_fail(e, "svb_expectation");
    return SVB_OK;
}

}  // extern "C"

extern "C" svb_status svb_autotune(svb_sim* s, const svb_gate* gates, size_t n_gates, svb_tune_result* out)
{
    using namespace svb;
    if (!s || (n_gates && !gates)) return invalid("svb_autotune: NULL argument");
    if (s->dm_qubits) return invalid("svb_autotune: not for density-matrix handles");
    SVB_CUDA(cudaSetDevice(s->device), "cudaSetDevice");
    std::vector<EOp> eops;
    double sweeps = 0;
    svb_status st = validate_and_lower(s, gates, n_gates, eops, &sweeps);
    if (st != SVB_OK) return st;
    const int n = (int)s->n;
    const bool fp64 = s->precision == SVB_FP64;
    const bool matrices = fusable(eops);
    const auto key = structure_key(s, eops);
    // candidates: (engine, tile bits, fusion width)
    std::vector<TuneChoice> cands;
    if (n <= 26) cands.push_back({SVB_ENGINE_PER_GATE, 0, 0});
    for (int M = fp64 ? 10 : 11; M <= (fp64 ? 12 : 13); M++)
        if (n >= M) cands.push_back({SVB_ENGINE_STAGED, M, 0});
    if (n >= PR_TILE_BITS && matrices) {
        if (fp64) cands.push_back({SVB_ENGINE_PAIRS, 0, 0});
        else
            for (int k = FT_MIN_K; k <= FT_MAX_K; k++) cands.push_back({SVB_ENGINE_FUSED, 0, k});
    }
    // the prefix timed: the whole circuit up to 360 gates (the choice holds for the structure)
    const size_t P = std::min<size_t>(n_gates, 360);
    const int req_e = s->engine_req, req_t = s->tile_bits_req, req_k = s->fusion_req;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned.erase(key);                      // the default choice is timed as well
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SVB_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
    SVB_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
    TuneChoice best;
    double best_ms = 1e300, default_ms = -1;
    int tried = 0;
    // the static default first (engine AUTO with no tuned choice)
    std::vector<TuneChoice> order = {TuneChoice{}};
    order.insert(order.end(), cands.begin(), cands.end());
    for (size_t ci = 0; ci < order.size(); ci++) {
        const TuneChoice& c = order[ci];
        s->engine_req = c.engine;
        s->tile_bits_req = c.tile_bits;
        s->fusion_req = c.fusion_width;
        if (svb_set_circuit(s, gates, P) != SVB_OK) continue;
        svb_reset_state(s);
        float ms = 0.f;
        cudaError_t e = svb_run(s, nullptr) == SVB_OK ? cudaSuccess : cudaErrorUnknown;     // warm-up
        if (e == cudaSuccess) e = cudaEventRecord(e0, nullptr);
        if (e == cudaSuccess) e = svb_run(s, nullptr) == SVB_OK ? cudaSuccess : cudaErrorUnknown;
        if (e == cudaSuccess) e = cudaEventRecord(e1, nullptr);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess || svb_synchronize(s) != SVB_OK) {
            (void)cudaGetLastError();
            continue;
        }
        if (ci == 0) {
            default_ms = ms;
            continue;
        }
        tried++;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->engine_req = req_e;
    s->tile_bits_req = req_t;
    s->fusion_req = req_k;
    if (tried == 0) {
        set_error("svb_autotune: no candidate engine could run the circuit");
        return SVB_ERR_UNSUPPORTED;
    }
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[key] = best;
    }
    if (out) {
        out->engine = best.engine;
        out->tile_bits = best.tile_bits;
        out->fusion_width = best.fusion_width;
        out->candidates = tried;
        out->best_ms = best_ms;
        out->default_ms = default_ms;
        out->timed_gates = (uint64_t)P;
    }
    // the handle ends with the circuit planned for its own engine request (AUTO: the
    // tuned choice) and the state at |0..0>
    st = svb_set_circuit(s, gates, n_gates);
    if (st != SVB_OK) return st;
    return svb_reset_state(s);
}

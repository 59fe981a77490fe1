// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// C glue around the reference's own CPU backends, compiled in place from the
// reference tree by oracle/Makefile (outputs under oracle/_ref/).  One build per
// backend selected with -DREF_BACKEND_SIN or -DREF_BACKEND_OMP:
//   svsim/src/svsim_cpu_sin.hpp  (single thread,   Simulation(n, unused))
//   svsim/src/svsim_cpu_omp.hpp  (OpenMP, Simulation(n, n_cpus), :199-218, :288-320)
//
// The glue only drives the reference's public API — Simulation ctor, append,
// upload, sim, measure, sv_real/sv_imag — exactly like its unit tests do
// (svsim/unit_test/unit_test_cpu_sin.cpp:41-55).  It adds two conveniences:
//   * the reference seeds rand() with time(0) inside measure()
//     (svsim/src/config.hpp:44, svsim_cpu_sin.hpp:330); the glue maps that
//     `time(...)` call onto a settable seed so sampling becomes reproducible;
//   * the per-run printf of sim() (svsim_cpu_sin.hpp:296-301) can be silenced by
//     pointing fd 1 at /dev/null around the call.

#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include <unistd.h>
#include <fcntl.h>
#include <sys/time.h>
#include <assert.h>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include <chrono>
#ifdef REF_BACKEND_OMP
#include <omp.h>
#endif

static unsigned long g_ref_seed = 1;
static time_t ref_fixed_time(time_t*) { return (time_t)g_ref_seed; }
// Only the `time(0)` inside the reference's RAND_SEED macro is affected: every
// system header that declares time() was included above.
#define time(x) ref_fixed_time(x)

#include "util_cpu.h"
#if defined(REF_BACKEND_SIN)
#include "svsim_cpu_sin.hpp"
#elif defined(REF_BACKEND_OMP)
#include "svsim_cpu_omp.hpp"
#else
#error "define REF_BACKEND_SIN or REF_BACKEND_OMP"
#endif
#undef time

using namespace SVSim;

extern "C" {

// Same layout as svb_gate in include/svsim_b200.h (48 bytes).
typedef struct ref_gate {
    uint32_t op;
    uint32_t qb[5];
    double theta, phi, lambda;
} ref_gate;

int ref_idx_bits(void) { return (int)(8 * sizeof(IdxType)); }

static int quiet_begin(int quiet) {
    if (!quiet) return -1;
    fflush(stdout);
    int saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
    return saved;
}
static void quiet_end(int saved) {
    if (saved < 0) return;
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
}

// Runs `gates` on |0..0> with the reference backend and returns the SoA state.
// n_threads is the OpenMP thread count (ignored by the single-thread backend).
// sim_ms receives the wall time of sim() alone, which is what the reference's
// own cpu_timer brackets.  If shots > 0, measure(shots) is also called with
// rand() seeded by `seed`, and the samples are written to `samples`.
int ref_simulate(uint32_t n_qubits, int n_threads, const ref_gate* gates, uint64_t n_gates,
                 double* out_re, double* out_im, double* sim_ms,
                 uint32_t shots, unsigned long seed, uint64_t* samples, int quiet)
{
    if (n_qubits == 0 || n_qubits > 8 * sizeof(IdxType) - 4) return -1;
    Simulation sim((IdxType)n_qubits, (IdxType)(n_threads > 0 ? n_threads : 1));
    for (uint64_t i = 0; i < n_gates; i++) {
        const ref_gate& g = gates[i];
        Gate tmp((enum OP)g.op, g.qb[0], g.qb[1], g.qb[2], g.qb[3], g.qb[4],
                 g.theta, g.phi, g.lambda);
        sim.append(&tmp);
    }
    sim.upload();
    int saved = quiet_begin(quiet);
    auto t0 = std::chrono::steady_clock::now();
    sim.sim();
    auto t1 = std::chrono::steady_clock::now();
    quiet_end(saved);
    if (sim_ms) *sim_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    const uint64_t dim = 1ull << n_qubits;
    if (out_re) memcpy(out_re, sim.sv_real, dim * sizeof(double));
    if (out_im) memcpy(out_im, sim.sv_imag, dim * sizeof(double));
    if (shots > 0 && samples) {
        g_ref_seed = seed;
        saved = quiet_begin(quiet);
        IdxType* res = sim.measure(shots);
        quiet_end(saved);
        for (uint32_t i = 0; i < shots; i++) samples[i] = (uint64_t)res[i];
        delete[] res;
    }
    return 0;
}

// A persistent reference Simulation for timing loops: the state is allocated and
// set to |0..0> once (ctor, svsim_cpu_omp.hpp:199-218); every ref_handle_run then
// appends a circuit, uploads it, runs sim() on the current state and clears the
// circuit again (clear_circuit keeps the state), as the reference's own re-run
// pattern does.  Returns sim()'s wall time in ms through sim_ms.
void* ref_handle_open(uint32_t n_qubits, int n_threads)
{
    if (n_qubits == 0 || n_qubits > 8 * sizeof(IdxType) - 4) return nullptr;
    return new Simulation((IdxType)n_qubits, (IdxType)(n_threads > 0 ? n_threads : 1));
}

int ref_handle_run(void* h, const ref_gate* gates, uint64_t n_gates, double* sim_ms, int quiet)
{
    Simulation& sim = *static_cast<Simulation*>(h);
    for (uint64_t i = 0; i < n_gates; i++) {
        const ref_gate& g = gates[i];
        Gate tmp((enum OP)g.op, g.qb[0], g.qb[1], g.qb[2], g.qb[3], g.qb[4],
                 g.theta, g.phi, g.lambda);
        sim.append(&tmp);
    }
    sim.upload();
    int saved = quiet_begin(quiet);
    auto t0 = std::chrono::steady_clock::now();
    sim.sim();
    auto t1 = std::chrono::steady_clock::now();
    quiet_end(saved);
    sim.clear_circuit();
    if (sim_ms) *sim_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return 0;
}

void ref_handle_close(void* h) { delete static_cast<Simulation*>(h); }

}  // extern "C"

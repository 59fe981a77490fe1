// BASELINE INFRASTRUCTURE ONLY — never linked into the product library.
//
// Drives the reference's own single-GPU backend, svsim/src/svsim_nvgpu_sin.cuh, compiled
// in place from the reference tree by oracle/Makefile (target ref_gpu, output
// oracle/_ref/ref_gpu_driver), so that its GPU kernel can be timed on this hardware
// beside the B200 engine (context only: the timed reference arm is the CPU path).
//
// Usage: ref_gpu_driver <gates.bin> <n_qubits> <repetitions>
//   gates.bin: svb_gate records (48 bytes: op, 5 qubits, theta, phi, lambda).
// The circuit is built with the reference's public API (Simulation(n, 0), append,
// upload) and sim() is called `repetitions` times on the evolving state; sim() itself
// prints its event-timed kernel time ("sim:%.3lf ms", svsim_nvgpu_sin.cuh:306-339,
// PRINT_MEA_PER_CIRCUIT in config.hpp:25), which the caller parses.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "util_nvgpu.cuh"
#include "svsim_nvgpu_sin.cuh"

using namespace SVSim;

struct GateRecord {
    uint32_t op;
    uint32_t qb[5];
    double theta, phi, lambda;
};

int main(int argc, char** argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: %s gates.bin n_qubits repetitions\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", argv[1]);
        return 2;
    }
    std::vector<GateRecord> recs;
    GateRecord r;
    while (fread(&r, sizeof(r), 1, f) == 1) recs.push_back(r);
    fclose(f);
    const int n = atoi(argv[2]);
    const int reps = atoi(argv[3]);
    if (n < 1 || n > 28 || reps < 1) {
        fprintf(stderr, "n_qubits must be 1..28 (the shipped 32-bit IdxType), repetitions >= 1\n");
        return 2;
    }
    Simulation sim((IdxType)n, 0);
    for (const GateRecord& g : recs) {
        Gate tmp((enum OP)g.op, g.qb[0], g.qb[1], g.qb[2], g.qb[3], g.qb[4], g.theta, g.phi, g.lambda);
        sim.append(&tmp);
    }
    sim.upload();
    for (int i = 0; i < reps; i++) sim.sim();
    return 0;
}

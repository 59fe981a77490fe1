/* TEST INFRASTRUCTURE ONLY — the CPU oracle.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline arm load this; the product library never does.
 *
 * A plain-C restatement of the reference's single-GPU state-vector path
 * (svsim/src/svsim_nvgpu_sin.cuh and its CPU twin svsim/src/svsim_cpu_sin.hpp):
 * the 38 gate operations on an SoA complex<double> state, and the host-side
 * measurement of Simulation::measure with the uniforms injected instead of drawn
 * from rand().  Indices are 64-bit, so n up to 34 is representable (memory
 * permitting); the reference itself stops at n = 28 with its 32-bit IdxType.
 */
#ifndef SVSIM_ORACLE_H
#define SVSIM_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gate record; byte-identical to svb_gate of include/svsim_b200.h. */
typedef struct oracle_gate {
    uint32_t op;      /* reference enum OP (svsim_nvgpu_sin.cuh:42-48) */
    uint32_t qb[5];
    double theta, phi, lambda;
} oracle_gate;

typedef struct oracle_pauli {
    double coef;
    uint64_t x_mask;  /* qubits carrying X or Y */
    uint64_t z_mask;  /* qubits carrying Z or Y */
} oracle_pauli;

/* |0..0> */
void oracle_reset(uint32_t n, double* re, double* im);
/* Apply one reference gate in place; returns 0, or -1 for an unknown op. */
int oracle_apply_gate(uint32_t n, const oracle_gate* g, double* re, double* im);
/* Reset, then apply gates[0..n_gates) in order. */
int oracle_run(uint32_t n, const oracle_gate* gates, size_t n_gates, double* re, double* im);
/* Apply without resetting first. */
int oracle_apply(uint32_t n, const oracle_gate* gates, size_t n_gates, double* re, double* im);
/* Simulation::measure with injected uniforms (svsim_cpu_sin.hpp:324-346).
 * total (may be NULL) receives the last scan value, sum of |a|^2. */
void oracle_measure_uniforms(uint32_t n, const double* re, const double* im,
                             const double* uniforms, uint32_t shots, uint64_t* out, double* total);
/* <psi| sum_t coef_t P_t |psi>, real part; terms use the X/Z-mask encoding. */
double oracle_expectation(uint32_t n, const double* re, const double* im,
                          const oracle_pauli* terms, size_t n_terms);
/* number of elementary sweeps the reference GPU path spends on one op. */
int oracle_elementary_count(uint32_t op);

#ifdef __cplusplus
}
#endif
#endif

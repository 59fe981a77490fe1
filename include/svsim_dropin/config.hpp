// Drop-in configuration header for code written against SV-Sim's single-GPU backend.
//
// Same macro and type names as the reference's svsim/src/config.hpp (:25-58), because
// user programs and svsim/src/py_wrapper.cpp use them by name.  Two differences:
//   * IdxType is 64-bit: the engine indexes states up to 2^36 amplitudes (the
//     reference's 32-bit IdxType stops at n = 28);
//   * no device-side settings remain (the kernels live in libsvsim_b200.so).
#ifndef CONFIG_HPP
#define CONFIG_HPP

// per-run timing printout of Simulation::sim()
#define PRINT_MEA_PER_CIRCUIT

namespace SVSim
{
using IdxType = unsigned long long;   // basis-state index
using ValType = double;               // amplitude component
}  // namespace SVSim

// seed of rand() in Simulation::measure()
#define RAND_SEED time(0)
// tolerance of the probability-sum check in Simulation::measure()
#define ERROR_BAR (1e-3)
#define PI 3.14159265358979323846
#define S2I 0.70710678118654752440
// kept for source compatibility; the engine chooses its own launch shapes
#define THREADS_PER_BLOCK 256
#define TILE 16

#endif

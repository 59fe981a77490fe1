// Drop-in utility header for code written against SV-Sim's single-GPU backend: the
// host helpers of the reference's svsim/src/util_nvgpu.cuh (:66-155) that user
// programs call — CHECK_NULL_POINTER, cpu_timer, print_binary, print_measurement —
// with the same names.  The engine's CUDA error handling lives behind the C ABI
// (status codes, svb_last_error), so the cudaSafeCall/SAFE_ALOC_* macros are gone.
#ifndef UTIL_NVPUG_CUH
#define UTIL_NVPUG_CUH

#include <stdio.h>
#include <stdlib.h>
#include <assert.h>
#include <sys/time.h>

#include "config.hpp"

namespace SVSim
{

#define CHECK_NULL_POINTER(X) ::SVSim::check_null_pointer_(__FILE__, __LINE__, (const void*)(X))
inline void check_null_pointer_(const char* file, int line, const void* p)
{
    if (p == NULL) {
        fprintf(stderr, "Error: NULL pointer at %s:%i.\n", file, line);
        exit(-1);
    }
}

inline double get_cpu_timer()
{
    struct timeval tp;
    gettimeofday(&tp, NULL);
    return (double)tp.tv_sec * 1e3 + (double)tp.tv_usec * 1e-3;   // milliseconds
}

typedef struct CPU_Timer {
    CPU_Timer() : start(0.0), stop(0.0) {}
    void start_timer() { start = get_cpu_timer(); }
    void stop_timer() { stop = get_cpu_timer(); }
    double measure() { return stop - start; }
    double start;
    double stop;
} cpu_timer;

inline void print_binary(IdxType v, int width)
{
    for (int i = width - 1; i >= 0; i--) putchar('0' + (int)((v >> i) & 1));
}

inline void print_measurement(IdxType* res_state, IdxType n_qubits, int repetition)
{
    assert(res_state != NULL);
    printf("\n===============  Measurement (tests=%d) ================\n", repetition);
    for (int i = 0; i < repetition; i++) {
        printf("Test-%d: ", i);
        print_binary(res_state[i], (int)n_qubits);
        printf("\n");
    }
}

}  // namespace SVSim

#endif

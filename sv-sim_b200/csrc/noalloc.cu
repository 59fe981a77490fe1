// Measurement entry point that allocates nothing (svb_measure_noalloc).
//
// svb_measure needs scratch space on the device for its FP64 block sums and their
// prefix, and obtains it with cudaMalloc through the handle.  Some callers cannot do
// that: an application that reserves all device memory for its own pool at start-up
// (a later cudaMalloc fails or eats into the pool), or one that owns the state buffer
// itself and wants no hidden allocations, frees or the device-wide synchronisation a
// cudaFree can bring.  svb_measure_noalloc serves them: the caller passes device
// buffers for the state, the uniforms and the results, and the scratch comes from a
// fixed array in this library's device image.
//
// The array is sized for states of up to SVB_NOALLOC_MAX_QUBITS qubits (one FP64 sum per
// 4096 amplitudes, plus the prefix of those sums: about 4 MiB).  Every device that loads
// the library holds it until the process exits.  All calls on a device share it, so
// calls whose work overlaps on the GPU (on different streams, or from different host
// threads) race on it and must be serialised by the caller.  The kernels overwrite every
// entry they later read, so nothing needs clearing between calls.
#include "svb_internal.h"

namespace svb {
namespace {

constexpr int kNoallocMaxQubits = SVB_NOALLOC_MAX_QUBITS;
constexpr size_t kNoallocBlocks = size_t(1) << (kNoallocMaxQubits - MEAS_BLOCK_BITS);

// block sums [0, kNoallocBlocks), then their exclusive prefix [kNoallocBlocks, 2 kNoallocBlocks + 1)
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoallocBlocks + 2];

// Device address of g_noalloc_scratch per device, looked up once (host code cannot use
// the symbol's name as a device address).
double* scratch_address(int dev, svb_status* st)
{
    static double* addr[64] = {nullptr};
    *st = SVB_OK;
    if (dev < 0 || dev >= 64) {
        set_error("svb_measure_noalloc: device index out of range");
        *st = SVB_ERR_INVALID;
        return nullptr;
    }
    if (!addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("svb_measure_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            (void)cudaGetLastError();
            *st = SVB_ERR_CUDA;
            return nullptr;
        }
        addr[dev] = static_cast<double*>(p);
    }
    return addr[dev];
}

}  // namespace
}  // namespace svb

using namespace svb;

extern "C" svb_status svb_measure_noalloc(const void* state, uint32_t n_qubits, int precision,
                                          const double* uniforms, uint32_t shots, uint64_t* samples,
                                          double* prob_total, void* stream)
{
    if (!state) { set_error("svb_measure_noalloc: state is NULL"); return SVB_ERR_INVALID; }
    if (n_qubits < 1 || n_qubits > (uint32_t)kNoallocMaxQubits) {
        set_error("svb_measure_noalloc: n_qubits must be in [1, " + std::to_string(kNoallocMaxQubits) +
                  "]: the static scratch holds block sums for at most that many qubits");
        return SVB_ERR_INVALID;
    }
    if (precision != SVB_FP64 && precision != SVB_FP32) {
        set_error("svb_measure_noalloc: precision must be SVB_FP64 or SVB_FP32");
        return SVB_ERR_INVALID;
    }
    if (shots > 0 && (!uniforms || !samples)) {
        set_error("svb_measure_noalloc: uniforms and samples are required when shots > 0");
        return SVB_ERR_INVALID;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("svb_measure_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return SVB_ERR_CUDA;
    }
    svb_status st;
    double* scratch = scratch_address(dev, &st);
    if (!scratch) return st;
    MeasureScratch scr;
    scr.block_sums = scratch;
    scr.block_prefix = scratch + kNoallocBlocks;
    scr.cap_blocks = kNoallocBlocks;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    e = precision == SVB_FP64
            ? measure_device<double>(state, (int)n_qubits, uniforms, shots, samples, prob_total, scr, s)
            : measure_device<float>(state, (int)n_qubits, uniforms, shots, samples, prob_total, scr, s);
    if (e != cudaSuccess) {
        set_error(std::string("svb_measure_noalloc: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return SVB_ERR_CUDA;
    }
    return SVB_OK;
}

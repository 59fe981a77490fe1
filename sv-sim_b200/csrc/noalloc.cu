// Measurement entry point that allocates nothing (svb_measure_noalloc).
//
// svb_measure needs scratch space on the device for its measurement workspace (the
// approximate block sums, the per-block and per-superblock grid deltas and the exact
// CDF value at every block start), and obtains it with cudaMalloc through the handle.
// Some callers cannot do that: an application that reserves all device memory for its
// own pool at start-up (a later cudaMalloc fails or eats into the pool), or one that
// owns the state buffer itself and wants no hidden allocations, frees or the
// device-wide synchronisation a cudaFree can bring.  svb_measure_noalloc serves them:
// the caller passes device buffers for the state, the uniforms and the results, and
// the scratch comes from a fixed array in this library's device image.
//
// The array is sized for states of up to SVB_NOALLOC_MAX_QUBITS qubits (the workspace
// of measure_layout(30): about 4.1 MiB).  Every device that loads the library holds it
// until the process exits.  All calls on a device share it, so calls whose work
// overlaps on the GPU (on different streams, or from different host threads) race on
// it and must be serialised by the caller.  The kernels overwrite every entry they
// later read, so nothing needs clearing between calls.
//
// Since CUDA 12.2 modules load lazily: the module holding the array (and the
// measurement kernels) is loaded, and its ~4 MiB committed, by the first call on a
// device.  A caller that reserves the whole device afterwards should make one call
// first (shots = 0 is enough), or run with CUDA_MODULE_LOADING=EAGER.
#include <atomic>
#include <mutex>

#include "svb_internal.h"

namespace svb {
namespace {

constexpr int kNoallocMaxQubits = SVB_NOALLOC_MAX_QUBITS;
constexpr size_t kNoallocDoubles = (size_t)measure_layout(kNoallocMaxQubits).doubles;

static __device__ __align__(256) double g_noalloc_scratch[kNoallocDoubles];

constexpr int kMaxDevices = 64;
std::atomic<double*> g_addr[kMaxDevices];
std::mutex g_addr_mutex;

// Device address of g_noalloc_scratch on device `dev` (the current device), looked up
// once per device: host code cannot use the symbol's name as a device address.  The
// first lookup on a device happens under a mutex, so host threads making their first
// call at the same time do not race on the cache.
double* scratch_address(int dev, svb_status* st)
{
    *st = SVB_OK;
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("svb_measure_noalloc: device index out of range");
        *st = SVB_ERR_INVALID;
        return nullptr;
    }
    double* p = g_addr[dev].load(std::memory_order_acquire);
    if (p) return p;
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    p = g_addr[dev].load(std::memory_order_relaxed);
    if (p) return p;
    void* q = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&q, g_noalloc_scratch);
    if (e != cudaSuccess || !q) {
        set_error(std::string("svb_measure_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        *st = SVB_ERR_CUDA;
        return nullptr;
    }
    p = static_cast<double*>(q);
    g_addr[dev].store(p, std::memory_order_release);
    return p;
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
                  "]: the static scratch holds the measurement workspace of at most that many qubits");
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
    scr.cdf = scratch;
    scr.cap_doubles = kNoallocDoubles;
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

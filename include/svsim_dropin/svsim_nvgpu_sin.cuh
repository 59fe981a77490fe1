// Drop-in replacement of SV-Sim's single-GPU backend header
// (svsim/src/svsim_nvgpu_sin.cuh) for B200.
//
// The public C++ surface is the reference's: enum OP and OP_NAMES (:42-56), class Gate
// with its 9-argument constructor and dump (:99-188), class Simulation with
// Simulation(n_qubits, i_gpu), append, upload, sim, clear_circuit, reset, reset_sv,
// measure, dump, print_res_sv and the 38 static gate factories in the same argument
// order (:190-584), and the public members n_qubits, i_gpu, dim, half_dim, sv_size,
// n_gates, sv_real_cpu, sv_imag_cpu, gpu_mem, circuit.  A program that includes the
// reference header, or svsim/src/py_wrapper.cpp, compiles unchanged against this one
// (-I include/svsim_dropin -I include) and links libsvsim_b200.so.
//
// Everything behind the surface is new: the header holds no CUDA code at all; each
// call goes through the C ABI of include/svsim_b200.h into the sm_100a kernels.
// Behavioural differences, all deliberate:
//   * errors throw std::runtime_error / std::out_of_range instead of exit(-1) or assert
//     (util_nvgpu.cuh:29-65, svsim_nvgpu_sin.cuh:259-264); pybind11 turns them into
//     Python exceptions;
//   * upload() is one host-side validation + planning step, not O(gates) cudaMalloc /
//     cudaMemcpy calls (:110-160);
//   * measure() samples on the GPU with the reference's rule and its rand() draws;
//   * sv_real_cpu / sv_imag_cpu are filled lazily: sim() leaves the state on the GPU and
//     the first read of either array after it (sv_real_cpu[i], or taking it as a
//     ValType*) copies the whole state back once.  The reference copies 2^n x 16 bytes
//     back after every sim() (svsim_nvgpu_sin.cuh:328-329) whether or not the caller
//     reads them; a program that only samples never pays that copy here.  The host
//     arrays are ordinary heap memory, zero pages mapped lazily.
#ifndef SVSIM_NVGPU_SIN_CUH
#define SVSIM_NVGPU_SIN_CUH

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "config.hpp"
#include "svsim_b200.h"

namespace SVSim
{

using namespace std;

enum OP
{
    U3, U2, U1, CX, ID, X, Y, Z, H, S,
    SDG, T, TDG, RX, RY, RZ, CZ, CY, SWAP, CH,
    CCX, CSWAP, CRX, CRY, CRZ, CU1, CU3, RXX, RZZ, RCCX,
    RC3X, C3X, C3SQRTX, C4X, R, SRN, W, RYY
};

static const char* OP_NAMES[] = {
    "U3", "U2", "U1", "CX", "ID", "X", "Y", "Z", "H", "S",
    "SDG", "T", "TDG", "RX", "RY", "RZ", "CZ", "CY", "SWAP", "CH",
    "CCX", "CSWAP", "CRX", "CRY", "CRZ", "CU1", "CU3", "RXX", "RZZ", "RCCX",
    "RC3X", "C3X", "C3SQRTX", "C4X", "R", "SRN", "W", "RYY"
};

class Gate
{
public:
    Gate(enum OP _op_name,
         IdxType _qb0, IdxType _qb1, IdxType _qb2, IdxType _qb3, IdxType _qb4,
         ValType _theta, ValType _phi, ValType _lambda)
        : op_name(_op_name), qb0(_qb0), qb1(_qb1), qb2(_qb2), qb3(_qb3), qb4(_qb4),
          theta(_theta), phi(_phi), lambda(_lambda) {}
    ~Gate() {}

    void dump(std::stringstream& ss)
    {
        ss << OP_NAMES[op_name] << "(" << qb0 << "," << qb1 << "," << qb2 << "," << qb3 << ","
           << qb4 << "," << theta << "," << phi << "," << lambda << ");" << std::endl;
    }

    svb_gate to_record() const
    {
        svb_gate g;
        g.op = (uint32_t)op_name;
        g.qb[0] = (uint32_t)qb0; g.qb[1] = (uint32_t)qb1; g.qb[2] = (uint32_t)qb2;
        g.qb[3] = (uint32_t)qb3; g.qb[4] = (uint32_t)qb4;
        g.theta = theta; g.phi = phi; g.lambda = lambda;
        return g;
    }

    enum OP op_name;
    IdxType qb0;
    IdxType qb1;
    IdxType qb2;
    IdxType qb3;
    IdxType qb4;
    ValType theta;
    ValType phi;
    ValType lambda;
};

class Simulation;

// One of the two host arrays of the state.  Indexing it, or converting it to ValType*,
// first brings the host copy up to date with the device state (both arrays at once).
class HostStateArray
{
public:
    ValType& operator[](IdxType i) { sync(); return data_[i]; }
    const ValType& operator[](IdxType i) const { sync(); return data_[i]; }
    operator ValType*() { sync(); return data_; }
    operator const ValType*() const { sync(); return data_; }

private:
    friend class Simulation;
    HostStateArray() : data_(NULL), owner_(NULL) {}
    inline void sync() const;
    ValType* data_;
    Simulation* owner_;
};

class Simulation
{
public:
    Simulation(IdxType _n_qubits, IdxType _i_gpu = 0)
        : n_qubits(_n_qubits), i_gpu(_i_gpu),
          dim((IdxType)1 << _n_qubits), half_dim((IdxType)1 << (_n_qubits - 1)),
          sv_size(((IdxType)1 << _n_qubits) * (IdxType)sizeof(ValType)),
          n_gates(0), gpu_mem(0), handle(NULL), host_stale(false)
    {
        check(svb_create((uint32_t)n_qubits, (int)i_gpu, SVB_FP64, &handle), "Simulation");
        sv_real_cpu.owner_ = this;
        sv_imag_cpu.owner_ = this;
        sv_real_cpu.data_ = static_cast<ValType*>(std::calloc(dim, sizeof(ValType)));
        sv_imag_cpu.data_ = static_cast<ValType*>(std::calloc(dim, sizeof(ValType)));
        if (!sv_real_cpu.data_ || !sv_imag_cpu.data_) {
            std::free(sv_real_cpu.data_);
            std::free(sv_imag_cpu.data_);
            svb_destroy(handle);
            throw std::runtime_error("Simulation: host state allocation failed");
        }
        sv_real_cpu.data_[0] = 1.;
        gpu_mem = (ValType)(2 * sv_size);
    }

    ~Simulation()
    {
        clear_circuit();
        svb_destroy(handle);
        std::free(sv_real_cpu.data_);
        std::free(sv_imag_cpu.data_);
    }

    // Copies the device state into sv_real_cpu / sv_imag_cpu if it changed since the
    // last copy (called by the arrays themselves on access).
    void sync_host_state()
    {
        if (!host_stale) return;
        check(svb_get_state_soa(handle, sv_real_cpu.data_, sv_imag_cpu.data_), "sv_real_cpu");
        host_stale = false;
    }

    void reset()
    {
        clear_circuit();
        reset_sv();
    }

    void reset_sv()
    {
        check(svb_reset_state(handle), "reset_sv");
        std::memset(sv_real_cpu.data_, 0, sv_size);
        std::memset(sv_imag_cpu.data_, 0, sv_size);
        sv_real_cpu.data_[0] = 1;
        host_stale = false;
    }

    // The gate is copied (pybind11 owns and frees the factory's object).
    void append(Gate* g)
    {
        if (g == NULL) throw std::invalid_argument("append: NULL gate");
        if (g->qb0 >= n_qubits || g->qb1 >= n_qubits || g->qb2 >= n_qubits ||
            g->qb3 >= n_qubits || g->qb4 >= n_qubits)
            throw std::out_of_range("append: qubit index >= n_qubits");
        circuit.push_back(new Gate(*g));
        n_gates++;
    }

    Simulation* upload()
    {
        std::vector<svb_gate> recs;
        recs.reserve(circuit.size());
        for (size_t t = 0; t < circuit.size(); t++) recs.push_back(circuit[t]->to_record());
        check(svb_set_circuit(handle, recs.data(), recs.size()), "upload");
        return this;
    }

    std::string dump()
    {
        std::stringstream ss;
        for (IdxType t = 0; t < n_gates; t++) circuit[t]->dump(ss);
        return ss.str();
    }

    // Runs the uploaded circuit on the device state.  sv_real_cpu / sv_imag_cpu follow
    // on their next read (the reference copies them back here, :328-329).
    void sim()
    {
        const double t0 = wall_ms();
        check(svb_run(handle, NULL), "sim");
        check(svb_synchronize(handle), "sim");
        const double sim_time = wall_ms() - t0;
        host_stale = true;
#ifdef PRINT_MEA_PER_CIRCUIT
        printf("\n============== SV-Sim: NVIDIA-GPU-SIN (B200) ===============\n");
        printf("nqubits:%llu, ngates:%llu, ncores:%d, sim:%.3lf ms, mem:%.3lf MB, mem_per_gpu:%.3lf MB\n",
               (unsigned long long)n_qubits, (unsigned long long)n_gates, 1, sim_time,
               gpu_mem / 1024 / 1024, gpu_mem / 1024 / 1024);
        printf("=======================================================\n");
#endif
    }

    void clear_circuit()
    {
        for (size_t i = 0; i < circuit.size(); i++) delete circuit[i];
        circuit.clear();
        n_gates = 0;
        svb_clear_circuit(handle);
    }

    // Samples `repetition` basis states with rand()/RAND_MAX draws after
    // srand(RAND_SEED), as the reference does; the caller frees with delete[].
    IdxType* measure(unsigned repetition = 10)
    {
        std::vector<double> u(repetition);
        srand(RAND_SEED);
        for (unsigned i = 0; i < repetition; i++) u[i] = (ValType)rand() / (ValType)RAND_MAX;
        std::vector<uint64_t> out(repetition);
        double total = 0;
        check(svb_measure(handle, u.data(), repetition, out.data(), &total), "measure");
        IdxType* res_state = new IdxType[repetition];
        for (unsigned i = 0; i < repetition; i++) res_state[i] = (IdxType)out[i];
        if (std::fabs(total - 1.0) > ERROR_BAR)
            printf("Sum of probability is far from 1.0 with %lf\n", total);
        return res_state;
    }

    void print_res_sv()
    {
        printf("----- Real SV ------\n");
        for (IdxType i = 0; i < dim; i++) printf("%lf ", sv_real_cpu[i]);
        printf("\n");
        printf("----- Imag SV ------\n");
        for (IdxType i = 0; i < dim; i++) printf("%lf ", sv_imag_cpu[i]);
        printf("\n");
    }

    // ---- static gate factories (argument order of :397-584) ----
    static Gate* U3(ValType theta, ValType phi, ValType lambda, IdxType m)
    { return new Gate(OP::U3, m, 0, 0, 0, 0, theta, phi, lambda); }
    static Gate* U2(ValType phi, ValType lambda, IdxType m)
    { return new Gate(OP::U2, m, 0, 0, 0, 0, 0., phi, lambda); }
    static Gate* U1(ValType lambda, IdxType m)
    { return new Gate(OP::U1, m, 0, 0, 0, 0, 0., 0., lambda); }
    static Gate* CX(IdxType m, IdxType n) { return new Gate(OP::CX, m, n, 0, 0, 0, 0., 0., 0.); }
    static Gate* ID(IdxType m) { return new Gate(OP::ID, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* X(IdxType m) { return new Gate(OP::X, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* Y(IdxType m) { return new Gate(OP::Y, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* Z(IdxType m) { return new Gate(OP::Z, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* H(IdxType m) { return new Gate(OP::H, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* S(IdxType m) { return new Gate(OP::S, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* SDG(IdxType m) { return new Gate(OP::SDG, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* T(IdxType m) { return new Gate(OP::T, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* TDG(IdxType m) { return new Gate(OP::TDG, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* RX(ValType theta, IdxType m)
    { return new Gate(OP::RX, m, 0, 0, 0, 0, theta, 0., 0.); }
    static Gate* RY(ValType theta, IdxType m)
    { return new Gate(OP::RY, m, 0, 0, 0, 0, theta, 0., 0.); }
    static Gate* RZ(ValType phi, IdxType m)
    { return new Gate(OP::RZ, m, 0, 0, 0, 0, 0., phi, 0.); }
    static Gate* CZ(IdxType m, IdxType n) { return new Gate(OP::CZ, m, n, 0, 0, 0, 0., 0., 0.); }
    static Gate* CY(IdxType m, IdxType n) { return new Gate(OP::CY, m, n, 0, 0, 0, 0., 0., 0.); }
    static Gate* SWAP(IdxType m, IdxType n) { return new Gate(OP::SWAP, m, n, 0, 0, 0, 0., 0., 0.); }
    static Gate* CH(IdxType m, IdxType n) { return new Gate(OP::CH, m, n, 0, 0, 0, 0., 0., 0.); }
    static Gate* CCX(IdxType l, IdxType m, IdxType n)
    { return new Gate(OP::CCX, l, m, n, 0, 0, 0., 0., 0.); }
    static Gate* CSWAP(IdxType l, IdxType m, IdxType n)
    { return new Gate(OP::CSWAP, l, m, n, 0, 0, 0., 0., 0.); }
    static Gate* CRX(ValType lambda, IdxType m, IdxType n)
    { return new Gate(OP::CRX, m, n, 0, 0, 0, 0., 0., lambda); }
    static Gate* CRY(ValType lambda, IdxType m, IdxType n)
    { return new Gate(OP::CRY, m, n, 0, 0, 0, 0., 0., lambda); }
    static Gate* CRZ(ValType lambda, IdxType m, IdxType n)
    { return new Gate(OP::CRZ, m, n, 0, 0, 0, 0., 0., lambda); }
    static Gate* CU1(ValType lambda, IdxType m, IdxType n)
    { return new Gate(OP::CU1, m, n, 0, 0, 0, 0., 0., lambda); }
    static Gate* CU3(ValType theta, ValType phi, ValType lambda, IdxType m, IdxType n)
    { return new Gate(OP::CU3, m, n, 0, 0, 0, theta, phi, lambda); }
    static Gate* RXX(ValType theta, IdxType m, IdxType n)
    { return new Gate(OP::RXX, m, n, 0, 0, 0, theta, 0., 0.); }
    static Gate* RZZ(ValType theta, IdxType m, IdxType n)
    { return new Gate(OP::RZZ, m, n, 0, 0, 0, theta, 0., 0.); }
    static Gate* RCCX(IdxType l, IdxType m, IdxType n)
    { return new Gate(OP::RCCX, l, m, n, 0, 0, 0., 0., 0.); }
    static Gate* RC3X(IdxType l, IdxType m, IdxType n, IdxType o)
    { return new Gate(OP::RC3X, l, m, n, o, 0, 0., 0., 0.); }
    static Gate* C3X(IdxType l, IdxType m, IdxType n, IdxType o)
    { return new Gate(OP::C3X, l, m, n, o, 0, 0., 0., 0.); }
    static Gate* C3SQRTX(IdxType l, IdxType m, IdxType n, IdxType o)
    { return new Gate(OP::C3SQRTX, l, m, n, o, 0, 0., 0., 0.); }
    static Gate* C4X(IdxType l, IdxType m, IdxType n, IdxType o, IdxType p)
    { return new Gate(OP::C4X, l, m, n, o, p, 0., 0., 0.); }
    static Gate* R(ValType theta, IdxType m) { return new Gate(OP::R, m, 0, 0, 0, 0, theta, 0., 0.); }
    static Gate* SRN(IdxType m) { return new Gate(OP::SRN, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* W(IdxType m) { return new Gate(OP::W, m, 0, 0, 0, 0, 0., 0., 0.); }
    static Gate* RYY(ValType theta, IdxType m, IdxType n)
    { return new Gate(OP::RYY, m, n, 0, 0, 0, theta, 0., 0.); }

public:
    const IdxType n_qubits;
    const IdxType i_gpu;
    const IdxType dim;
    const IdxType half_dim;
    const IdxType sv_size;
    IdxType n_gates;
    HostStateArray sv_real_cpu;   // host copy of the state, filled on first read after sim()
    HostStateArray sv_imag_cpu;
    ValType gpu_mem;          // bytes of device state, as a double (as the reference)
    vector<Gate*> circuit;
    svb_sim* handle;          // the engine behind this simulation
    bool host_stale;          // the device state changed since the last host copy

private:
    static void check(svb_status st, const char* where)
    {
        if (st != SVB_OK) throw std::runtime_error(std::string(where) + ": " + svb_last_error());
    }
    static double wall_ms()
    {
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
    }
    Simulation(const Simulation&);
    Simulation& operator=(const Simulation&);
};

inline void HostStateArray::sync() const
{
    if (owner_) owner_->sync_host_state();
}

}  // namespace SVSim

#endif

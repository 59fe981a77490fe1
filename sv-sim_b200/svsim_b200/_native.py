"""ctypes binding of libsvsim_b200.so (C ABI in include/svsim_b200.h).

The library is loaded from the package's lib/ directory.  There is no fallback: if
the library is missing or was built for another architecture, importing this module
raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .gates import GATE_DTYPE, PARAM_DTYPE, PAULI_DTYPE

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libsvsim_b200.so")

SVB_OK, SVB_ERR_INVALID, SVB_ERR_CUDA, SVB_ERR_OOM, SVB_ERR_UNSUPPORTED, SVB_ERR_STATE = range(6)
SVB_FP64, SVB_FP32 = 0, 1
ENGINE_AUTO, ENGINE_PER_GATE, ENGINE_STAGED, ENGINE_FUSED, ENGINE_PAIRS = 0, 1, 2, 3, 4


class SvbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[svb status {status}] {message}")
        self.status = status


class PlanInfo(ctypes.Structure):
    _fields_ = [("n_gates", ctypes.c_uint64), ("n_elementary", ctypes.c_uint64),
                ("n_passes", ctypes.c_uint64), ("n_sweeps_model", ctypes.c_uint64),
                ("state_bytes", ctypes.c_double), ("model_bytes", ctypes.c_double),
                ("moved_bytes", ctypes.c_double), ("plan_bytes", ctypes.c_uint64),
                ("engine", ctypes.c_int),
                ("tile_bits", ctypes.c_int), ("n_blocks", ctypes.c_uint64)]


class QaoaStats(ctypes.Structure):
    _fields_ = [("n_instances", ctypes.c_uint32), ("p", ctypes.c_uint32),
                ("tile_bits", ctypes.c_uint32), ("graphed", ctypes.c_uint32),
                ("total_amplitudes", ctypes.c_uint64), ("tiles_per_pass", ctypes.c_uint64),
                ("moved_bytes", ctypes.c_double), ("grid", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class TuneResult(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_int), ("tile_bits", ctypes.c_int), ("fusion_width", ctypes.c_int),
                ("candidates", ctypes.c_int), ("best_ms", ctypes.c_double), ("default_ms", ctypes.c_double),
                ("timed_gates", ctypes.c_uint64)]


class CbatchStats(ctypes.Structure):
    _fields_ = [("n_circuits", ctypes.c_uint32), ("n_phases", ctypes.c_uint32),
                ("tile_bits", ctypes.c_uint32), ("threads", ctypes.c_uint32),
                ("pool_amplitudes", ctypes.c_uint64), ("items", ctypes.c_uint64),
                ("grid", ctypes.c_uint32), ("graphed", ctypes.c_uint32),
                ("moved_bytes", ctypes.c_double), ("tuned", ctypes.c_uint32),
                ("n_passes", ctypes.c_uint32), ("pair_circuits", ctypes.c_uint32),
                ("pair_passes", ctypes.c_uint32), ("pair_phases", ctypes.c_uint32),
                ("pair_grid", ctypes.c_uint32)]


_lib = None

_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)

_SIGS = {
    "svb_create": ([ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
    "svb_destroy": ([_vp], ctypes.c_int),
    "svb_reset_state": ([_vp], ctypes.c_int),
    "svb_set_circuit": ([_vp, _vp, ctypes.c_size_t], ctypes.c_int),
    "svb_clear_circuit": ([_vp], ctypes.c_int),
    "svb_set_engine": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "svb_get_plan_info": ([_vp, ctypes.POINTER(PlanInfo)], ctypes.c_int),
    "svb_run": ([_vp, _vp], ctypes.c_int),
    "svb_synchronize": ([_vp], ctypes.c_int),
    "svb_get_state_soa": ([_vp, _dp, _dp], ctypes.c_int),
    "svb_set_state_soa": ([_vp, _dp, _dp], ctypes.c_int),
    "svb_state_device_ptr": ([_vp, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "svb_measure": ([_vp, _dp, ctypes.c_uint32, _u64p, _dp], ctypes.c_int),
    "svb_measure_seeded": ([_vp, ctypes.c_uint32, ctypes.c_uint32, _u64p, _dp], ctypes.c_int),
    "svb_norm2": ([_vp, _dp], ctypes.c_int),
    "svb_expectation": ([_vp, _vp, ctypes.c_size_t, _dp], ctypes.c_int),
    "svb_adjoint": ([_vp, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, _vp, ctypes.c_size_t, _dp, _dp],
                    ctypes.c_int),
    "svb_compare_states": ([_vp, _vp, _dp, _dp], ctypes.c_int),
    "svb_qaoa_create": ([ctypes.c_int, ctypes.c_int, ctypes.c_uint32, _vp, _vp, _vp, _vp, ctypes.c_uint32,
                         ctypes.POINTER(_vp)], ctypes.c_int),
    "svb_qaoa_run": ([_vp, _dp, _dp, _dp, _dp], ctypes.c_int),
    "svb_qaoa_launch": ([_vp, _vp], ctypes.c_int),
    "svb_qaoa_info": ([_vp, ctypes.POINTER(QaoaStats)], ctypes.c_int),
    "svb_qaoa_destroy": ([_vp], ctypes.c_int),
    "svb_apply_controlled": ([_vp, ctypes.c_uint32, ctypes.c_uint64, _dp, _vp], ctypes.c_int),
    "svb_measure_qubit": ([_vp, ctypes.c_uint32, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                           _dp], ctypes.c_int),
    "svb_dm_create": ([ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
    "svb_dm_set_circuit": ([_vp, _vp, ctypes.c_size_t, _dp, ctypes.c_uint32], ctypes.c_int),
    "svb_dm_set_circuit_superops": ([_vp, _vp, ctypes.c_size_t, _dp, ctypes.c_uint32, _vp, ctypes.c_size_t],
                                    ctypes.c_int),
    "svb_dm_probabilities": ([_vp, _dp], ctypes.c_int),
    "svb_autotune": ([_vp, _vp, ctypes.c_size_t, ctypes.POINTER(TuneResult)], ctypes.c_int),
    "svb_cbatch_create": ([ctypes.c_int, ctypes.c_int, ctypes.c_uint32, _vp, _vp, _vp, _vp, _vp, ctypes.c_int,
                           ctypes.POINTER(_vp)], ctypes.c_int),
    "svb_cbatch_run": ([_vp, _vp, _dp], ctypes.c_int),
    "svb_cbatch_get_state": ([_vp, ctypes.c_uint32, _dp, _dp], ctypes.c_int),
    "svb_cbatch_info": ([_vp, ctypes.POINTER(CbatchStats)], ctypes.c_int),
    "svb_cbatch_destroy": ([_vp], ctypes.c_int),
    "svb_last_error": ([], ctypes.c_char_p),
    "svb_version": ([], ctypes.c_char_p),
    "svb_fp64_mma_peak": ([ctypes.c_int, _dp], ctypes.c_int),
    "svb_l2_copy_peak": ([ctypes.c_int, _dp], ctypes.c_int),
    "svb_selftest_waits": ([ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
                           ctypes.c_int),
}


def lib():
    """The loaded library; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libsvsim_b200.so not built ({LIB_PATH}); run "
                              "`python sv-sim_b200/svsim_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(status: int):
    if status != SVB_OK:
        raise SvbError(status, lib().svb_last_error().decode())


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def fp64_mma_peak(device: int = 0) -> float:
    """FP64 tensor-core rate in TFLOP/s measured on `device` (svb_fp64_mma_peak)."""
    v = ctypes.c_double()
    check(lib().svb_fp64_mma_peak(device, ctypes.byref(v)))
    return v.value


def selftest_waits(device: int = 0) -> tuple[bool, bool]:
    """(mbarrier wait gave up, grid barrier gave up) for waits made to run out on purpose
    (svb_selftest_waits); both must be True."""
    m, g = ctypes.c_int(), ctypes.c_int()
    check(lib().svb_selftest_waits(device, ctypes.byref(m), ctypes.byref(g)))
    return bool(m.value), bool(g.value)


def l2_copy_peak(device: int = 0) -> float:
    """L2 copy bandwidth in GB/s measured on `device` (svb_l2_copy_peak)."""
    v = ctypes.c_double()
    check(lib().svb_l2_copy_peak(device, ctypes.byref(v)))
    return v.value


class Handle:
    """Owns one svb_sim*."""

    def __init__(self, n_qubits: int, device: int = 0, precision: int = SVB_FP64):
        h = _vp()
        check(lib().svb_create(n_qubits, device, precision, ctypes.byref(h)))
        self.ptr = h
        self.n = n_qubits
        self.precision = precision

    def close(self):
        if getattr(self, "ptr", None):
            lib().svb_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- wrappers ------------------------------------------------------------------
    def set_engine(self, engine=ENGINE_AUTO, tile_bits=0, fusion_width=0):
        check(lib().svb_set_engine(self.ptr, engine, tile_bits, fusion_width))

    def autotune(self, gates: np.ndarray) -> TuneResult:
        """Times the engines that can run `gates` and keeps the fastest for circuits of this
        structure (svb_autotune); the handle ends with `gates` set and the state at |0..0>."""
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        r = TuneResult()
        check(lib().svb_autotune(self.ptr, g.ctypes.data, len(g), ctypes.byref(r)))
        return r

    def set_circuit(self, gates: np.ndarray):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        check(lib().svb_set_circuit(self.ptr, g.ctypes.data, len(g)))

    def clear_circuit(self):
        check(lib().svb_clear_circuit(self.ptr))

    def reset(self):
        check(lib().svb_reset_state(self.ptr))

    def run(self, stream: int = 0):
        check(lib().svb_run(self.ptr, _vp(stream) if stream else None))

    def sync(self):
        check(lib().svb_synchronize(self.ptr))

    def plan_info(self) -> PlanInfo:
        info = PlanInfo()
        check(lib().svb_get_plan_info(self.ptr, ctypes.byref(info)))
        return info

    def get_state(self):
        dim = 1 << self.n
        re = np.empty(dim)
        im = np.empty(dim)
        check(lib().svb_get_state_soa(self.ptr, dptr(re), dptr(im)))
        return re, im

    def set_state(self, re, im):
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        check(lib().svb_set_state_soa(self.ptr, dptr(re), dptr(im)))

    def device_ptr(self):
        p = _vp()
        prec = ctypes.c_int()
        check(lib().svb_state_device_ptr(self.ptr, ctypes.byref(p), ctypes.byref(prec)))
        return p.value, prec.value

    def measure(self, uniforms):
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        out = np.zeros(len(u), dtype=np.uint64)
        tot = ctypes.c_double()
        check(lib().svb_measure(self.ptr, dptr(u), len(u), out.ctypes.data_as(_u64p),
                                ctypes.byref(tot)))
        return out, tot.value

    def measure_seeded(self, seed: int, shots: int):
        """The reference's measure() with srand(seed) in place of srand(time(0))."""
        out = np.zeros(shots, dtype=np.uint64)
        tot = ctypes.c_double()
        check(lib().svb_measure_seeded(self.ptr, ctypes.c_uint32(seed), shots, out.ctypes.data_as(_u64p),
                                       ctypes.byref(tot)))
        return out, tot.value

    def norm2(self) -> float:
        v = ctypes.c_double()
        check(lib().svb_norm2(self.ptr, ctypes.byref(v)))
        return v.value

    def expectation(self, terms) -> float:
        t = np.ascontiguousarray(terms, dtype=PAULI_DTYPE)
        v = ctypes.c_double()
        check(lib().svb_expectation(self.ptr, t.ctypes.data, len(t), ctypes.byref(v)))
        return v.value

    def compare(self, other: "Handle"):
        """(fidelity, max |a_i - b_i|) against another handle's state, in FP64."""
        f = ctypes.c_double()
        d = ctypes.c_double()
        check(lib().svb_compare_states(self.ptr, other.ptr, ctypes.byref(f), ctypes.byref(d)))
        return f.value, d.value

    def apply_controlled(self, target: int, controls, matrix, stream: int = 0):
        """Applies the complex 2x2 `matrix` to `target` where every qubit in `controls`
        is 1 (the Q# variant's masked controlled gates)."""
        mask = 0
        for c in controls:
            mask |= 1 << int(c)
        u = np.asarray(matrix, dtype=np.complex128).reshape(2, 2)
        m = np.array([u[0, 0].real, u[0, 0].imag, u[0, 1].real, u[0, 1].imag,
                      u[1, 0].real, u[1, 0].imag, u[1, 1].real, u[1, 1].imag])
        check(lib().svb_apply_controlled(self.ptr, target, mask, dptr(m), _vp(stream)))

    def measure_qubit(self, qubit: int, r: float, pauli: int = 0):
        """Mid-circuit measurement with collapse: returns (outcome, P(1))."""
        out = ctypes.c_int()
        p1 = ctypes.c_double()
        check(lib().svb_measure_qubit(self.ptr, qubit, pauli, float(r), ctypes.byref(out), ctypes.byref(p1)))
        return out.value, p1.value

    def adjoint(self, gates, bindings, n_params, terms):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        b = np.ascontiguousarray(bindings, dtype=PARAM_DTYPE)
        t = np.ascontiguousarray(terms, dtype=PAULI_DTYPE)
        grad = np.zeros(max(n_params, 1))
        e = ctypes.c_double()
        check(lib().svb_adjoint(self.ptr, g.ctypes.data, b.ctypes.data, len(g), n_params,
                                t.ctypes.data, len(t), ctypes.byref(e), dptr(grad)))
        return e.value, grad[:n_params]


class QaoaBatch:
    """A batch of MaxCut QAOA instances (svb_qaoa_create): energy and gradient of every
    instance per call of ``run``."""

    def __init__(self, instances, device: int = 0, precision: int = SVB_FP64):
        ps = {len(inst.gammas) for inst in instances}
        if len(ps) != 1:
            raise ValueError("all instances of a batch need the same depth p")
        self.p = ps.pop()
        self.n_inst = len(instances)
        nq = np.array([inst.n for inst in instances], dtype=np.uint32)
        counts = np.array([len(inst.edges) for inst in instances], dtype=np.uint32)
        eoff = np.zeros(self.n_inst + 1, dtype=np.uint32)
        np.cumsum(counts, out=eoff[1:])
        edges = np.ascontiguousarray(np.concatenate([np.asarray(i.edges, dtype=np.uint32).reshape(-1, 2)
                                                     for i in instances]), dtype=np.uint32)
        w = np.ascontiguousarray(np.concatenate([np.asarray(i.weights, dtype=np.float64)
                                                 for i in instances]))
        self.ptr = _vp()
        check(lib().svb_qaoa_create(device, precision, self.n_inst, nq.ctypes.data, eoff.ctypes.data,
                                    edges.ctypes.data, w.ctypes.data, self.p, ctypes.byref(self.ptr)))

    def close(self):
        if self.ptr:
            lib().svb_qaoa_destroy(self.ptr)
            self.ptr = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, gammas, betas):
        """gammas, betas: [n_instances, p].  Returns (energies [n], grads [n, 2p])."""
        g = np.ascontiguousarray(gammas, dtype=np.float64).reshape(self.n_inst, self.p)
        b = np.ascontiguousarray(betas, dtype=np.float64).reshape(self.n_inst, self.p)
        e = np.zeros(self.n_inst)
        gr = np.zeros((self.n_inst, 2 * self.p))
        check(lib().svb_qaoa_run(self.ptr, dptr(g), dptr(b), dptr(e), dptr(gr)))
        return e, gr

    def launch(self, stream: int = 0):
        check(lib().svb_qaoa_launch(self.ptr, _vp(stream)))

    def info(self) -> QaoaStats:
        st = QaoaStats()
        check(lib().svb_qaoa_info(self.ptr, ctypes.byref(st)))
        return st


CBATCH_PAIRS = -1   # svb_cbatch_create: the pair engine where it can run


class CircuitBatch:
    """Many independent circuits (each its own qubit count, 1..24) run together by one
    persistent, graph-replayed launch (svb_cbatch_*), with an optional Pauli-sum energy per
    circuit.  tile_bits=0 lets the autotuner choose the tile and block sizes and whether the
    pair engine runs the FP64 circuits of 12 or more qubits; CBATCH_PAIRS asks for the pair
    engine; 6..13 for shared-memory sweeps of that tile size."""

    def __init__(self, circuits, terms=None, device: int = 0, precision: int = SVB_FP64, tile_bits: int = 0):
        """circuits: list of (n_qubits, gate record array); terms: None or a list (one per
        circuit) of Pauli-term arrays (PAULI_DTYPE) or None."""
        self.n = np.array([int(c[0]) for c in circuits], dtype=np.uint32)
        self.gate_arrays = [np.ascontiguousarray(c[1], dtype=GATE_DTYPE) for c in circuits]
        self.gate_off = np.zeros(len(circuits) + 1, dtype=np.uint64)
        np.cumsum([len(g) for g in self.gate_arrays], out=self.gate_off[1:])
        gates = np.ascontiguousarray(np.concatenate(self.gate_arrays) if len(self.gate_arrays) else
                                     np.zeros(0, dtype=GATE_DTYPE))
        self._gates = gates
        toff = None
        t = None
        if terms is not None:
            ts = [np.zeros(0, dtype=PAULI_DTYPE) if x is None else np.ascontiguousarray(x, dtype=PAULI_DTYPE)
                  for x in terms]
            toff = np.zeros(len(circuits) + 1, dtype=np.uint64)
            np.cumsum([len(x) for x in ts], out=toff[1:])
            t = np.ascontiguousarray(np.concatenate(ts) if ts else np.zeros(0, dtype=PAULI_DTYPE))
        self._terms, self._toff = t, toff
        self.ptr = _vp()
        check(lib().svb_cbatch_create(device, precision, len(circuits), self.n.ctypes.data,
                                      self.gate_off.ctypes.data, gates.ctypes.data if len(gates) else None,
                                      toff.ctypes.data if toff is not None else None,
                                      t.ctypes.data if t is not None and len(t) else None,
                                      tile_bits, ctypes.byref(self.ptr)))

    def run(self, gates=None) -> np.ndarray:
        """Energies of every circuit (zeros without terms); `gates`: the concatenated gate
        records with new angles (same ops and qubits), or None."""
        e = np.zeros(len(self.n))
        g = None
        if gates is not None:
            g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
            if len(g) != len(self._gates):
                raise ValueError("gates: the batch's gate count")
        check(lib().svb_cbatch_run(self.ptr, g.ctypes.data if g is not None else None, dptr(e)))
        return e

    def state(self, i: int) -> np.ndarray:
        dim = 1 << int(self.n[i])
        re = np.empty(dim)
        im = np.empty(dim)
        check(lib().svb_cbatch_get_state(self.ptr, i, dptr(re), dptr(im)))
        return re + 1j * im

    def info(self) -> CbatchStats:
        st = CbatchStats()
        check(lib().svb_cbatch_info(self.ptr, ctypes.byref(st)))
        return st

    def close(self):
        if self.ptr:
            lib().svb_cbatch_destroy(self.ptr)
            self.ptr = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

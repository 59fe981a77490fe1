"""TEST INFRASTRUCTURE ONLY — ctypes access to the CPU checkers.

  * ``Oracle``    — the C restatement (oracle/_build/liboracle.so, built from
                    svsim_oracle.c); always available once ``make -C oracle oracle`` ran.
  * ``RefBackend`` — the reference's own CPU backends compiled in place by
                    oracle/Makefile into oracle/_ref/ (absent when the reference tree was
                    not there at build time).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline arm import this
module; the product path never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference tree is read from when the checkers are built (the one setting;
# oracle/Makefile takes it as REF).
REFERENCE = os.environ.get("SVSIM_REFERENCE", "/root/reference")
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


def build(reference: bool = True) -> None:
    """Build the restatement, and the reference backends when the reference tree exists."""
    targets = ["oracle"]
    if reference and os.path.isdir(os.path.join(REFERENCE, "svsim", "src")):
        targets += ["ref", "ref_gpu"]
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE}"] + targets, check=True)


class Oracle:
    def __init__(self):
        path = os.path.join(BUILD, "liboracle.so")
        if not os.path.exists(path):
            build(reference=False)
        self.lib = lib = ctypes.CDLL(path)
        lib.oracle_run.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_size_t, _dp, _dp]
        lib.oracle_apply.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_size_t, _dp, _dp]
        lib.oracle_measure_uniforms.argtypes = [ctypes.c_uint32, _dp, _dp, _dp, ctypes.c_uint32,
                                                _u64p, _dp]
        lib.oracle_expectation.argtypes = [ctypes.c_uint32, _dp, _dp, ctypes.c_void_p,
                                           ctypes.c_size_t]
        lib.oracle_expectation.restype = ctypes.c_double
        lib.oracle_elementary_count.argtypes = [ctypes.c_uint32]

    def run(self, n: int, gates: np.ndarray, state=None):
        """Returns (re, im) after applying `gates` to |0..0> (or to `state`=(re, im))."""
        gates = np.ascontiguousarray(gates)
        if state is None:
            re = np.empty(1 << n)
            im = np.empty(1 << n)
            rc = self.lib.oracle_run(n, gates.ctypes.data, len(gates), _ptr(re), _ptr(im))
        else:
            re = np.array(state[0], dtype=np.float64, copy=True)
            im = np.array(state[1], dtype=np.float64, copy=True)
            rc = self.lib.oracle_apply(n, gates.ctypes.data, len(gates), _ptr(re), _ptr(im))
        if rc != 0:
            raise ValueError("oracle: unknown gate op")
        return re, im

    def measure(self, n, re, im, uniforms):
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        out = np.zeros(len(u), dtype=np.uint64)
        tot = ctypes.c_double()
        self.lib.oracle_measure_uniforms(n, _ptr(re), _ptr(im), _ptr(u), len(u), _ptr(out, _u64p),
                                         ctypes.byref(tot))
        return out, tot.value

    def expectation(self, n, re, im, terms):
        terms = np.ascontiguousarray(terms)
        return self.lib.oracle_expectation(n, _ptr(re), _ptr(im), terms.ctypes.data, len(terms))

    def elementary_count(self, op: int) -> int:
        return self.lib.oracle_elementary_count(op)


class RefBackend:
    """The reference's svsim_cpu_sin.hpp / svsim_cpu_omp.hpp behind ref_glue.cpp."""

    def __init__(self, kind: str = "sin"):
        name = {"sin": "libref_cpu_sin.so", "omp": "libref_cpu_omp.so",
                "omp64": "libref_cpu_omp64.so"}[kind]
        path = os.path.join(REF, name)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.kind = kind
        self.lib = lib = ctypes.CDLL(path)
        lib.ref_simulate.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_uint64, _dp, _dp, _dp, ctypes.c_uint32,
                                     ctypes.c_ulong, _u64p, ctypes.c_int]
        lib.ref_idx_bits.restype = ctypes.c_int
        self.idx_bits = lib.ref_idx_bits()

    @staticmethod
    def available(kind: str = "sin") -> bool:
        try:
            RefBackend(kind)
            return True
        except (FileNotFoundError, OSError):
            return False

    def open(self, n: int, threads: int):
        """A persistent reference Simulation (state kept across runs)."""
        L = self.lib
        L.ref_handle_open.argtypes = [ctypes.c_uint32, ctypes.c_int]
        L.ref_handle_open.restype = ctypes.c_void_p
        L.ref_handle_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, _dp,
                                     ctypes.c_int]
        L.ref_handle_close.argtypes = [ctypes.c_void_p]
        h = L.ref_handle_open(n, threads)
        if not h:
            raise ValueError(f"reference backend rejected n={n}")
        return h

    def run_on(self, h, gates: np.ndarray) -> float:
        gates = np.ascontiguousarray(gates)
        ms = ctypes.c_double()
        self.lib.ref_handle_run(h, gates.ctypes.data, len(gates), ctypes.byref(ms), 1)
        return ms.value

    def close(self, h):
        self.lib.ref_handle_close(h)

    def simulate(self, n: int, gates: np.ndarray, threads: int = 1, shots: int = 0,
                 seed: int = 1, want_state: bool = True):
        """Returns dict(re, im, sim_ms, samples)."""
        gates = np.ascontiguousarray(gates)
        re = np.empty(1 << n) if want_state else None
        im = np.empty(1 << n) if want_state else None
        ms = ctypes.c_double()
        samples = np.zeros(max(shots, 1), dtype=np.uint64)
        rc = self.lib.ref_simulate(n, threads, gates.ctypes.data, len(gates), _ptr(re), _ptr(im),
                                   ctypes.byref(ms), shots, seed, _ptr(samples, _u64p), 1)
        if rc != 0:
            raise ValueError(f"reference backend rejected n={n}")
        return {"re": re, "im": im, "sim_ms": ms.value, "samples": samples[:shots]}


def libc_uniforms(seed: int, count: int) -> np.ndarray:
    """r_i = rand()/RAND_MAX after srand(seed): the draws Simulation::measure makes
    (svsim_cpu_sin.hpp:330-334) once its seed is fixed."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(seed))
    RAND_MAX = 2147483647
    return np.array([libc.rand() / RAND_MAX for _ in range(count)], dtype=np.float64)

"""Python mirror of the reference's ``Simulation`` API over the C ABI.

Same names, argument meaning and call order as the reference's pybind11 module
(svsim/src/py_wrapper.cpp:53-109): ``Simulation(n_qubits, i_gpu)``, ``append``,
``upload``, ``run``, ``clear_circuit``, ``reset``, ``measure(repetition)`` and the 38
static gate factories.  Differences, all deliberate:

* ``append`` validates eagerly and raises ``ValueError`` (the reference asserts,
  svsim_nvgpu_sin.cuh:259-264, and its asserts vanish under -DNDEBUG);
* ``run`` leaves the state on the GPU; ``state()`` / ``sv_real_cpu`` copy it back on
  demand instead of after every run (:328-329);
* ``measure`` samples on the GPU with the reference's rule; its uniforms are the
  reference's ``rand()/RAND_MAX`` draws after ``srand(time(0))`` (:367-371), or the
  caller's via ``measure_with_uniforms``.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import gates as _g
from ._native import (ENGINE_AUTO, SVB_FP32, SVB_FP64, Handle)


def _libc_uniforms(count: int, seed: int | None = None) -> np.ndarray:
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(int(time.time()) if seed is None else seed))
    RAND_MAX = 2147483647
    return np.array([libc.rand() / RAND_MAX for _ in range(count)], dtype=np.float64)


class Simulation:
    def __init__(self, n_qubits: int, i_gpu: int = 0, precision: str = "fp64",
                 engine: int = ENGINE_AUTO, tile_bits: int = 0):
        prec = {"fp64": SVB_FP64, "fp32": SVB_FP32}[precision]
        self.n_qubits = int(n_qubits)
        self.i_gpu = int(i_gpu)
        self.dim = 1 << self.n_qubits
        self.half_dim = self.dim >> 1
        self._h = Handle(self.n_qubits, self.i_gpu, prec)
        self._h.set_engine(engine, tile_bits, 0)
        self.circuit: list[_g.Gate] = []
        self._uploaded = False

    @classmethod
    def from_qasm(cls, source: str, i_gpu: int = 0, precision: str = "fp64",
                  engine: int = ENGINE_AUTO, tile_bits: int = 0, strict: bool = False) -> "Simulation":
        """A Simulation holding an OpenQASM 2.0 program (a file path or the program text),
        with one qubit per declared qubit (registers in declaration order).  The
        program's measure records are kept in ``qasm_measured`` and the statements dropped
        as the reference's translator drops them (reset, if, opaque) in ``qasm_skipped``;
        ``strict=True`` rejects those instead."""
        import os
        from . import qasm
        prog = (qasm.load(source, strict=strict) if os.path.isfile(source)
                else qasm.loads(source, strict=strict))
        sim = cls(prog.n_qubits, i_gpu, precision, engine, tile_bits)
        for g in _g.from_array(prog.gates):
            sim.append(g)
        sim.qasm_measured = prog.measured
        sim.qasm_skipped = prog.skipped
        return sim

    # ---- circuit ----------------------------------------------------------------------
    @property
    def n_gates(self) -> int:
        return len(self.circuit)

    def append(self, g: _g.Gate):
        if g is None:
            raise ValueError("append: NULL gate")
        for q in g.qb:
            if not 0 <= q < self.n_qubits:
                raise ValueError(f"append: qubit {q} out of range for {self.n_qubits} qubits")
        self.circuit.append(_g.Gate(g.op, *g.qb, g.theta, g.phi, g.lam))
        self._uploaded = False

    def upload(self):
        self._h.set_circuit(_g.to_array(self.circuit))
        self._uploaded = True
        return self

    def run(self):
        if not self._uploaded:
            self.upload()
        self._h.run()
        self._h.sync()

    sim = run

    def clear_circuit(self):
        self.circuit = []
        self._h.clear_circuit()
        self._uploaded = False

    def reset_sv(self):
        self._h.reset()

    def reset(self):
        self.clear_circuit()
        self.reset_sv()

    def dump(self) -> str:
        return "\n".join(repr(g) for g in self.circuit) + ("\n" if self.circuit else "")

    # ---- results ----------------------------------------------------------------------
    def state(self) -> np.ndarray:
        re, im = self._h.get_state()
        return re + 1j * im

    @property
    def sv_real_cpu(self) -> np.ndarray:
        return self._h.get_state()[0]

    @property
    def sv_imag_cpu(self) -> np.ndarray:
        return self._h.get_state()[1]

    def measure_with_uniforms(self, uniforms) -> np.ndarray:
        samples, total = self._h.measure(uniforms)
        if abs(total - 1.0) > 1e-3:     # ERROR_BAR, config.hpp:50; message of :379-380
            print(f"Sum of probability is far from 1.0 with {total:f}")
        return samples

    def measure(self, repetition: int = 10) -> list[int]:
        return [int(x) for x in self.measure_with_uniforms(_libc_uniforms(repetition))]

    def plan_info(self):
        return self._h.plan_info()

    def close(self):
        self._h.close()


# the reference's static factories (:397-584) are also reachable from the class
for _name in _g.OP_NAMES:
    setattr(Simulation, _name, staticmethod(_g.FACTORIES[_name]))

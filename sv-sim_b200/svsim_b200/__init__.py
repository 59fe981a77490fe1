"""svsim_b200 — B200-native state-vector engine behind SV-Sim's Simulation/Gate API.

The compute path is libsvsim_b200.so (hand-written sm_100a kernels behind a C ABI,
include/svsim_b200.h); this package is its Python host side: gate records, seeded
workloads, a ``Simulation`` class with the reference's names, and the autograd binding.
"""
from . import circuits, gates  # noqa: F401
from .gates import Gate, OP, OP_NAMES  # noqa: F401


def __getattr__(name):
    # the native pieces load lazily so that gate/circuit utilities import without a GPU
    if name == "Simulation":
        from .simulation import Simulation
        return Simulation
    if name in ("AdjointEnergy", "adjoint_energy"):
        from . import autograd
        return getattr(autograd, name)
    raise AttributeError(name)

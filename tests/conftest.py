import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "sv-sim_b200"))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "native"))

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


def fidelity(a: np.ndarray, b: np.ndarray) -> float:
    """|<a|b>|^2 / (<a|a><b|b>) for complex vectors."""
    num = abs(np.vdot(a, b)) ** 2
    den = np.vdot(a, a).real * np.vdot(b, b).real
    return float(num / den)


def load_golden(name: str):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def cx_dense_circuit(n: int = 12, layers: int = 30, seed: int = 1):
    """Per layer an RY on every qubit, then a CX from every qubit to a partner that moves
    with the layer: many distinct two-qubit blocks per pass, so a pair-engine pass holds
    more gate fragments than fit beside the tile in shared memory."""
    from svsim_b200 import gates as G
    rng = np.random.default_rng(seed)
    gl = []
    for layer in range(layers):
        for i in range(n):
            gl.append(G.RY(float(rng.uniform(0, 2 * np.pi)), i))
        for i in range(n):
            gl.append(G.CX(i, (i + 1 + layer % 5) % n))
    return G.to_array(gl)

"""The reference's own front-end sources, compiled unchanged against the drop-in headers
(sv-sim_b200/svsim_b200/dropin.py), running on the B200 engine."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
from svsim_b200 import gates as G

pytestmark = pytest.mark.gpu

LIB = os.path.join(ROOT, "sv-sim_b200", "svsim_b200", "lib")


def adder_gates():
    """svsim/example/adder_n10_nvgpu_sin.cu: X on 1,5,6,7,8, then the Cuccaro adder."""
    pre = [G.X(1), G.X(5), G.X(6), G.X(7), G.X(8)]
    body = []

    def maj(a, b, c):
        body.extend([G.CX(c, b), G.CX(c, a), G.CCX(a, b, c)])

    def unmaj(a, b, c):
        body.extend([G.CCX(a, b, c), G.CX(c, a), G.CX(a, b)])
    maj(0, 5, 1); maj(1, 6, 2); maj(2, 7, 3); maj(3, 8, 4)
    body.append(G.CX(4, 9))
    unmaj(3, 8, 4); unmaj(2, 7, 3); unmaj(1, 6, 2); unmaj(0, 5, 1)
    return G.to_array(pre + body)


def test_reference_unit_tests_pass():
    exe = os.path.join(LIB, "dropin_unit_test")
    if not os.path.exists(exe):
        pytest.skip("drop-in unit test not built (reference tree absent at build time)")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if "gate test:" in ln]
    assert len(lines) == 14, out.stdout
    assert all(ln.endswith("Success") for ln in lines), out.stdout


def test_reference_adder_example(oracle):
    exe = os.path.join(LIB, "dropin_adder_n10")
    if not os.path.exists(exe):
        pytest.skip("drop-in adder not built")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    re, im = oracle.run(10, adder_gates())
    want = int(np.argmax(re ** 2 + im ** 2))
    shots = [ln.split(":")[1].strip() for ln in out.stdout.splitlines() if ln.startswith("Test-")]
    assert shots and all(int(s, 2) == want for s in shots), out.stdout


def test_reference_python_binding(oracle):
    """Module libsvsim built from svsim/src/py_wrapper.cpp, driven like
    svsim/example/adder_n10.py."""
    if not any(f.startswith("libsvsim.") for f in os.listdir(LIB)):
        pytest.skip("drop-in module not built")
    sys.path.insert(0, LIB)
    import libsvsim as svsim
    sim = svsim.Simulation(10, 0)
    for q in (1, 5, 6, 7, 8):
        sim.append(sim.X(q))
    sim.upload()
    sim.run()
    sim.clear_circuit()
    for g in G.from_array(adder_gates())[5:]:
        f = getattr(sim, g.name)
        sim.append(f(*g.qubits()))
    sim.upload()
    sim.run()
    res = sim.measure(10)
    re, im = oracle.run(10, adder_gates())
    want = int(np.argmax(re ** 2 + im ** 2))
    assert res == [want] * 10

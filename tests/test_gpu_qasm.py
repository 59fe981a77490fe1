"""OpenQASM 2.0 programs through the engines on the GPU, against the oracle."""
import numpy as np
import pytest

from svsim_b200 import circuits, gates as G
from svsim_b200.qasm import loads

pytestmark = pytest.mark.gpu


def program_text(n, depth, seed):
    """A QASM program written out from the random-matching recipe, with a user gate for
    the entangling step and whole-register broadcasts."""
    rng = np.random.default_rng(seed)
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg lo[{n // 2}];", f"qreg hi[{n - n // 2}];",
             "gate ent(t) a, b { cx a, b; rz(t) b; cx a, b; }", "h lo;"]
    regs = [f"lo[{k}]" for k in range(n // 2)] + [f"hi[{k}]" for k in range(n - n // 2)]
    for _ in range(depth):
        for q in regs:
            a = [float(x) for x in rng.uniform(0, 2 * np.pi, size=3)]
            lines.append(f"u3({a[0]!r}, {a[1]!r}, {a[2]!r}) {q};")
        perm = rng.permutation(n)
        for i in range(n // 2):
            lines.append(f"ent({float(rng.uniform(-1, 1))!r}*pi) {regs[perm[2 * i]]}, {regs[perm[2 * i + 1]]};")
    lines.append("measure lo[0] -> c[0];")
    return "\n".join(lines)


@pytest.mark.parametrize("engine", ["staged", "pairs", "per_gate"])
def test_qasm_program_on_engines(oracle, engine):
    from svsim_b200 import _native as nat
    from svsim_b200.simulation import Simulation
    n = 16
    text = program_text(n, 6, seed=3)
    prog = loads(text)
    assert prog.n_qubits == n and prog.measured == [(0, "c", 0)]
    eng = {"staged": nat.ENGINE_STAGED, "pairs": nat.ENGINE_PAIRS, "per_gate": nat.ENGINE_PER_GATE}[engine]
    sim = Simulation.from_qasm(text, engine=eng)
    sim.run()
    st = sim.state()
    ore, oim = oracle.run(n, prog.gates)
    assert np.max(np.abs(st - (ore + 1j * oim))) <= 1e-12
    sim.close()

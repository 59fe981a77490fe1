"""OpenQASM 2.0 front end (svsim_b200.qasm): register layout, broadcasting, gate
definitions, parameter expressions, measure records and errors; the loaded circuits
against hand-built gate lists on the oracle."""
import math

import numpy as np
import pytest

from svsim_b200 import gates as G
from svsim_b200.qasm import QasmError, eval_expr, loads

PROGRAM = """
OPENQASM 2.0;
include "qelib1.inc";
// two registers, concatenated in declaration order
qreg a[2];
qreg b[3];
creg c[3];
gate bell(theta) p, q { h p; cx p, q; rz(theta/2) q; }
gate twice p { x p; x p; }
h a;                          // broadcast over a[0], a[1]
cx a[0], b[1];
u3(pi/2, -pi/4, 2*pi/3) b;    // broadcast over b
bell(pi^2) a[1], b[2];
twice b[0];
barrier a, b;
cu1(sin(pi/6)) b[0], a[0];
ccx a[0], a[1], b[2];
measure b -> c;
"""


def expected():
    gl = [G.H(0), G.H(1), G.CX(0, 3)]
    gl += [G.U3(math.pi / 2, -math.pi / 4, 2 * math.pi / 3, q) for q in (2, 3, 4)]
    gl += [G.H(1), G.CX(1, 4), G.RZ(math.pi ** 2 / 2, 4)]
    gl += [G.X(2), G.X(2)]
    gl += [G.CU1(math.sin(math.pi / 6), 2, 0), G.CCX(0, 1, 4)]
    return G.to_array(gl)


def test_program_structure():
    p = loads(PROGRAM)
    assert p.n_qubits == 5
    assert p.qregs == {"a": (0, 2), "b": (2, 3)}
    assert p.measured == [(2, "c", 0), (3, "c", 1), (4, "c", 2)]
    e = expected()
    assert len(p.gates) == len(e)
    assert np.array_equal(p.gates["op"], e["op"]) and np.array_equal(p.gates["qb"], e["qb"])
    for f in ("theta", "phi", "lam"):
        assert np.allclose(p.gates[f], e[f], rtol=0, atol=1e-15)


def test_loaded_circuit_matches_hand_built_on_oracle(oracle):
    p = loads(PROGRAM)
    re1, im1 = oracle.run(p.n_qubits, p.gates)
    re2, im2 = oracle.run(p.n_qubits, expected())
    assert np.max(np.abs(re1 - re2)) == 0 and np.max(np.abs(im1 - im2)) == 0


def test_every_reference_op_by_qasm_name(oracle):
    names = {"U3": "u3", "U2": "u2", "U1": "u1", "CX": "cx", "ID": "id", "X": "x", "Y": "y", "Z": "z",
             "H": "h", "S": "s", "SDG": "sdg", "T": "t", "TDG": "tdg", "RX": "rx", "RY": "ry",
             "RZ": "rz", "CZ": "cz", "CY": "cy", "SWAP": "swap", "CH": "ch", "CCX": "ccx",
             "CSWAP": "cswap", "CRX": "crx", "CRY": "cry", "CRZ": "crz", "CU1": "cu1", "CU3": "cu3",
             "RXX": "rxx", "RZZ": "rzz", "RCCX": "rccx", "RC3X": "rc3x", "C3X": "c3x",
             "C3SQRTX": "c3sqrtx", "C4X": "c4x", "R": "r", "SRN": "srn", "W": "w", "RYY": "ryy"}
    assert set(names) == set(G.OP_NAMES)
    rng = np.random.default_rng(1)
    lines, gl = ["OPENQASM 2.0;", "qreg q[6];"], []
    for name in G.OP_NAMES:
        nq = G.N_QUBITS[name]
        npar = {"U3": 3, "U2": 2, "CU3": 3}.get(name, 1 if name in (
            "U1", "RX", "RY", "RZ", "CRX", "CRY", "CRZ", "CU1", "RXX", "RZZ", "RYY", "R") else 0)
        qs = [int(x) for x in rng.permutation(6)[:nq]]
        ps = [float(rng.uniform(-3, 3)) for _ in range(npar)]
        par = "(" + ", ".join(repr(x) for x in ps) + ")" if ps else ""
        lines.append(f"{names[name]}{par} " + ", ".join(f"q[{k}]" for k in qs) + ";")
        gl.append(G.FACTORIES[name](*(ps + qs)))
    p = loads("\n".join(lines))
    e = G.to_array(gl)
    assert np.array_equal(p.gates, e)
    re1, im1 = oracle.run(6, p.gates)
    re2, im2 = oracle.run(6, e)
    assert np.array_equal(re1, re2) and np.array_equal(im1, im2)


def test_expressions():
    assert eval_expr("pi/2") == math.pi / 2
    assert eval_expr("-pi + 2*pi") == math.pi
    assert eval_expr("2^3") == 8.0
    assert abs(eval_expr("sqrt(2)*cos(pi/4)") - 1.0) < 1e-15
    assert eval_expr("ln(exp(1.5))") == pytest.approx(1.5)
    with pytest.raises(QasmError):
        eval_expr("__import__('os')")
    with pytest.raises(QasmError):
        eval_expr("theta + 1")


@pytest.mark.parametrize("bad,msg", [
    ("OPENQASM 2.0; qreg q[2]; foo q[0];", "unknown gate"),
    ("OPENQASM 2.0; qreg q[2]; h q[2];", "outside register"),
    ("OPENQASM 2.0; qreg q[2]; cx q[0], q[0];", "repeats a qubit"),
    ("OPENQASM 2.0; qreg q[2]; u3(1, 2) q[0];", "parameters"),
    ("OPENQASM 2.0; qreg q[2]; qreg r[3]; cx q, r;", "different sizes"),
    ("OPENQASM 3.0; qreg q[2];", "OpenQASM 2"),
    ("OPENQASM 2.0; qreg q[2]; h q[0]", "without ';'"),
])
def test_errors_name_the_problem(bad, msg):
    with pytest.raises(QasmError, match=msg):
        loads(bad)


def test_reset_if_opaque_dropped_as_the_reference_translator_does():
    """The reference's translator drops `reset`, `if (...) <gate>` and unknown statements
    whole (svsim_qasm_cplus.py:104, :325-326); the loader does the same by default and
    records them, and rejects them with strict=True."""
    src = ("OPENQASM 2.0;\ninclude \"qelib1.inc\";\nqreg q[2];\ncreg c[2];\nh q[0];\nreset q[1];\n"
           "measure q[0] -> c[0];\nif(c==1) x q[1];\nif (c == 0) cx q[0], q[1];\ncx q[0], q[1];\n")
    prog = loads(src)
    assert [int(g["op"]) for g in prog.gates] == [G.OP["H"], G.OP["CX"]]
    assert [ln for ln, _ in prog.skipped] == [6, 8, 9]
    assert prog.skipped[1][1].replace(" ", "") == "if(c==1)xq[1]"
    for bad in ("OPENQASM 2.0; qreg q[2]; reset q[0];", "OPENQASM 2.0; qreg q[1]; creg c[1]; if(c==1) x q[0];"):
        with pytest.raises(QasmError, match="not supported"):
            loads(bad, strict=True)

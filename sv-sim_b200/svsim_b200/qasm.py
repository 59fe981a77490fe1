"""OpenQASM 2.0 front end: program text in, the engine's gate records out.

The reference turns a QASM file into C++ with ``svsim/tool/svsim_qasm_cplus.py`` (a
Python 2 script, :233-336) and compiles that.  This loader reads the same language
subset and yields gate records directly, so a QASM program runs on any engine without a
compile step:

* ``qreg`` declarations are concatenated into one qubit index space in declaration
  order (the translator's global array, :109-134);
* the qelib1 gates the translator knows (its STANDARD and COMPOSITION tables: u3 u2 u1
  cx id x y z h s sdg t tdg rx ry rz cz cy swap ch ccx cswap crx cry crz cu1 cu3 rxx rzz
  rccx rc3x c3x c3sqrtx c4x), plus the reference ops it has no QASM name for (r, srn, w,
  ryy) and QASM's own ``U`` and ``CX``, map to the reference factories with their
  argument order;
* an argument naming a whole register applies the gate once per index (registers used
  together must have equal sizes), as the translator's paramlist expansion does
  (:137-170);
* ``gate`` definitions are expanded at each call with the call's parameters and qubits;
* parameters are arithmetic expressions over numbers, ``pi`` and sin/cos/tan/exp/ln/
  sqrt, evaluated with a restricted evaluator (no Python ``eval``);
* ``measure`` records (qubit, classical bit) pairs; ``barrier``, ``creg``, ``include``
  and the ``OPENQASM`` header carry no gate;
* ``reset``, an ``if (...)`` statement with the gate it conditions, and ``opaque`` have no
  counterpart in the reference's state-vector circuits: its translator drops those
  statements whole (its ``other_keys`` list, :104, skipped at :325-326), and so does this
  loader by default, recording each one in ``QasmProgram.skipped``.  With
  ``strict=True`` they are rejected instead, with an error naming the line.
"""
from __future__ import annotations

import ast
import math
import operator
import re
from dataclasses import dataclass, field

import numpy as np

from . import gates as G

# QASM name -> (reference op name, number of parameters)
_BUILTIN = {
    "u3": ("U3", 3), "u2": ("U2", 2), "u1": ("U1", 1), "cx": ("CX", 0), "id": ("ID", 0),
    "x": ("X", 0), "y": ("Y", 0), "z": ("Z", 0), "h": ("H", 0), "s": ("S", 0), "sdg": ("SDG", 0),
    "t": ("T", 0), "tdg": ("TDG", 0), "rx": ("RX", 1), "ry": ("RY", 1), "rz": ("RZ", 1),
    "cz": ("CZ", 0), "cy": ("CY", 0), "swap": ("SWAP", 0), "ch": ("CH", 0), "ccx": ("CCX", 0),
    "cswap": ("CSWAP", 0), "crx": ("CRX", 1), "cry": ("CRY", 1), "crz": ("CRZ", 1),
    "cu1": ("CU1", 1), "cu3": ("CU3", 3), "rxx": ("RXX", 1), "rzz": ("RZZ", 1),
    "rccx": ("RCCX", 0), "rc3x": ("RC3X", 0), "c3x": ("C3X", 0), "c3sqrtx": ("C3SQRTX", 0),
    "c4x": ("C4X", 0), "r": ("R", 1), "srn": ("SRN", 0), "w": ("W", 0), "ryy": ("RYY", 1),
    "U": ("U3", 3), "CX": ("CX", 0),
}


class QasmError(ValueError):
    pass


# ---- parameter expressions -----------------------------------------------------------
_BINOPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul,
           ast.Div: operator.truediv, ast.Pow: operator.pow}
_FUNCS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp, "ln": math.log,
          "sqrt": math.sqrt}


def eval_expr(text: str, env: dict[str, float] | None = None) -> float:
    """Value of a QASM parameter expression (``^`` is the power operator)."""
    env = env or {}
    try:
        tree = ast.parse(text.replace("^", "**").strip(), mode="eval")
    except SyntaxError as e:
        raise QasmError(f"bad expression {text!r}") from e

    def ev(node):
        if isinstance(node, ast.Expression):
            return ev(node.body)
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
            return float(node.value)
        if isinstance(node, ast.Name):
            if node.id == "pi":
                return math.pi
            if node.id in env:
                return float(env[node.id])
            raise QasmError(f"unknown name {node.id!r} in {text!r}")
        if isinstance(node, ast.BinOp) and type(node.op) in _BINOPS:
            return _BINOPS[type(node.op)](ev(node.left), ev(node.right))
        if isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.USub, ast.UAdd)):
            v = ev(node.operand)
            return -v if isinstance(node.op, ast.USub) else v
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id in _FUNCS
                and len(node.args) == 1 and not node.keywords):
            return _FUNCS[node.func.id](ev(node.args[0]))
        raise QasmError(f"unsupported expression {text!r}")

    return ev(tree)


def _split_top(text: str, sep: str = ",") -> list[str]:
    """Splits on `sep` outside parentheses."""
    out, depth, cur = [], 0, []
    for ch in text:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return [s.strip() for s in out if s.strip()]


# ---- program --------------------------------------------------------------------------
@dataclass
class GateDef:
    params: list[str]
    qargs: list[str]
    body: list[str]


@dataclass
class QasmProgram:
    n_qubits: int
    gates: np.ndarray                                   # GATE_DTYPE records
    qregs: dict[str, tuple[int, int]] = field(default_factory=dict)   # name -> (offset, size)
    measured: list[tuple[int, str, int]] = field(default_factory=list)  # (qubit, creg, bit)
    skipped: list[tuple[int, str]] = field(default_factory=list)        # (line, statement)


_CALL = re.compile(r"^([A-Za-z_][A-Za-z0-9_]*)\s*(\((.*)\))?\s*(.*)$", re.S)


def _statements(text: str) -> list[tuple[int, str]]:
    """(line, statement) pairs; comments removed, gate bodies kept as one statement."""
    lines = text.splitlines()
    clean = []
    for i, ln in enumerate(lines, 1):
        if "//" in ln:
            ln = ln[: ln.index("//")]
        clean.append((i, ln))
    out, cur, start, depth = [], [], None, 0
    for i, ln in clean:
        for ch in ln:
            if start is None and not ch.isspace():
                start = i
            cur.append(ch)
            if ch == "{":
                depth += 1
            elif ch == "}":
                depth -= 1
                if depth == 0:
                    out.append((start, "".join(cur).strip()))
                    cur, start = [], None
            elif ch == ";" and depth == 0:
                out.append((start, "".join(cur).strip()[:-1].strip()))
                cur, start = [], None
        cur.append(" ")
    if "".join(cur).strip():
        raise QasmError(f"line {start}: statement without ';'")
    return out


def loads(text: str, strict: bool = False) -> QasmProgram:
    """Parses an OpenQASM 2.0 program.  ``reset``, ``if`` and ``opaque`` statements are
    dropped as the reference's translator drops them (``strict=False``) or rejected."""
    qregs: dict[str, tuple[int, int]] = {}
    skipped: list[tuple[int, str]] = []
    gate_defs: dict[str, GateDef] = {}
    rows: list = []
    measured: list[tuple[int, str, int]] = []
    n_qubits = 0

    def qubits_of(arg: str, line: int) -> list[int]:
        m = re.fullmatch(r"([A-Za-z_][A-Za-z0-9_]*)\s*(\[\s*(\d+)\s*\])?", arg.strip())
        if not m or m.group(1) not in qregs:
            raise QasmError(f"line {line}: unknown qubit argument {arg!r}")
        off, size = qregs[m.group(1)]
        if m.group(2) is None:
            return [off + k for k in range(size)]
        k = int(m.group(3))
        if k >= size:
            raise QasmError(f"line {line}: index {k} outside register {m.group(1)}[{size}]")
        return [off + k]

    def emit(name: str, params: list[float], qs: list[int], line: int):
        opname, npar = _BUILTIN[name]
        if len(params) != npar:
            raise QasmError(f"line {line}: {name} takes {npar} parameters, got {len(params)}")
        if len(qs) != G.N_QUBITS[opname]:
            raise QasmError(f"line {line}: {name} acts on {G.N_QUBITS[opname]} qubits, got {len(qs)}")
        if len(set(qs)) != len(qs):
            raise QasmError(f"line {line}: {name} repeats a qubit")
        g = G.FACTORIES[opname](*(params + qs))
        rows.append((g.op, g.qb, g.theta, g.phi, g.lam))

    def call(name: str, params: list[float], qs: list[int], line: int, depth: int = 0):
        if depth > 64:
            raise QasmError(f"line {line}: gate definitions nest too deeply")
        if name in gate_defs:
            d = gate_defs[name]
            if len(params) != len(d.params) or len(qs) != len(d.qargs):
                raise QasmError(f"line {line}: {name} takes {len(d.params)} parameters and "
                                f"{len(d.qargs)} qubits")
            env = dict(zip(d.params, params))
            qmap = dict(zip(d.qargs, qs))
            for st in d.body:
                m = _CALL.match(st)
                if not m:
                    raise QasmError(f"line {line}: bad statement {st!r} in gate {name}")
                sub = m.group(1)
                if sub == "barrier":
                    continue
                ps = [eval_expr(e, env) for e in _split_top(m.group(3))] if m.group(2) else []
                args = _split_top(m.group(4))
                try:
                    sq = [qmap[a] for a in args]
                except KeyError as e:
                    raise QasmError(f"line {line}: gate {name} uses undeclared argument {e}") from None
                call(sub, ps, sq, line, depth + 1)
        elif name in _BUILTIN:
            emit(name, params, qs, line)
        else:
            raise QasmError(f"line {line}: unknown gate {name!r}")

    for line, st in _statements(text):
        if not st:
            continue
        head = st.split(None, 1)[0]
        if head == "OPENQASM":
            if not st.split(None, 1)[1].strip().startswith("2"):
                raise QasmError(f"line {line}: only OpenQASM 2 is supported")
            continue
        if head in ("include", "creg", "barrier"):
            continue
        word = re.match(r"[A-Za-z_][A-Za-z0-9_]*", head)
        if word and word.group(0) in ("reset", "if", "opaque"):
            if strict:
                raise QasmError(f"line {line}: {word.group(0)!r} is not supported")
            skipped.append((line, st))
            continue
        if head == "qreg":
            m = re.fullmatch(r"qreg\s+([A-Za-z_][A-Za-z0-9_]*)\s*\[\s*(\d+)\s*\]", st)
            if not m:
                raise QasmError(f"line {line}: bad qreg {st!r}")
            if m.group(1) in qregs:
                raise QasmError(f"line {line}: register {m.group(1)} declared twice")
            qregs[m.group(1)] = (n_qubits, int(m.group(2)))
            n_qubits += int(m.group(2))
            continue
        if head == "gate":
            m = re.fullmatch(r"gate\s+([A-Za-z_][A-Za-z0-9_]*)\s*(\(([^)]*)\))?\s*([^{]*)\{(.*)\}", st, re.S)
            if not m:
                raise QasmError(f"line {line}: bad gate definition")
            params = _split_top(m.group(3) or "")
            qargs = _split_top(m.group(4))
            body = [b.strip() for b in m.group(5).split(";") if b.strip()]
            gate_defs[m.group(1)] = GateDef(params, qargs, body)
            continue
        if head == "measure":
            m = re.fullmatch(r"measure\s+(.+?)\s*->\s*(.+)", st)
            if not m:
                raise QasmError(f"line {line}: bad measure {st!r}")
            qs = qubits_of(m.group(1), line)
            cm = re.fullmatch(r"([A-Za-z_][A-Za-z0-9_]*)\s*(\[\s*(\d+)\s*\])?", m.group(2).strip())
            if not cm:
                raise QasmError(f"line {line}: bad classical target {m.group(2)!r}")
            bits = [int(cm.group(3))] if cm.group(2) else list(range(len(qs)))
            if len(bits) != len(qs):
                raise QasmError(f"line {line}: measure sizes differ")
            measured += [(q, cm.group(1), b) for q, b in zip(qs, bits)]
            continue
        m = _CALL.match(st)
        if not m:
            raise QasmError(f"line {line}: cannot parse {st!r}")
        name = m.group(1)
        params = [eval_expr(e) for e in _split_top(m.group(3))] if m.group(2) else []
        args = [qubits_of(a, line) for a in _split_top(m.group(4))]
        if not args:
            raise QasmError(f"line {line}: {name} without qubits")
        width = max(len(a) for a in args)
        for a in args:
            if len(a) not in (1, width):
                raise QasmError(f"line {line}: registers of different sizes in one call")
        for k in range(width):
            call(name, params, [a[k] if len(a) > 1 else a[0] for a in args], line)

    arr = np.zeros(len(rows), dtype=G.GATE_DTYPE)
    for i, r in enumerate(rows):
        arr[i] = r
    return QasmProgram(n_qubits, arr, qregs, measured, skipped)


def load(path: str, strict: bool = False) -> QasmProgram:
    with open(path, encoding="utf-8") as f:
        return loads(f.read(), strict=strict)

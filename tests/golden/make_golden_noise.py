"""Generates tests/golden/noise.npz from the reference's density-matrix noise variant
(svsim_qsharp_noise/), read as text:

  * the superoperator tables of its noisy gates, noise_gate_{AD,DP,BCSZ}_{0.98,0.99}.cuh:
    for each of X, Y, Z and H the 16 complex entries e_rc (XR0..XR15, XI0..XI15, ...)
    that C2_GATE (svsim_nvgpu_sin.cuh:1727-1800) applies to the amplitudes
    (pos0, pos1, pos2, pos3) of the pair (qubit, qubit + n_qubits) as
    out[r] = sum_c e_rc in[c];
  * the known answers of its unit tests (unit_test_nvgpu_sin.cu:41-727): for each test
    the qubit count (AllocateQubit calls), the operations in order (name and numeric
    arguments, PI and the control masks evaluated) and the expected density matrix
    (sv_real_expected / sv_imag_expected, a C initialiser that may be shorter than
    2^(2n) and is then zero-padded), compared by the reference to ERROR_BAR = 1e-3.

Run in a container that has the reference tree:  python tests/golden/make_golden_noise.py
"""
from __future__ import annotations

import math
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import REFERENCE  # noqa: E402

SRC = os.path.join(REFERENCE, "svsim_qsharp_noise")
TABLES = ["DP_0.99", "DP_0.98", "AD_0.99", "AD_0.98", "BCSZ_0.99", "BCSZ_0.98"]
GATES = "XYZH"


def parse_table(path):
    d = {}
    for m in re.finditer(r"#define\s+([A-Z]+)(\d+)\s+(\S+)", open(path).read()):
        d[(m.group(1), int(m.group(2)))] = float(m.group(3))
    return np.array([[d[(g + "R", k)] + 1j * d[(g + "I", k)] for k in range(16)] for g in GATES])


def evaluate(arg: str) -> float:
    a = arg.strip().replace("((IdxType)1<<", "(1<<").replace("PI", repr(math.pi))
    if not re.fullmatch(r"[0-9eE+\-*/.() <]*", a):
        raise ValueError(f"unexpected argument {arg!r}")
    return float(eval(a))            # digits, PI, arithmetic and shifts only (checked above)


def parse_initialiser(text, dim):
    vals = [float(v) for v in text.split(",") if v.strip()]
    return np.array(vals + [0.0] * (dim - len(vals)))


def parse_kats(path):
    src = open(path).read()
    kats = []
    for m in re.finditer(r"bool (test_\w+)\(\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        n = body.count("AllocateQubit()")
        dim = 1 << (2 * n)
        ops = []
        for call in re.finditer(r"sim\.(\w+)\(([^;]*)\);", body):
            op, args = call.group(1), call.group(2)
            if op in ("AllocateQubit", "sim", "print_res_sv"):
                continue
            parts = [p for p in re.split(r",(?![^(]*\))", args) if p.strip()]
            ops.append((op, [evaluate(p) for p in parts]))
        re_m = re.search(r"sv_real_expected\[dim\]\s*=\s*\{([^}]*)\}", body)
        im_m = re.search(r"sv_imag_expected\[dim\]\s*=\s*\{([^}]*)\}", body)
        kats.append((name, n, ops, parse_initialiser(re_m.group(1), dim), parse_initialiser(im_m.group(1), dim)))
    return kats


def main():
    tables = np.stack([parse_table(os.path.join(SRC, f"noise_gate_{t}.cuh")) for t in TABLES])
    kats = parse_kats(os.path.join(SRC, "unit_test_nvgpu_sin.cu"))
    op_names, op_args, op_kat = [], [], []
    for k, (_, _, ops, _, _) in enumerate(kats):
        for op, args in ops:
            op_names.append(op)
            op_args.append(args + [np.nan] * (3 - len(args)))
            op_kat.append(k)
    out = os.path.join(HERE, "noise.npz")
    np.savez_compressed(
        out, table_names=np.array(TABLES), table_gates=np.array(list(GATES)), tables=tables,
        kat_names=np.array([k[0] for k in kats]), kat_n=np.array([k[1] for k in kats]),
        kat_re=np.concatenate([k[3] for k in kats]), kat_im=np.concatenate([k[4] for k in kats]),
        op_names=np.array(op_names), op_args=np.array(op_args), op_kat=np.array(op_kat),
        error_bar=np.array([1e-3]))
    print(out, os.path.getsize(out), len(kats), "tests,", len(op_names), "operations")


if __name__ == "__main__":
    main()

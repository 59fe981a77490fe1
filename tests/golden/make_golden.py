"""Generates the golden fixtures in tests/golden/ from the REFERENCE ITSELF.

Every expected value here is produced by the reference's own CPU backend
(svsim/src/svsim_cpu_sin.hpp, compiled in place by oracle/Makefile into oracle/_ref/
and driven through its public Simulation API by oracle/ref_glue.cpp), except the
``kat_expected`` table, which holds the 3-decimal known answers of the reference's
unit tests (svsim/unit_test/unit_test_cpu_sin.cpp:41-301).

Run in a container that has the reference tree:  python tests/golden/make_golden.py
The fixtures are small (a few hundred KiB) and committed; tests never need the
reference tree at run time.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "sv-sim_b200"))
sys.path.insert(0, ROOT)

from svsim_b200 import circuits, gates as G  # noqa: E402
from oracle.oracle import RefBackend, libc_uniforms, build  # noqa: E402

PI = 3.14159265358979323846


def checksum_weights(n: int) -> np.ndarray:
    """Fixed complex weights w_i = cos(0.7 i) + i sin(1.3 i) for a weighted checksum."""
    i = np.arange(1 << n, dtype=np.float64)
    return np.cos(0.7 * i) + 1j * np.sin(1.3 * i)


def kat_cases():
    """(name, n, gates, expected_re, expected_im) — unit_test_cpu_sin.cpp:41-301."""
    s = 0.707
    return [
        ("X", 1, [G.X(0)], [0, 1], [0, 0]),
        ("Y", 1, [G.Y(0)], [0, 0], [0, 1]),
        ("Z", 1, [G.H(0), G.Z(0)], [s, -s], [0, 0]),
        ("H", 1, [G.H(0)], [s, s], [0, 0]),
        ("S", 1, [G.H(0), G.S(0)], [s, 0], [0, s]),
        ("SDG", 1, [G.H(0), G.SDG(0)], [s, 0], [0, -s]),
        ("T", 1, [G.H(0), G.T(0)], [s, 0.5], [0, 0.5]),
        ("TDG", 1, [G.H(0), G.TDG(0)], [s, 0.5], [0, -0.5]),
        ("RX", 1, [G.RX(PI / 3.0, 0)], [0.866, 0], [0, -0.5]),
        ("RY", 1, [G.RY(PI / 6.0, 0)], [0.966, 0.259], [0, 0]),
        ("U1", 1, [G.H(0), G.U1(PI / 5.0, 0)], [s, 0.572], [0, 0.416]),
        ("U2", 1, [G.H(0), G.U2(PI / 4.0, PI / 5.0, 0)], [0.095, 0.432], [-0.294, 0.847]),
        ("U3", 1, [G.H(0), G.U3(PI / 4.0, PI / 5.0, PI / 6.0, 0)], [0.419, 0.485], [-0.135, 0.756]),
        ("CX", 2, [G.H(0), G.CX(0, 1)], [s, 0, 0, s], [0, 0, 0, 0]),
    ]


def n_params(name):
    if name in ("U3", "CU3"):
        return 3
    if name == "U2":
        return 2
    if name in ("U1", "RX", "RY", "RZ", "CRX", "CRY", "CRZ", "CU1", "RXX", "RZZ", "RYY", "R"):
        return 1
    return 0


def all_ops_cases(n=6, reps=3, seed=11):
    """Every op of the reference, `reps` random placements each, after a prep layer."""
    rng = np.random.default_rng(seed)
    prep = circuits.random_matching_circuit(n, 2, seed=seed)
    out = []
    for name in G.OP_NAMES:
        for r in range(reps):
            qs = [int(x) for x in rng.permutation(n)[:G.N_QUBITS[name]]]
            par = [float(x) for x in rng.uniform(-math.pi, math.pi, n_params(name))]
            g = G.FACTORIES[name](*(par + qs))
            out.append((name, np.concatenate([prep, G.to_array([g])])))
    return out


def main():
    build(reference=True)
    ref = RefBackend("sin")
    data = {}

    # 1. the reference's unit-test known answers, plus its full-precision states
    kats = kat_cases()
    kat_gates, kat_off, kat_n, kat_exp_re, kat_exp_im, kat_ref_re, kat_ref_im = [], [0], [], [], [], [], []
    for name, n, gl, er, ei in kats:
        arr = G.to_array(gl)
        r = ref.simulate(n, arr)
        kat_gates.append(arr)
        kat_off.append(kat_off[-1] + len(arr))
        kat_n.append(n)
        kat_exp_re += er
        kat_exp_im += ei
        kat_ref_re += list(r["re"])
        kat_ref_im += list(r["im"])
    np.savez(os.path.join(HERE, "kat.npz"),
             names=np.array([k[0] for k in kats]), n=np.array(kat_n), gates=np.concatenate(kat_gates),
             gate_offsets=np.array(kat_off), expected_re=np.array(kat_exp_re),
             expected_im=np.array(kat_exp_im), ref_re=np.array(kat_ref_re),
             ref_im=np.array(kat_ref_im))

    # 2. every op, full states from the reference
    cases = all_ops_cases()
    gl, offs, names, sre, sim = [], [0], [], [], []
    for name, arr in cases:
        r = ref.simulate(6, arr)
        gl.append(arr)
        offs.append(offs[-1] + len(arr))
        names.append(name)
        sre.append(r["re"])
        sim.append(r["im"])
    np.savez(os.path.join(HERE, "all_ops_n6.npz"), names=np.array(names), gates=np.concatenate(gl),
             gate_offsets=np.array(offs), re=np.array(sre), im=np.array(sim))

    # 3. the brickwork recipe at n = 12 (full state) and n = 16 (the 470-gate circuit:
    #    sampled amplitudes, weighted checksums and the reference's own 1024 samples
    #    from measure() with rand() seeded by SAMPLE_SEED)
    g12 = circuits.brickwork_circuit(12, 20, seed=1234)
    r12 = ref.simulate(12, g12)
    SAMPLE_SEED = 4242
    g16 = circuits.brickwork_circuit(16, 20, seed=1234)
    r16 = ref.simulate(16, g16, shots=1024, seed=SAMPLE_SEED)
    rng = np.random.default_rng(77)
    idx = np.sort(rng.choice(1 << 16, size=4096, replace=False))
    w = checksum_weights(16)
    amp16 = r16["re"] + 1j * r16["im"]
    np.savez(os.path.join(HERE, "brickwork.npz"),
             gates12=g12, re12=r12["re"], im12=r12["im"],
             gates16=g16, idx16=idx, re16_at=r16["re"][idx], im16_at=r16["im"][idx],
             checksum16=np.array([np.sum(amp16 * w)]),
             norm16=np.array([np.sum(np.abs(amp16) ** 2)]),
             samples16=r16["samples"], sample_seed=np.array([SAMPLE_SEED]),
             uniforms16=libc_uniforms(SAMPLE_SEED, 1024))

    # 4. the random-matching recipe at n = 12 (full state)
    gm = circuits.random_matching_circuit(12, 10, seed=2024)
    rm = ref.simulate(12, gm)
    np.savez(os.path.join(HERE, "matching_n12.npz"), gates=gm, re=rm["re"], im=rm["im"])
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()

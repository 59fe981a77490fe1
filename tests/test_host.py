"""Seeded workloads and gate records (host only)."""
import math

import numpy as np

from svsim_b200 import circuits, gates as G


def test_gate_record_layout():
    assert G.GATE_DTYPE.itemsize == 48
    assert G.GATE_DTYPE.fields["theta"][1] == 24
    assert G.PARAM_DTYPE.itemsize == 40
    assert G.PAULI_DTYPE.itemsize == 24
    assert len(G.OP_NAMES) == 38 and G.OP["RYY"] == 37 and G.OP["U3"] == 0


def test_factory_argument_order():
    g = G.U3(0.1, 0.2, 0.3, 4)
    assert (g.op, g.qb[0], g.theta, g.phi, g.lam) == (0, 4, 0.1, 0.2, 0.3)
    g = G.RZ(0.5, 2)
    assert g.phi == 0.5 and g.theta == 0 and g.lam == 0     # RZ reads phi (:474)
    g = G.CRZ(0.5, 1, 2)
    assert g.lam == 0.5 and g.qb[:2] == (1, 2)              # CRZ reads lambda (:507)
    g = G.CU3(0.1, 0.2, 0.3, 5, 6)
    assert g.qb[:2] == (5, 6) and (g.theta, g.phi, g.lam) == (0.1, 0.2, 0.3)
    assert repr(G.CX(0, 1)) == "CX(0,1,0,0,0,0,0,0);"


def test_brickwork_recipe():
    g = circuits.brickwork_circuit(16, 20, seed=1234)
    assert len(g) == 470
    assert (g["op"] == G.OP["U3"]).sum() == 320 and (g["op"] == G.OP["CX"]).sum() == 150
    u3 = g[g["op"] == G.OP["U3"]]
    assert u3["theta"].min() >= 0 and u3["theta"].max() < 2 * math.pi


def test_random_matching_recipe():
    g = circuits.random_matching_circuit(30, 40)
    assert len(g) == 1800
    cx = g[g["op"] == G.OP["CX"]]
    assert len(cx) == 600
    for layer in range(40):
        pairs = cx[layer * 15:(layer + 1) * 15]["qb"][:, :2]
        assert len(set(pairs.ravel().tolist())) == 30      # a perfect matching


def test_ansatz_and_hamiltonian():
    pc = circuits.hardware_efficient_ansatz()
    assert len(pc.gates) == 720 and len(pc.params) == 480
    assert np.all(np.abs(pc.params) <= math.pi)
    assert np.array_equal(pc.evaluated(pc.params), pc.gates)
    h = circuits.zz_x_hamiltonian(20)
    assert len(h) == 40 and h["coef"].sum() == 20 + 0.5 * 20


def test_qaoa_instances():
    inst = circuits.qaoa_instances(count=64)
    ns = [i.n for i in inst]
    assert min(ns) >= 10 and max(ns) <= 22
    i0 = inst[0]
    assert np.all((i0.weights >= 0.5) & (i0.weights <= 1.5))
    assert len(i0.gammas) == 4 and np.all(i0.betas <= math.pi / 2)
    assert len(i0.circuit()) == i0.n + 4 * (len(i0.edges) + i0.n)

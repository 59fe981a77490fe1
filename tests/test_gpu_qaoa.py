"""Batched QAOA (svb_qaoa_*): energies against the oracle's state, gradients against
central finite differences (of the oracle and of the batch itself) and against the
general adjoint engine (svb_adjoint) on the same circuit, FP32 against FP64."""
import numpy as np
import pytest

from svsim_b200 import circuits

pytestmark = pytest.mark.gpu


def oracle_energy(oracle, inst, gammas=None, betas=None):
    if gammas is not None:
        inst = circuits.QaoaInstance(inst.n, inst.edges, inst.weights, gammas, betas)
    re, im = oracle.run(inst.n, inst.circuit())
    return float(np.dot(inst.cost_table(), re * re + im * im))


def params_of(instances):
    g = np.stack([i.gammas for i in instances])
    b = np.stack([i.betas for i in instances])
    return g, b


@pytest.fixture(scope="module")
def mixed():
    """Instances on both sides of the 12-qubit FP64 tile: one-tile (n <= 12), high pass
    with wide (n = 13..16) and narrow (n = 20..24) contiguous runs."""
    out = []
    for k, n in enumerate([2, 3, 5, 8, 11, 12, 13, 14, 16, 12, 9, 20, 22, 23, 24]):
        out += circuits.qaoa_instances(count=1, n_min=n, n_max=n, seed=100 + k)
    return out


def test_energies_match_oracle_fp64(oracle, mixed):
    from svsim_b200 import _native as nat
    b = nat.QaoaBatch(mixed, 0, nat.SVB_FP64)
    e, _ = b.run(*params_of(mixed))
    for inst, ei in zip(mixed, e):
        if inst.n > 20:
            continue                      # checked against svb_adjoint below
        ref = oracle_energy(oracle, inst)
        assert abs(ei - ref) <= 1e-12 * max(1.0, abs(ref)), (inst.n, ei, ref)


def test_gradients_match_oracle_finite_differences(oracle):
    from svsim_b200 import _native as nat
    insts = [circuits.qaoa_instances(count=1, n_min=n, n_max=n, seed=7 + n)[0] for n in (4, 7, 13)]
    b = nat.QaoaBatch(insts, 0, nat.SVB_FP64)
    _, grad = b.run(*params_of(insts))
    h = 1e-5
    for inst, gi in zip(insts, grad):
        p = len(inst.gammas)
        fd = np.zeros(2 * p)
        for k in range(2 * p):
            g0, b0 = inst.gammas.copy(), inst.betas.copy()
            vec = np.concatenate([g0, b0])
            vp, vm = vec.copy(), vec.copy()
            vp[k] += h
            vm[k] -= h
            ep = oracle_energy(oracle, inst, vp[:p], vp[p:])
            em = oracle_energy(oracle, inst, vm[:p], vm[p:])
            fd[k] = (ep - em) / (2 * h)
        assert np.max(np.abs(gi - fd)) <= 1e-7 * max(1.0, np.max(np.abs(fd))), (inst.n, gi, fd)


def test_matches_general_adjoint_engine(mixed):
    """Energy and all 2p derivatives agree with svb_adjoint running the reference gate
    list (H, RZZ = CX.U1.CX, RX) with C as a Pauli sum, on the large instances."""
    from svsim_b200 import _native as nat
    b = nat.QaoaBatch(mixed, 0, nat.SVB_FP64)
    e, grad = b.run(*params_of(mixed))
    for inst, ei, gi in zip(mixed, e, grad):
        if inst.n < 13:
            continue
        pc = inst.param_circuit()
        h = nat.Handle(inst.n, 0, nat.SVB_FP64)
        ea, ga = h.adjoint(pc.gates, pc.binding, len(pc.params), inst.maxcut_terms())
        h.close()
        assert abs(ei - ea) <= 1e-11 * max(1.0, abs(ea)), (inst.n, ei, ea)
        assert np.max(np.abs(gi - ga)) <= 1e-10 * max(1.0, np.max(np.abs(ga))), (inst.n, gi, ga)


def test_fp32_batch_tracks_fp64(mixed):
    from svsim_b200 import _native as nat
    g, bt = params_of(mixed)
    e64, g64 = nat.QaoaBatch(mixed, 0, nat.SVB_FP64).run(g, bt)
    e32, g32 = nat.QaoaBatch(mixed, 0, nat.SVB_FP32).run(g, bt)
    scale = np.maximum(1.0, np.abs(e64))
    assert np.max(np.abs(e32 - e64) / scale) <= 1e-4
    assert np.max(np.abs(g32 - g64)) <= 1e-3 * max(1.0, np.max(np.abs(g64)))


def test_repeated_runs_are_bitwise_identical_and_params_update(mixed):
    from svsim_b200 import _native as nat
    b = nat.QaoaBatch(mixed, 0, nat.SVB_FP64)
    g, bt = params_of(mixed)
    e1, g1 = b.run(g, bt)
    e2, g2 = b.run(g + 0.1, bt)
    e3, g3 = b.run(g, bt)
    assert np.array_equal(e1, e3) and np.array_equal(g1, g3)
    assert not np.array_equal(e1, e2)
    assert b.info().graphed == 1


def test_headline_batch_512_instances():
    """512 instances, n in [10, 22], p = 4: energies and gradients of every instance
    against central differences of the batch itself (all instances shifted at once),
    energies against the general engine on a sample, FP32 against FP64."""
    from svsim_b200 import _native as nat
    insts = circuits.qaoa_instances(512)
    g, bt = params_of(insts)
    b = nat.QaoaBatch(insts, 0, nat.SVB_FP64)
    st = b.info()
    assert st.n_instances == 512 and st.p == 4
    e, grad = b.run(g, bt)
    assert np.all(e >= 0) and np.all(np.isfinite(grad))
    h = 1e-5
    p = 4
    fd = np.zeros_like(grad)
    for k in range(2 * p):
        gp, bp, gm, bm = g.copy(), bt.copy(), g.copy(), bt.copy()
        if k < p:
            gp[:, k] += h
            gm[:, k] -= h
        else:
            bp[:, k - p] += h
            bm[:, k - p] -= h
        fd[:, k] = (b.run(gp, bp)[0] - b.run(gm, bm)[0]) / (2 * h)
    err = np.max(np.abs(grad - fd), axis=1) / np.maximum(1.0, np.max(np.abs(fd), axis=1))
    assert np.max(err) <= 1e-6, float(np.max(err))
    for i in range(0, 512, 64):
        inst = insts[i]
        hd = nat.Handle(inst.n, 0, nat.SVB_FP64)
        hd.set_circuit(inst.circuit())
        hd.run()
        ref = hd.expectation(inst.maxcut_terms())
        hd.close()
        assert abs(e[i] - ref) <= 1e-11 * max(1.0, abs(ref)), (i, e[i], ref)
    b.close()
    e32, g32 = nat.QaoaBatch(insts, 0, nat.SVB_FP32).run(g, bt)
    assert np.max(np.abs(e32 - e) / np.maximum(1.0, np.abs(e))) <= 1e-4


def test_sharded_wrapper_single_process_equals_batch():
    """ShardedQaoa without torch.distributed is the plain batch on one GPU."""
    from svsim_b200 import _native as nat
    from svsim_b200.sharding import ShardedQaoa
    insts = circuits.qaoa_instances(24, n_min=6, n_max=16, seed=4)
    g, bt = params_of(insts)
    e0, g0 = nat.QaoaBatch(insts, 0, nat.SVB_FP64).run(g, bt)
    sq = ShardedQaoa(insts, device=0, precision=nat.SVB_FP64)
    e1, g1 = sq.run(g, bt)
    sq.close()
    assert np.array_equal(e0, e1) and np.array_equal(g0, g1)

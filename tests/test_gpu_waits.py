"""Failure detection on the GPU without a GPU fault: the bounded waits the persistent
kernels rely on (the fused engines' tensor-core completion wait on an mbarrier, the
batched engines' grid barrier) are made to run out on purpose — an mbarrier nothing
arrives at, a grid barrier whose count is never reached.  Each must give up within its
limit and report it, and the context must stay usable afterwards."""
import time

import numpy as np
import pytest

from conftest import fidelity
from svsim_b200 import circuits

pytestmark = pytest.mark.gpu


def test_bounded_waits_give_up_and_report(oracle):
    from svsim_b200 import _native as nat
    t0 = time.time()
    mbar, grid = nat.selftest_waits(0)
    dt = time.time() - t0
    assert mbar and grid
    assert dt < 30.0                     # 2 s + a little over 1 s, with margin
    # the context still runs circuits, on the fused engine too
    n = 13
    g = circuits.random_matching_circuit(n, 4, seed=8)
    ore, oim = oracle.run(n, g)
    h = nat.Handle(n, 0, nat.SVB_FP32)
    h.set_engine(nat.ENGINE_FUSED, 0, 5)
    h.set_circuit(g)
    h.run()
    h.sync()
    re, im = h.get_state()
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) <= 1e-6

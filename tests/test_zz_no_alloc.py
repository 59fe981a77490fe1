"""svb_measure_noalloc: the measurement entry point that allocates nothing.

It is for callers that cannot allocate device memory themselves or through the library
(an application that has reserved the whole device for its own pool, or one that owns
the state buffer and wants no hidden cudaMalloc/cudaFree).  They pass device buffers for
the state, the uniforms and the results; the FP64 scratch comes from a fixed array in the
library.  Its samples and probability total must equal those of the allocating entry
point, svb_measure, call after call (the array keeps the previous call's contents)."""
import ctypes

import numpy as np
import pytest

from svsim_b200 import circuits

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.svb_measure_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_noalloc_measure_matches_allocating_entry_point():
    import torch
    from svsim_b200 import _native as nat
    lib = nat.lib()
    measure = _noalloc(lib)
    shots = 2048
    # two different states, measured one after the other through the shared scratch
    cases = [(16, circuits.brickwork_circuit(16, 20, seed=1234), nat.SVB_FP64),
             (21, circuits.random_matching_circuit(21, 6, seed=3), nat.SVB_FP32)]
    for call, (n, g, prec) in enumerate(cases):
        h = nat.Handle(n, 0, prec)
        h.set_circuit(g)
        h.run()
        h.sync()
        u = np.random.default_rng(call).random(shots)
        want, want_total = h.measure(u)                    # allocating entry point
        dstate, dprec = h.device_ptr()
        du = torch.from_numpy(u).to("cuda:0")
        dout = torch.full((shots,), -1, dtype=torch.int64, device="cuda:0")
        dtot = torch.zeros(1, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        rc = measure(dstate, n, dprec, du.data_ptr(), shots, dout.data_ptr(), dtot.data_ptr(), None)
        assert rc == nat.SVB_OK, lib.svb_last_error()
        torch.cuda.synchronize()
        got = dout.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want)
        assert abs(dtot.item() - want_total) <= 1e-12


def test_noalloc_rejects_states_beyond_the_static_scratch():
    from svsim_b200 import _native as nat
    lib = nat.lib()
    measure = _noalloc(lib)
    h = nat.Handle(12, 0, nat.SVB_FP64)
    dstate, dprec = h.device_ptr()
    rc = measure(dstate, 31, dprec, None, 0, None, None, None)
    assert rc == nat.SVB_ERR_INVALID
    assert b"30" in lib.svb_last_error()

"""torch.autograd binding of the adjoint gradient (svb_adjoint in the C ABI).

``adjoint_energy(params, circuit, observable, sim)`` returns E(params) =
<psi(params)| H |psi(params)> as a 0-d float64 tensor whose backward is the adjoint
gradient computed on the GPU in the same call (one forward sweep, one reverse sweep
over psi and lambda = H psi).  ``circuit`` is a ``circuits.ParamCircuit``: gate records
plus, per gate, which parameter each angle depends on and with which coefficient.
"""
from __future__ import annotations

import numpy as np
import torch

from ._native import SVB_FP64, Handle


class AdjointEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params: torch.Tensor, circuit, terms, handle: Handle):
        p = params.detach().to("cpu", torch.float64).numpy()
        gates = circuit.evaluated(p)
        energy, grad = handle.adjoint(gates, circuit.binding, len(p), terms)
        ctx.save_for_backward(torch.from_numpy(np.asarray(grad, dtype=np.float64)))
        ctx.param_device = params.device
        ctx.param_dtype = params.dtype
        return torch.tensor(energy, dtype=torch.float64, device=params.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        g = g.to(ctx.param_device, ctx.param_dtype)
        return grad_out.to(g.dtype) * g, None, None, None


def adjoint_energy(params: torch.Tensor, circuit, terms, handle: Handle | None = None,
                   device: int = 0) -> torch.Tensor:
    if handle is None:
        handle = Handle(circuit.n, device, SVB_FP64)
    return AdjointEnergy.apply(params, circuit, terms, handle)

"""torch.autograd integration: <psi(theta)|H|psi(theta)> as a differentiable function of the
parameters of a ParametricCircuit, with the gradient from the engine's batched adjoint
kernels (one forward and one backward statevector sweep per parameter set) instead of the
reference's parameter-shift rule (src/algorithms/vqe.cpp:68-94)."""
from __future__ import annotations

import numpy as np
import torch

from .algorithms import adjoint_gradient, batched_energy
from .circuit import ParametricCircuit


class AdjointExpectation(torch.autograd.Function):
    """energies = E(params); params is (P,) or (B, P).  When the parameters need a
    gradient it is computed together with the energy in forward() (the adjoint sweep shares
    the forward pass) and reused by backward(); otherwise forward() runs only the batched
    forward pass.  The parameter sets cross the C ABI as one host array (B x P doubles) and
    the energies and gradients come back the same way."""

    @staticmethod
    def forward(ctx, params: torch.Tensor, ansatz: ParametricCircuit, hamiltonian,
                max_resident: int = 0):
        p = params.detach().to("cpu", torch.float64).numpy()
        single = p.ndim == 1
        sets = p.reshape(1, -1) if single else p   # (B, P), also for P = 0
        if ctx.needs_input_grad[0]:
            e, g = adjoint_gradient(hamiltonian, ansatz, sets, max_resident=max_resident)
            grad = torch.as_tensor(np.asarray(g), dtype=params.dtype, device=params.device)
            if single:
                grad = grad.reshape(-1)
            ctx.save_for_backward(grad)
        else:
            e = batched_energy(hamiltonian, ansatz, sets, max_resident=max_resident)
        energies = torch.as_tensor(np.asarray(e), dtype=params.dtype, device=params.device)
        if single:
            energies = energies.reshape(())
        return energies

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (grad,) = ctx.saved_tensors
        if grad_out.dim() == 0:
            return grad_out * grad, None, None, None
        return grad_out.unsqueeze(-1) * grad, None, None, None


def expectation(params: torch.Tensor, ansatz: ParametricCircuit, hamiltonian,
                max_resident: int = 0) -> torch.Tensor:
    """Differentiable <psi(params)|H|psi(params)>; hamiltonian = [(coeff, pauli), ...]."""
    return AdjointExpectation.apply(params, ansatz, hamiltonian, max_resident)

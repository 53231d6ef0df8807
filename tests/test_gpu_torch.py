"""torch.autograd.Function over the batched adjoint kernels: gradients equal the reference's
parameter-shift gradient within 1e-9, for one parameter set and for a batch."""
import numpy as np
import pytest
import torch

from litequantumcomputingsimulator_b200 import torch_ops
from litequantumcomputingsimulator_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_autograd_single_and_batched(ref):
    pc, theta = W.random_pauli_ansatz(6, 14, seed=41, max_w=6)
    h = W.random_hamiltonian(6, 20, seed=42)
    t = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    e = torch_ops.expectation(t, pc, h)
    e.backward()
    want = ref.parameter_shift_gradient(h, pc, theta)
    assert np.max(np.abs(t.grad.numpy() - want)) < 1e-9
    assert abs(e.item() - ref.expectation(ref.run_statevector(pc.bind(theta)), h)) < 1e-11

    sets = W.random_parameter_sets(pc.num_parameters(), 4, seed=43)
    tb = torch.tensor(sets, dtype=torch.float64, device="cuda", requires_grad=True)
    eb = torch_ops.expectation(tb, pc, h, max_resident=2)
    weights = torch.tensor([1.0, -2.0, 0.5, 3.0], dtype=torch.float64, device="cuda")
    (eb * weights).sum().backward()
    for b in range(4):
        g = ref.parameter_shift_gradient(h, pc, sets[b])
        assert np.max(np.abs(tb.grad[b].cpu().numpy() - weights[b].item() * g)) < 1e-8


def test_forward_without_gradient_runs_the_energy_pass_only(ref):
    """Parameters that need no gradient: the energies equal the gradient path's and the
    reference's, and nothing is saved for backward."""
    pc, theta = W.random_pauli_ansatz(7, 12, seed=44, max_w=6)
    h = W.random_hamiltonian(7, 15, seed=45)
    sets = W.random_parameter_sets(pc.num_parameters(), 3, seed=46)
    with torch.no_grad():
        e0 = torch_ops.expectation(torch.tensor(sets, dtype=torch.float64), pc, h)
    t = torch.tensor(sets, dtype=torch.float64, requires_grad=True)
    e1 = torch_ops.expectation(t, pc, h)
    assert not e0.requires_grad and e1.requires_grad
    assert torch.max(torch.abs(e0 - e1.detach())).item() < 1e-12
    for b in range(3):
        want = ref.expectation(ref.run_statevector(pc.bind(sets[b])), h)
        assert abs(e0[b].item() - want) < 1e-11

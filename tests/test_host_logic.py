"""Host-side logic of the engine that runs without a GPU: gate matrices computed by the
C++ host code against the oracle's restatement (bit for bit), the fusion planner's
invariants, and the seeded workload generators."""
import ctypes as C
import math

import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import _native as N
from litequantumcomputingsimulator_b200 import workloads as W
from oracle.oracle import base_matrix

from helpers import random_circuit


def test_cpp_gate_matrices_equal_oracle_bitwise():
    rng = np.random.default_rng(3)
    for t in lq.GateType:
        if t in (lq.GateType.Measure, lq.GateType.Reset, lq.GateType.Barrier, lq.GateType.Kraus):
            continue
        params = list(rng.uniform(-4, 4, 3))
        g = lq.Gate(t, params[:3] if t == lq.GateType.U else params[:1])
        if t == lq.GateType.Unitary:
            q, _ = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
            g = lq.Gate(t, [], 0, list(q.reshape(-1)))
        if t == lq.GateType.Permutation:
            g = lq.Gate(t, [], 0, [], [2, 0, 3, 1])
        if t == lq.GateType.PauliRotation:
            g = lq.Gate(t, [0.77], 0, pauli="XYZI")
        got = g.base_matrix()
        want = base_matrix(int(t), g.params, g.mat, g.perm, g.pauli)
        assert np.array_equal(got, want), t


def _plan(qc, width):
    arr, n, _k = qc.c_instructions()
    cap = max(1, n)
    widths = (C.c_uint32 * cap)()
    gates = (C.c_uint32 * cap)()
    nb = C.c_uint64(0)
    N.call("lqcs_fusion_plan", qc.num_qubits(), arr, n, width, 0, cap, widths, gates, C.byref(nb))
    return list(widths[: nb.value]), list(gates[: nb.value])


@pytest.mark.parametrize("width", [1, 2, 3, 4, 5, 6])
def test_fusion_plan_invariants(width):
    qc = random_circuit(12, 300, seed=width, max_unitary=2)
    widths, gates = _plan(qc, width)
    assert sum(gates) == qc.num_instructions()
    wide = sum(1 for i in qc.instructions() if len(i.qubits) > width)
    assert sum(1 for w in widths if w > width) <= wide
    assert all(g >= 1 for g in gates)


def test_fusion_reduces_brickwork_passes():
    qc = W.brickwork(30, 40, seed=2025)
    assert qc.num_instructions() == 1800
    w2, _ = _plan(qc, 2)
    w4, _ = _plan(qc, 4)
    assert len(w4) < len(w2) < 1800
    assert max(w4) <= 4


def test_barrier_splits_fusion():
    qc = lq.QuantumCircuit(2)
    qc.h(0).h(1).barrier().x(0).x(1)
    widths, gates = _plan(qc, 2)
    assert sum(gates) == 4 and len(widths) == 2


def test_workloads_are_deterministic():
    a = W.brickwork(8, 3, seed=1)
    b = W.brickwork(8, 3, seed=1)
    assert [(i.gate.type, i.qubits, i.gate.params) for i in a.instructions()] == \
        [(i.gate.type, i.qubits, i.gate.params) for i in b.instructions()]
    cx = [i.qubits for i in a.instructions() if i.gate.n_controls == 1]
    assert len(cx) == 3 * 4
    for layer in range(3):
        used = sum(cx[layer * 4:(layer + 1) * 4], [])
        assert sorted(used) == list(range(8))
    pc, theta = W.random_pauli_ansatz(16, 200, seed=11)
    assert pc.num_parameters() == 200 and theta.shape == (200,)
    assert all(-math.pi <= t <= math.pi for t in theta)
    h = W.random_hamiltonian(16, 500, seed=12)
    assert len(h) == 500 and all(any(c != "I" for c in p) for _, p in h)
    st = W.gaussian_state(10, seed=3)
    assert abs(np.vdot(st, st).real - 1) < 1e-12


def test_alg_bytes_rules():
    qc = lq.QuantumCircuit(10)
    qc.u(0.1, 0.2, 0.3, 0).cx(0, 1).t(2).cz(0, 3).swap(1, 2).ccx(0, 1, 2)
    n = 1 << 10
    want = 32 * n * (1 + 0.5 + 0.5 + 0.25 + 0.5 + 0.25)   # u, cx, t, cz, swap, ccx
    assert W.alg_bytes(qc) == want

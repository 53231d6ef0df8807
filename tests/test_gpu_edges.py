"""Edge cases the reference's own tests exercise (test_statevector.cpp, test_measurement.cpp,
test_expectation.cpp): empty and barrier-only circuits, one- to four-qubit registers on every
path, single shots, empty Hamiltonians and parameter lists, diagonal-only passes, states too
large for the device (a clean error and a usable context afterwards)."""
import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import workloads as W

from helpers import random_circuit

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("n", [1, 2, 5, 12])
def test_empty_and_barrier_only_circuits(n):
    for fuse in (True, False):
        qc = lq.QuantumCircuit(n)
        psi = lq.StatevectorSimulator(fuse_gates=fuse).run_statevector(qc).to_numpy()
        want = np.zeros(1 << n, dtype=np.complex128)
        want[0] = 1
        assert np.array_equal(psi, want)
        qc.barrier()
        qc.barrier()
        assert np.array_equal(lq.StatevectorSimulator(fuse_gates=fuse).run_statevector(qc).to_numpy(), want)
    m = lq.QuantumCircuit(n, n)
    m.measure_all()
    counts = lq.StatevectorSimulator(seed=1).run(m, 17).counts()
    assert counts == {"0" * n: 17}


@pytest.mark.parametrize("n", [1, 2, 3, 4])
@pytest.mark.parametrize("mode", [0, 1, 3, 4])
def test_tiny_registers_every_path(port, ref, n, mode):
    qc = random_circuit(n, 40, seed=10 * n + mode, max_controls=max(0, n - 1),
                        max_unitary=min(3, n))
    init = W.gaussian_state(n, seed=n)
    want = port.run_statevector(qc, fuse=False, state=init)
    sv = lq.Statevector.from_numpy(init)
    sv.apply(qc, fuse_gates=mode != 3, fusion_mode=mode)
    assert np.max(np.abs(sv.to_numpy() - want)) < TOL
    meas = lq.QuantumCircuit(n, n)
    meas.compose(qc)
    meas.measure_all()
    got = lq.StatevectorSimulator(seed=5, fusion_mode=mode).run_registers(meas, 300)
    vals, cnt = np.unique(got, return_counts=True)
    assert {int(v): int(c) for v, c in zip(vals, cnt)} == ref.run(meas, 300, 5)


def test_single_shot_and_zero_shots(ref):
    qc = lq.QuantumCircuit(3, 3)
    qc.h(0).cx(0, 1).ry(0.4, 2).measure_all()
    one = lq.StatevectorSimulator(seed=9).run_registers(qc, 1)
    assert one.shape == (1,)
    assert {int(one[0]): 1} == ref.run(qc, 1, 9)
    with pytest.raises(ValueError, match="shots must be >= 1"):
        lq.StatevectorSimulator(seed=9).run(qc, 0)


def test_empty_hamiltonian_and_parameter_free_ansatz(ref):
    sv = lq.StatevectorSimulator().run_statevector(W.brickwork(6, 2, seed=2))
    assert lq.algorithms.expectation(sv, []) == 0.0
    pc = lq.ParametricCircuit(4)
    pc.h(0)
    pc.cx(0, 1)
    h = [(0.7, "ZZII"), (-0.2, "IXYZ")]
    e, g = lq.algorithms.adjoint_gradient(h, pc, np.zeros(0))
    assert np.asarray(g).size == 0
    want = ref.expectation(ref.run_statevector(pc.bind([])), h)
    assert abs(float(e) - want) < TOL


@pytest.mark.parametrize("n", [12, 13])
def test_diagonal_only_passes(port, n):
    """Tile passes made of phase and diagonal operations only (no remap needed)."""
    qc = lq.QuantumCircuit(n)
    rng = np.random.default_rng(n)
    for _ in range(120):
        a, b = (int(x) for x in rng.permutation(n)[:2])
        k = int(rng.integers(4))
        if k == 0:
            qc.cp(float(rng.uniform(0, 6)), a, b)
        elif k == 1:
            qc.rzz(float(rng.uniform(0, 6)), a, b)
        elif k == 2:
            qc.t(a)
        else:
            qc.rz(float(rng.uniform(0, 6)), a)
    init = W.gaussian_state(n, seed=3)
    want = port.run_statevector(qc, fuse=False, state=init)
    sv = lq.Statevector.from_numpy(init)
    sv.apply(qc, fuse_gates=True, fusion_mode=4)
    assert np.max(np.abs(sv.to_numpy() - want)) < TOL


@pytest.mark.parametrize("k,controls", [(12, 0), (15, 0), (16, 0), (15, 1)])
def test_wide_permutations(port, k, controls):
    """Permutation tables of 2^12..2^16 entries, plain and controlled: the widest ones
    exceed shared memory and take the kernel's global-table form."""
    n = 17
    rng = np.random.default_rng(k + controls)
    init = W.gaussian_state(n, seed=k)
    qubits = [int(q) for q in rng.permutation(n)[: k + controls]]
    table = [int(v) for v in rng.permutation(1 << k)]
    qc = lq.QuantumCircuit(n)
    if controls:
        from litequantumcomputingsimulator_b200.circuit import Gate, GateType, Instruction
        qc.append(Instruction(Gate(GateType.Permutation, [], controls, [], table), qubits))
    else:
        qc.permutation(table, qubits)
    qc.h(0)
    want = port.run_statevector(qc, fuse=False, state=init)
    sv = lq.Statevector.from_numpy(init)
    sv.apply(qc, fuse_gates=False)
    assert np.max(np.abs(sv.to_numpy() - want)) < TOL


def test_state_too_large_fails_cleanly():
    with pytest.raises((MemoryError, ValueError)):
        lq.Statevector(38)   # 4 TiB
    sv = lq.StatevectorSimulator().run_statevector(W.brickwork(8, 2, seed=1))
    assert abs(sv.norm() - 1.0) < 1e-12

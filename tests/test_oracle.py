"""Pins the oracle (the CPU restatement in oracle/) before it is trusted as a checker:

* against the known answers of the reference's own tests (analytic states, the QFT against
  the DFT formula, Pauli expectations, measurement format, gradients, the H2 ground energy,
  trajectory statistics) — tests/test_statevector.cpp, test_qft.cpp, test_expectation.cpp,
  test_measurement.cpp, test_pauli_rotation.cpp, test_vqe.cpp, test_trajectory.cpp of the
  reference project;
* against the reference library itself (oracle/_ref) bit for bit on random circuits of
  every gate type, on counts, expectations and gradients;
* the mt19937_64 restatement against the value the C++ standard requires.
"""
import math

import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import workloads as W
from oracle.oracle import MT64, Port, dm_probabilities_numpy

from helpers import random_circuit

TOL = 1e-12
S = math.sqrt(2) / 2


def sv(port, qc, fuse=True):
    return port.run_statevector(qc, fuse=fuse)


def test_mt19937_64_standard_value():
    g = MT64(5489)
    for _ in range(9999):
        g.next_u64()
    assert g.next_u64() == 9981545732273789042


def test_analytic_states(port):
    qc = lq.QuantumCircuit(1); qc.h(0)
    assert np.allclose(sv(port, qc), [S, S], atol=TOL)
    qc = lq.QuantumCircuit(2); qc.x(0)
    assert abs(sv(port, qc)[1] - 1) < TOL
    qc = lq.QuantumCircuit(2); qc.h(0).cx(0, 1)
    assert np.allclose(sv(port, qc), [S, 0, 0, S], atol=TOL)
    qc = lq.QuantumCircuit(3); qc.h(0).cx(0, 1).cx(1, 2)
    a = sv(port, qc)
    assert abs(a[0] - S) < TOL and abs(a[7] - S) < TOL and np.allclose(a[1:7], 0, atol=TOL)
    qc = lq.QuantumCircuit(2); qc.x(0).cx(0, 1)
    assert abs(sv(port, qc)[3] - 1) < TOL
    qc = lq.QuantumCircuit(2); qc.x(0).cx(1, 0)
    assert abs(sv(port, qc)[1] - 1) < TOL
    qc = lq.QuantumCircuit(2); qc.x(1).cx(1, 0)
    assert abs(sv(port, qc)[3] - 1) < TOL
    qc = lq.QuantumCircuit(2); qc.x(0).swap(0, 1)
    assert abs(sv(port, qc)[2] - 1) < TOL
    qc = lq.QuantumCircuit(2); qc.x(0).x(1).cz(0, 1)
    assert abs(sv(port, qc)[3] + 1) < TOL
    qc = lq.QuantumCircuit(2); qc.x(0).x(1).cp(0.81, 0, 1)
    assert abs(sv(port, qc)[3] - complex(math.cos(0.81), math.sin(0.81))) < TOL
    qc = lq.QuantumCircuit(1); qc.h(0).h(0)
    assert abs(sv(port, qc)[0] - 1) < TOL
    qc = lq.QuantumCircuit(4)
    qc.h(0).rx(0.3, 1).ry(1.1, 2).rz(2.2, 3).cx(0, 2).cz(1, 3).cp(0.5, 2, 3).swap(0, 1)
    qc.t(0).sdg(2).sx(3).u(0.4, 1.5, 2.6, 1)
    assert abs(np.linalg.norm(sv(port, qc)) - 1) < TOL
    qc = lq.QuantumCircuit(3); qc.x(0).x(1).ccx(0, 1, 2)
    assert abs(sv(port, qc)[7] - 1) < TOL
    qc = lq.QuantumCircuit(3); qc.x(0).ccx(0, 1, 2)
    assert abs(sv(port, qc)[1] - 1) < TOL
    qc = lq.QuantumCircuit(3); qc.x(0).x(1).cswap(0, 1, 2)
    assert abs(sv(port, qc)[5] - 1) < TOL
    cycle = [1, 2, 3, 0]
    qc = lq.QuantumCircuit(2); qc.x(0).permutation(cycle, [0, 1])
    assert abs(sv(port, qc)[2] - 1) < TOL
    g = lq.Gate(lq.GateType.Permutation, [], 1, [], cycle)
    qc = lq.QuantumCircuit(3); qc.x(0); qc.append(lq.Instruction(g, [2, 0, 1]))
    assert abs(sv(port, qc)[1] - 1) < TOL
    qc = lq.QuantumCircuit(3); qc.x(0).x(2); qc.append(lq.Instruction(g, [2, 0, 1]))
    assert abs(sv(port, qc)[6] - 1) < TOL
    qc = lq.QuantumCircuit(5); qc.x(4)
    assert abs(sv(port, qc)[16] - 1) < TOL


def _qft_circuit(n, x):
    qc = lq.QuantumCircuit(n)
    for b in range(n):
        if (x >> b) & 1:
            qc.x(b)
    qc.compose(lq.algorithms.qft(n))
    return qc


@pytest.mark.parametrize("n,x", [(3, 0), (3, 1), (3, 5), (4, 7), (4, 13), (5, 21)])
def test_qft_matches_dft(port, n, x):
    a = sv(port, _qft_circuit(n, x))
    dim = 1 << n
    k = np.arange(dim)
    want = np.exp(2j * np.pi * x * k / dim) / math.sqrt(dim)
    assert np.max(np.abs(a - want)) < TOL


def test_qft_inverse(port):
    qc = lq.QuantumCircuit(4)
    qc.x(1).x(3)
    q = lq.algorithms.qft(4)
    qc.compose(q).compose(q.inverse())
    assert abs(sv(port, qc)[10] - 1) < TOL


def test_expectations(port):
    qc = lq.QuantumCircuit(2); qc.x(0)
    a = sv(port, qc)
    for p, v in [("IZ", -1), ("ZI", 1), ("ZZ", -1), ("II", 1), ("IX", 0)]:
        assert abs(port.expectation_value(a, p) - v) < TOL
    qc = lq.QuantumCircuit(1); qc.h(0)
    a = sv(port, qc)
    for p, v in [("X", 1), ("Z", 0), ("Y", 0)]:
        assert abs(port.expectation_value(a, p) - v) < TOL
    qc = lq.QuantumCircuit(1); qc.h(0).s(0)
    a = sv(port, qc)
    assert abs(port.expectation_value(a, "Y") - 1) < TOL
    qc = lq.QuantumCircuit(2); qc.h(0).cx(0, 1)
    a = sv(port, qc)
    for p, v in [("XX", 1), ("ZZ", 1), ("YY", -1), ("ZI", 0), ("IX", 0)]:
        assert abs(port.expectation_value(a, p) - v) < TOL
    for th in (0.3, 1.1, 2.5):
        qc = lq.QuantumCircuit(1); qc.ry(th, 0)
        a = sv(port, qc)
        assert abs(port.expectation_value(a, "Z") - math.cos(th)) < TOL
        assert abs(port.expectation_value(a, "X") - math.sin(th)) < TOL
    qc = lq.QuantumCircuit(2); qc.x(0)
    a = sv(port, qc)
    assert abs(port.expectation(a, [(0.5, "IZ"), (2.0, "ZI"), (-1.0, "II")]) - 0.5) < TOL


def test_measurement_known_answers(port):
    qc = lq.QuantumCircuit(1, 1); qc.x(0).measure(0, 0)
    assert port.run(qc, 100, seed=7) == {1: 100}
    qc = lq.QuantumCircuit(2, 2); qc.x(0).measure(0, 1)
    assert port.run(qc, 10, seed=5) == {0b10: 10}
    qc = lq.QuantumCircuit(2, 2); qc.h(0).cx(0, 1).measure_all()
    c = port.run(qc, 4096, seed=42)
    assert set(c) <= {0, 3} and abs(c[0] - 2048) < 160
    qc = lq.QuantumCircuit(2, 2); qc.h(0).h(1).measure_all()
    assert port.run(qc, 1000, 123) == port.run(qc, 1000, 123)


H2 = [(-1.052373245772859, "II"), (0.39793742484318045, "IZ"), (-0.39793742484318045, "ZI"),
      (-0.01128010425623538, "ZZ"), (0.18093119978423156, "XX")]
H2_EXACT = -1.8572750302023824


def test_h2_ground_energy(port):
    pc = lq.ParametricCircuit(2)
    pc.x(0); pc.ry(1); pc.cx(1, 0)
    e = lambda t: port.expectation(port.run_statevector(pc.bind([t])), H2)
    lo, hi = -math.pi, math.pi
    grid = np.linspace(lo, hi, 721)
    t0 = grid[int(np.argmin([e(t) for t in grid]))]
    a, b = t0 - 0.01, t0 + 0.01
    g = (math.sqrt(5) - 1) / 2
    for _ in range(80):
        c, d = b - g * (b - a), a + g * (b - a)
        if e(c) < e(d):
            b = d
        else:
            a = c
    assert abs(e((a + b) / 2) - H2_EXACT) < 1e-9


def test_parameter_shift_known_answers(port):
    h = [(1.0, "ZZ"), (0.5, "XI"), (-0.3, "IZ")]
    pc = lq.ParametricCircuit(2)
    pc.ry(0); pc.ry(1); pc.cx(0, 1); pc.rz(0); pc.rp("XX", [0, 1])
    theta = [0.3, -0.8, 1.1, 0.5]
    g = port.parameter_shift_gradient(h, pc, theta)
    for k in range(4):
        p, m = list(theta), list(theta)
        p[k] += 1e-6
        m[k] -= 1e-6
        fd = (port.expectation(port.run_statevector(pc.bind(p)), h) -
              port.expectation(port.run_statevector(pc.bind(m)), h)) / 2e-6
        assert abs(g[k] - fd) < 1e-5
    pc = lq.ParametricCircuit(1)
    pc.ry(0)
    assert abs(port.parameter_shift_gradient([(1.0, "Z")], pc, [math.pi])[0]) < 1e-9


def test_trajectory_statistics(port):
    # phase damping: P(0) = 1/2 + 1/2 sqrt(1 - gamma) for H [PD] H [PD]
    g = 0.36
    qc = lq.QuantumCircuit(1, 1); qc.h(0).h(0).measure(0, 0)
    c = port.run(qc, 20000, 17, channels=[lq.KrausChannel.phase_damping(g).ops])
    assert abs(c.get(0, 0) / 20000 - (0.5 + 0.5 * math.sqrt(1 - g))) < 0.017
    # amplitude damping gamma = 1 always relaxes to |0>
    qc = lq.QuantumCircuit(1, 1); qc.x(0).measure(0, 0)
    assert port.run(qc, 200, 5, channels=[lq.KrausChannel.amplitude_damping(1.0).ops]) == {0: 200}
    # trajectories vs the exact density matrix
    qc = lq.QuantumCircuit(2, 2); qc.h(0).cx(0, 1).t(1).cx(1, 0).measure_all()
    ch = [lq.KrausChannel.depolarizing(0.15).ops]
    shots = 20000
    c = port.run(qc, shots, 99, channels=ch)
    exact = dm_probabilities_numpy(qc.instructions(), 2, ch)
    for i in range(4):
        assert abs(c.get(i, 0) / shots - exact[i]) < 0.0125


# ------------------------------------------------------------------ against the reference
@pytest.mark.parametrize("n,seed", [(1, 1), (2, 2), (3, 3), (5, 4), (7, 5), (10, 6), (12, 7)])
def test_port_equals_reference_bitwise(ref, port, n, seed):
    qc = random_circuit(n, 60, seed=seed)
    for fuse in (False, True):
        a = ref.run_statevector(qc, fuse=fuse)
        b = port.run_statevector(qc, fuse=fuse)
        assert np.array_equal(a, b)


def test_port_counts_equal_reference(ref, port):
    for n, d, shots, seed in [(2, 1, 4096, 42), (8, 6, 4096, 7), (12, 10, 2048, 9)]:
        qc = W.brickwork(n, d, seed + 3, measure=True)
        assert port.run(qc, shots, seed) == ref.run(qc, shots, seed)
    qc = lq.QuantumCircuit(2, 2)
    qc.h(0).measure(0, 0).cx(0, 1).reset(1).h(1).measure(1, 1)
    assert port.run(qc, 500, 11) == ref.run(qc, 500, 11)
    noise = lq.NoiseModel().add_all_qubit_channel(lq.KrausChannel.depolarizing(0.2))
    qc = lq.QuantumCircuit(3, 3)
    qc.h(0).cx(0, 1).cx(1, 2).measure_all()
    assert port.run(qc, 300, 123, channels=[c.ops for c in noise.channels()]) == \
        ref.run(qc, 300, 123, noise=noise)


def test_port_expectation_and_gradient_equal_reference(ref, port):
    a = W.gaussian_state(9, seed=1)
    rng = np.random.default_rng(2)
    for _ in range(20):
        p = "".join("IXYZ"[i] for i in rng.integers(0, 4, 9))
        assert port.expectation_value(a, p) == ref.expectation_value(a, p)
    pc, theta = W.random_pauli_ansatz(5, 12, seed=3, max_w=5)
    h = W.random_hamiltonian(5, 10, seed=4)
    assert np.max(np.abs(port.parameter_shift_gradient(h, pc, theta) -
                         ref.parameter_shift_gradient(h, pc, theta))) < 1e-13


def test_dm_numpy_equals_reference(ref):
    qc = W.brickwork(4, 2, seed=5, noise=(0.05, 0.1, 0.2))
    ref_p = ref.dm_probabilities(qc)
    ins = qc.instructions()
    mine = dm_probabilities_numpy(ins, 4)
    assert np.max(np.abs(mine - ref_p)) < 1e-12


def test_trajectory_driver_matches_reference_semantics(ref, port):
    noise = lq.NoiseModel().add_all_qubit_channel(lq.KrausChannel.amplitude_damping(0.3))
    qc = lq.QuantumCircuit(2, 2)
    qc.h(0).cx(0, 1).measure_all()
    regs = ref.trajectories(qc, 200, 77, noise=noise)
    vals, cnt = np.unique(regs, return_counts=True)
    assert {int(v): int(c) for v, c in zip(vals, cnt)} == ref.run(qc, 200, 77, noise=noise)

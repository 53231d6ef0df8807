"""Density-matrix backend on the GPU (DensityMatrixSimulator semantics): rho of n qubits as a
2n-qubit device state, gates as U (x) conj(U), channels as superoperators, all fused into
tile passes.  Checked against the compiled reference's DensityMatrix (probabilities within
1e-12, identical counts for the same seed), against |psi><psi| for every gate type, and used
for the config-3 trajectory cross-check at 12 qubits (beyond the reference's 10)."""
import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import workloads as W

from helpers import random_circuit

pytestmark = pytest.mark.gpu
TOL = 1e-12


def counts_of(regs):
    vals, cnt = np.unique(regs, return_counts=True)
    return {int(v): int(c) for v, c in zip(vals, cnt)}


@pytest.mark.parametrize("n", [4, 6, 9])
def test_pure_state_density_matrix_every_gate_type(port, n):
    qc = random_circuit(n, 60, seed=70 + n, max_controls=2, max_unitary=3)
    psi = port.run_statevector(qc, fuse=False)
    rho = lq.DensityMatrixSimulator().run_density_matrix(qc)
    want = np.outer(psi, psi.conj())
    assert np.max(np.abs(rho.to_numpy() - want)) < TOL
    assert abs(rho.trace() - 1.0) < 1e-12 and abs(rho.purity() - 1.0) < 1e-12
    assert abs(rho.element(1, 0) - want[1, 0]) < TOL


@pytest.mark.parametrize("n", [6, 10])
def test_noisy_probabilities_match_reference(ref, n):
    qc = W.brickwork(n, 5, seed=n, noise=(0.05, 0.1, 0.2))
    want = ref.dm_probabilities(qc)
    got = lq.DensityMatrixSimulator().run_density_matrix(qc).probabilities()
    assert np.max(np.abs(got - want)) < TOL


def test_noise_model_counts_identical(ref):
    noise = lq.NoiseModel()
    noise.add_all_qubit_channel(lq.KrausChannel.depolarizing(0.03))
    noise.add_all_qubit_channel(lq.KrausChannel.amplitude_damping(0.1))
    qc = W.brickwork(7, 4, seed=3, measure=True)
    want = ref.dm_run(qc, 2000, 11, noise=noise)
    got = counts_of(lq.DensityMatrixSimulator(seed=11, noise=noise).run_registers(qc, 2000))
    assert got == want
    want_p = ref.dm_probabilities(qc, noise=noise)
    got_p = lq.DensityMatrixSimulator(noise=noise).run_density_matrix(qc).probabilities()
    assert np.max(np.abs(got_p - want_p)) < TOL


def test_reference_errors():
    sim = lq.DensityMatrixSimulator(seed=1)
    qc = lq.QuantumCircuit(2, 2)
    qc.h(0).reset(1).measure_all()
    with pytest.raises(ValueError, match="Reset is not supported"):
        sim.run(qc, 10)
    qc = lq.QuantumCircuit(2, 2)
    qc.h(0).measure(0, 0).x(1).measure(1, 1)
    with pytest.raises(ValueError, match="mid-circuit measurement is not supported"):
        sim.run(qc, 10)
    qc = lq.QuantumCircuit(2)
    qc.h(0)
    with pytest.raises(ValueError, match="no measurements"):
        sim.run(qc, 10)


def test_config3_cross_check_12_qubits():
    """Config-3 noise at 12 qubits: the trajectory histogram's TVD to the GPU density matrix's
    distribution is within the spread of 1024 exact draws (seeded bootstrap)."""
    n, shots = 12, 1024
    qc = W.brickwork(n, 12, seed=2027, measure=True, noise=(1e-3, 1e-2, 1e-3))
    exact = lq.DensityMatrixSimulator().run_density_matrix(qc).probabilities()
    exact = exact / exact.sum()
    regs = lq.StatevectorSimulator(seed=98, max_resident=256).run_registers(qc, shots)
    freq = np.bincount(regs.astype(np.int64), minlength=1 << n) / shots
    tvd = 0.5 * np.abs(freq - exact).sum()
    rng = np.random.default_rng(0)
    boot = []
    for _ in range(200):
        draw = rng.choice(1 << n, size=shots, p=exact)
        boot.append(0.5 * np.abs(np.bincount(draw, minlength=1 << n) / shots - exact).sum())
    assert tvd <= np.quantile(boot, 0.999)

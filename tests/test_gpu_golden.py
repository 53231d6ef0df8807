"""The engine against the golden fixtures (tests/golden/: outputs of the reference library
itself on seeded cases), through the C ABI on the GPU — so parity holds on machines without
the reference sources.  Amplitudes within 1e-12 under every fusion mode; counts maps
identical (same seed, same uniforms); expectations within 1e-12; adjoint and
parameter-shift gradients within 1e-9 of the reference's parameter shift; density-matrix
probabilities within 1e-12."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import cases as G  # noqa: E402

import litequantumcomputingsimulator_b200 as lq  # noqa: E402
from litequantumcomputingsimulator_b200 import workloads as W  # noqa: E402

pytestmark = pytest.mark.gpu
ARRAYS, CASES = G.load()
TOL = 1e-12


@pytest.mark.parametrize("mode", [0, 1, 3, 4])
@pytest.mark.parametrize("name", sorted(G.AMPLITUDES))
def test_amplitudes(name, mode):
    spec = G.AMPLITUDES[name]
    qc = G.circuit(spec)
    if spec.get("init"):
        sv = lq.Statevector.from_numpy(W.gaussian_state(*spec["init"]))
        sv.apply(qc, fuse_gates=spec["fuse"] or mode != 0, fusion_mode=mode)
        got = sv.to_numpy()
    else:
        sim = lq.StatevectorSimulator(fuse_gates=spec["fuse"] or mode != 0, fusion_mode=mode)
        got = sim.run_statevector(qc).to_numpy()
    assert np.max(np.abs(got - ARRAYS[name])) < TOL


@pytest.mark.parametrize("name", sorted(G.COUNTS))
def test_counts(name):
    spec = G.COUNTS[name]
    qc = G.circuit(spec)
    want = {int(k): v for k, v in CASES[name]["counts"].items()}
    sim = lq.StatevectorSimulator(seed=spec["seed"], noise=G.noise_model(spec.get("noise_model")))
    regs = sim.run_registers(qc, spec["shots"])
    vals, cnt = np.unique(regs, return_counts=True)
    assert {int(v): int(c) for v, c in zip(vals, cnt)} == want
    n = qc.num_clbits()
    keys = {format(k, "b").zfill(n)[-n:]: v for k, v in want.items()}
    assert sim.run(qc, spec["shots"]).counts() == keys


@pytest.mark.parametrize("name", sorted(G.EXPECTATIONS))
def test_expectations(name):
    spec = CASES[name]
    sv = lq.Statevector.from_numpy(W.gaussian_state(*spec["state"]))
    h = W.random_hamiltonian(*spec["hamiltonian"])
    assert abs(lq.algorithms.expectation(sv, h) - spec["energy"]) < TOL
    got = lq.algorithms.expectation_terms(sv, [p for _, p in h[: spec["terms_each"]]])
    assert np.max(np.abs(np.asarray(got) - spec["term_values"])) < TOL


@pytest.mark.parametrize("name", sorted(G.GRADIENTS))
def test_gradients(name):
    spec = G.GRADIENTS[name]
    pc, theta = W.random_pauli_ansatz(*spec["ansatz"], max_w=spec["max_w"])
    h = W.random_hamiltonian(*spec["hamiltonian"])
    want = ARRAYS[name]
    _, g = lq.algorithms.adjoint_gradient(h, pc, theta)
    assert np.max(np.abs(g - want)) < 1e-9
    ps = np.array(lq.algorithms.parameter_shift_gradient(h, pc, theta))
    assert np.max(np.abs(ps - want)) < 1e-9


@pytest.mark.parametrize("name", sorted(G.DENSITY))
def test_density_probabilities(name):
    spec = G.DENSITY[name]
    qc = G.circuit(spec)
    sim = lq.DensityMatrixSimulator(noise=G.noise_model(spec.get("noise_model")))
    got = sim.run_density_matrix(qc).probabilities()
    assert np.max(np.abs(got - ARRAYS[name])) < TOL


@pytest.mark.parametrize("name", sorted(G.MODEXP))
@pytest.mark.parametrize("mode", [0, 3])
def test_modular_exponentiation(name, mode):
    """Controlled modular multiplications (singly controlled permutations of the work
    register) after X(work 0) and H on the counting register."""
    spec = G.MODEXP[name]
    nc, nw = spec["n_count"], spec["n_work"]
    qc = lq.QuantumCircuit(nc + nw)
    qc.x(nc)
    for j in range(nc):
        qc.h(j)
    qc.compose(lq.algorithms.modular_exponentiation(spec["a"], spec["N"], nc, nw))
    got = lq.StatevectorSimulator(fusion_mode=mode).run_statevector(qc).to_numpy()
    assert np.max(np.abs(got - ARRAYS[name])) < TOL


@pytest.mark.parametrize("name", sorted(G.SHOR))
def test_shor(name):
    """Seeded Shor runs: base, period, factors, attempts and the successful round's counts
    all equal the reference's."""
    spec = G.SHOR[name]
    want = CASES[name]["result"]
    got = lq.algorithms.shor(spec["N"], spec["shots"], spec["max_attempts"], spec["seed"])
    for key in ("success", "factor1", "factor2", "a", "period", "attempts"):
        assert getattr(got, key) == want[key], key
    n = 2 * spec["N"].bit_length()
    keys = {format(int(k), "b").zfill(n): v for k, v in want["counts"].items()}
    assert got.counts == keys

"""Pins the oracle to the committed golden fixtures (tests/golden/), which hold the outputs
of the reference library itself (compiled from its sources) on seeded cases: amplitudes,
counts maps, expectation values, parameter-shift gradients, density-matrix probabilities
and `Rng` uniforms.  These run without the reference sources."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import cases as G  # noqa: E402

from litequantumcomputingsimulator_b200 import workloads as W  # noqa: E402
from oracle.oracle import MT64, dm_probabilities_numpy  # noqa: E402

ARRAYS, CASES = G.load()
TOL = 1e-12


def test_fixture_covers_every_case():
    for group in (G.AMPLITUDES, G.COUNTS, G.EXPECTATIONS, G.GRADIENTS, G.DENSITY, G.UNIFORMS):
        for name in group:
            assert name in CASES
    for name in list(G.AMPLITUDES) + list(G.GRADIENTS) + list(G.DENSITY) + list(G.UNIFORMS):
        assert name in ARRAYS


@pytest.mark.parametrize("name", sorted(G.AMPLITUDES))
def test_oracle_amplitudes(port, name):
    spec = G.AMPLITUDES[name]
    qc = G.circuit(spec)
    init = W.gaussian_state(*spec["init"]) if spec.get("init") else None
    got = port.run_statevector(qc, fuse=spec["fuse"], state=init)
    assert np.max(np.abs(got - ARRAYS[name])) < TOL


@pytest.mark.parametrize("name", sorted(G.COUNTS))
def test_oracle_counts(port, name):
    spec = G.COUNTS[name]
    qc = G.circuit(spec)
    got = port.run(qc, spec["shots"], spec["seed"], channels=G.channel_ops(spec.get("noise_model")))
    want = {int(k): v for k, v in CASES[name]["counts"].items()}
    assert got == want


@pytest.mark.parametrize("name", sorted(G.EXPECTATIONS))
def test_oracle_expectations(port, name):
    spec = CASES[name]
    st = W.gaussian_state(*spec["state"])
    h = W.random_hamiltonian(*spec["hamiltonian"])
    assert abs(port.expectation(st, h) - spec["energy"]) < TOL
    for (_, p), want in zip(h, spec["term_values"]):
        assert abs(port.expectation_value(st, p) - want) < TOL


@pytest.mark.parametrize("name", sorted(G.GRADIENTS))
def test_oracle_gradients(port, name):
    spec = G.GRADIENTS[name]
    pc, theta = W.random_pauli_ansatz(*spec["ansatz"], max_w=spec["max_w"])
    assert np.array_equal(np.asarray(theta, dtype=np.float64), ARRAYS[name + "_theta"])
    h = W.random_hamiltonian(*spec["hamiltonian"])
    got = port.parameter_shift_gradient(h, pc, theta)
    assert np.max(np.abs(got - ARRAYS[name])) < 1e-10


@pytest.mark.parametrize("name", sorted(G.DENSITY))
def test_oracle_density_probabilities(name):
    spec = G.DENSITY[name]
    qc = G.circuit(spec)
    got = dm_probabilities_numpy(qc.instructions(), qc.num_qubits(),
                                 G.channel_ops(spec.get("noise_model")))
    assert np.max(np.abs(got - ARRAYS[name])) < TOL


@pytest.mark.parametrize("name", sorted(G.UNIFORMS))
def test_oracle_uniforms_bit_exact(name):
    spec = G.UNIFORMS[name]
    g = MT64(spec["seed"])
    assert np.array_equal(g.uniforms(spec["count"]), ARRAYS[name])

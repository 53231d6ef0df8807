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


# ---- Shor's classical side (no GPU: these cases end before any period finding)

@pytest.mark.parametrize("name", ["shor_21_gcd", "shor_27_power", "shor_97_prime"])
def test_shor_classical_paths(name):
    from litequantumcomputingsimulator_b200 import algorithms as A
    spec = G.SHOR[name]
    want = CASES[name]["result"]
    got = A.shor(spec["N"], spec["shots"], spec["max_attempts"], spec["seed"])
    for key in ("success", "factor1", "factor2", "a", "period", "attempts"):
        assert getattr(got, key) == want[key], key
    assert got.counts == {} and got.circuit is None


@pytest.mark.parametrize("name", sorted(G.SHOR))
def test_shor_first_base_draw(name):
    """The first base equals the reference's std::uniform_int_distribution draw."""
    from litequantumcomputingsimulator_b200 import algorithms as A
    spec = G.SHOR[name]
    want = CASES[name]["result"]
    if want["attempts"] == 0:
        pytest.skip("classical shortcut: no base drawn")
    assert want["attempts"] == 1
    assert A._Mt64Stream(spec["seed"]).uniform_int(2, spec["N"] - 2) == want["a"]


def test_rng_u64_matches_uniforms():
    """lqcs_rng_u64 gives the raw mt19937_64 draws (equal to the oracle's restatement, which
    is pinned to the C++ standard's 10000th value), from any starting position."""
    from litequantumcomputingsimulator_b200 import _native as N
    for name in sorted(G.UNIFORMS):
        spec = G.UNIFORMS[name]
        raw = np.empty(spec["count"], dtype=np.uint64)
        N.call("lqcs_rng_u64", spec["seed"], 0, raw.size, raw.ctypes.data)
        g = MT64(spec["seed"])
        assert [g.next_u64() for _ in range(raw.size)] == [int(v) for v in raw]
        tail = np.empty(5, dtype=np.uint64)
        N.call("lqcs_rng_u64", spec["seed"], 7, 5, tail.ctypes.data)
        assert np.array_equal(tail, raw[7:12])


def test_number_theory():
    from fractions import Fraction
    from litequantumcomputingsimulator_b200 import algorithms as A
    primes = [n for n in range(2, 400) if all(n % d for d in range(2, int(n ** 0.5) + 1))]
    assert [n for n in range(400) if A.is_prime(n)] == primes
    for n in range(4, 5000):
        b = A.perfect_power_base(n)
        ks = [(r, k) for k in range(2, n.bit_length() + 1)
              for r in (round(n ** (1 / k)) - 1, round(n ** (1 / k)), round(n ** (1 / k)) + 1)
              if r >= 2 and r ** k == n]
        assert b == (min(ks, key=lambda t: t[1])[0] if ks else 0), n
    rng = np.random.default_rng(5)
    for _ in range(300):
        den = 1 << int(rng.integers(4, 24))
        num = int(rng.integers(1, den))
        lim = int(rng.integers(2, 2000))
        got = A.continued_fraction_denominators(num, den, lim)
        x, want, conv = Fraction(num, den), [], []
        q2, q1, f = 1, 0, x
        while True:   # convergent denominators by the textbook recurrence
            a = f.numerator // f.denominator
            q = a * q1 + q2
            if q > lim:
                break
            want.append(q)
            q2, q1 = q1, q
            if f == a:
                break
            f = 1 / (f - a)
        assert got == want


def test_modular_exponentiation_builder():
    from litequantumcomputingsimulator_b200 import algorithms as A
    from litequantumcomputingsimulator_b200.circuit import GateType
    qc = A.modular_exponentiation(7, 15, 3, 4)
    insts = qc.instructions()
    assert qc.num_qubits() == 7 and len(insts) == 3
    for j, inst in enumerate(insts):
        assert inst.gate.type == GateType.Permutation and inst.gate.n_controls == 1
        assert list(inst.qubits) == [j, 3, 4, 5, 6]
        f = pow(7, 1 << j, 15)
        assert list(inst.gate.perm) == [(f * y) % 15 if y < 15 else y for y in range(16)]
    for args in ((7, 1, 3, 4), (7, 33, 3, 4), (6, 15, 3, 4)):
        with pytest.raises(ValueError):
            A.modular_exponentiation(*args)
    with pytest.raises(ValueError):
        A.shor(3)

"""GPU parity: the engine's CUDA path against the oracle (the C restatement and the
reference library itself) on the same seeded inputs.

Tolerances: amplitudes within 1e-12 (absolute, per amplitude) of the CPU path; counts
identical given the same seed; expectation values within 1e-12; gradients within 1e-9 of
the reference's parameter-shift gradient.
"""
import math

import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import workloads as W

from helpers import random_circuit, random_unitary

pytestmark = pytest.mark.gpu
TOL = 1e-12


def engine_state(qc, fuse=False, width=0, init=None):
    if init is None:
        sim = lq.StatevectorSimulator(fuse_gates=fuse, max_fusion_width=width)
        return sim.run_statevector(qc).to_numpy()
    sv = lq.Statevector.from_numpy(init)
    sv.apply(qc, fuse_gates=fuse, max_fusion_width=width)
    return sv.to_numpy()


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 9])
@pytest.mark.parametrize("seed", [1, 2])
def test_every_gate_type_unfused(port, n, seed):
    qc = random_circuit(n, 60, seed=100 * n + seed)
    want = port.run_statevector(qc, fuse=False)
    got = engine_state(qc, fuse=False)
    assert np.max(np.abs(got - want)) < TOL


@pytest.mark.parametrize("n", [3, 6, 8, 11])
@pytest.mark.parametrize("width", [1, 2, 3, 4, 5, 6])
def test_fused_blocks_match(port, n, width):
    qc = random_circuit(n, 80, seed=7 * n + width)
    want = port.run_statevector(qc, fuse=False)
    got = engine_state(qc, fuse=True, width=min(width, n))
    assert np.max(np.abs(got - want)) < TOL


@pytest.mark.parametrize("n", [5, 7, 12])
def test_from_random_state(port, n):
    init = W.gaussian_state(n, seed=3)
    qc = random_circuit(n, 40, seed=n)
    want = port.run_statevector(qc, fuse=False, state=init)
    for fuse in (False, True):
        got = engine_state(qc, fuse=fuse, init=init)
        assert np.max(np.abs(got - want)) < TOL


def test_single_qubit_every_target_and_control(port):
    n = 11
    init = W.gaussian_state(n, seed=11)
    rng = np.random.default_rng(0)
    for t in range(n):
        qc = lq.QuantumCircuit(n)
        qc.u(*rng.uniform(0, 2 * math.pi, 3), t)
        qc.rz(0.3, t).t(t).p(0.7, t)
        for c in range(n):
            if c != t:
                qc.cx(c, t).cp(0.4, c, t).crx(0.9, c, t)
        want = port.run_statevector(qc, fuse=False, state=init)
        got = engine_state(qc, fuse=False, init=init)
        assert np.max(np.abs(got - want)) < TOL, t


def test_two_qubit_and_block_every_pair(port):
    n = 8
    init = W.gaussian_state(n, seed=5)
    rng = np.random.default_rng(1)
    qc = lq.QuantumCircuit(n)
    for a in range(n):
        for b in range(n):
            if a != b:
                qc.unitary(random_unitary(2, rng), [a, b])
                qc.swap(a, b)
    want = port.run_statevector(qc, fuse=False, state=init)
    got = engine_state(qc, fuse=False, init=init)
    assert np.max(np.abs(got - want)) < TOL


def test_matches_reference_library(ref):
    for n, seed in [(4, 1), (9, 2), (13, 3)]:
        qc = random_circuit(n, 50, seed=seed)
        want = ref.run_statevector(qc, fuse=True)
        for fuse in (False, True):
            got = engine_state(qc, fuse=fuse)
            assert np.max(np.abs(got - want)) < TOL


def test_brickwork_20q_reference(ref):
    qc = W.brickwork(20, 20, seed=2024)
    want = ref.run_statevector(qc, fuse=True)
    for width in (0, 2, 4, 5):
        got = engine_state(qc, fuse=True, width=width)
        assert np.max(np.abs(got - want)) < TOL


def test_qft_random_state(ref):
    n = 14
    init = W.gaussian_state(n, seed=9)
    qc = lq.algorithms.qft(n)
    want = ref.evolve_from(qc, init)
    for fuse in (False, True):
        got = engine_state(qc, fuse=fuse, init=init)
        assert np.max(np.abs(got - want)) < TOL


@pytest.mark.parametrize("n,depth,shots,seed", [(2, 1, 4096, 42), (10, 6, 4096, 123),
                                                (16, 10, 8192, 9), (20, 20, 4096, 2024)])
def test_sampling_counts_identical(ref, n, depth, shots, seed):
    qc = W.brickwork(n, depth, seed=seed + 1, measure=True)
    want = ref.run(qc, shots, seed)
    got_regs = lq.StatevectorSimulator(seed=seed).run_registers(qc, shots)
    vals, cnt = np.unique(got_regs, return_counts=True)
    got = {int(v): int(c) for v, c in zip(vals, cnt)}
    assert got == want


def test_sample_margin_and_upper_bound(port):
    n = 12
    init = W.gaussian_state(n, seed=4)
    sv = lq.Statevector.from_numpy(init)
    u = W.UniformStream(77).take(5000)
    idx, margin = sv.sample(u)
    cum = np.cumsum(np.abs(init) ** 2)
    total = cum[-1]
    want = np.searchsorted(cum, u * total, side="right")
    assert np.array_equal(idx.astype(np.int64), want)
    assert margin > 0


def test_counts_fusion_on_off_identical():
    qc = lq.QuantumCircuit(3, 3)
    qc.h(0).t(0).cx(0, 1).rx(0.4, 2).sx(2).cx(1, 2).measure_all()
    on = lq.StatevectorSimulator(seed=5, fuse_gates=True).run(qc, 512).counts()
    off = lq.StatevectorSimulator(seed=5, fuse_gates=False).run(qc, 512).counts()
    assert on == off


def test_measurement_format_and_mapping():
    qc = lq.QuantumCircuit(2, 2)
    qc.x(0).measure(0, 1)
    r = lq.StatevectorSimulator(seed=5).run(qc, 10)
    assert r.counts() == {"10": 10}
    qc = lq.QuantumCircuit(1, 1)
    qc.x(0).measure(0, 0)
    assert lq.StatevectorSimulator(seed=7).run(qc, 100).counts() == {"1": 100}


@pytest.mark.parametrize("seed", [42, 7, 11])
def test_midcircuit_and_reset_counts_identical(ref, seed):
    circuits = []
    a = lq.QuantumCircuit(2, 2)
    a.h(0).measure(0, 0).cx(0, 1).measure(1, 1)
    circuits.append(a)
    b = lq.QuantumCircuit(1, 2)
    b.h(0).measure(0, 0).h(0).measure(0, 1)
    circuits.append(b)
    c = lq.QuantumCircuit(2, 2)
    c.h(0).cx(0, 1).reset(0).measure_all()
    circuits.append(c)
    d = lq.QuantumCircuit(6, 6)
    d.h(0).cx(0, 3).ry(0.3, 5).measure(3, 2).reset(3).cx(5, 3).h(1).measure_all()
    circuits.append(d)
    for qc in circuits:
        want = ref.run(qc, 512, seed)
        regs = lq.StatevectorSimulator(seed=seed).run_registers(qc, 512)
        vals, cnt = np.unique(regs, return_counts=True)
        assert {int(v): int(c) for v, c in zip(vals, cnt)} == want


def test_trajectory_counts_identical(ref):
    noise = lq.NoiseModel()
    noise.add_all_qubit_channel(lq.KrausChannel.depolarizing(0.15))
    noise.add_all_qubit_channel(lq.KrausChannel.amplitude_damping(0.1))
    qc = lq.QuantumCircuit(3, 3)
    qc.h(0).cx(0, 1).t(1).cx(1, 2).measure_all()
    want = ref.run(qc, 400, 99, noise=noise)
    regs = lq.StatevectorSimulator(seed=99, noise=noise).run_registers(qc, 400)
    vals, cnt = np.unique(regs, return_counts=True)
    got = {int(v): int(c) for v, c in zip(vals, cnt)}
    assert got == want


def test_trajectory_matches_density_matrix(ref):
    noise = lq.NoiseModel()
    noise.add_all_qubit_channel(lq.KrausChannel.depolarizing(0.15))
    qc = lq.QuantumCircuit(2, 2)
    qc.h(0).cx(0, 1).t(1).cx(1, 0).measure_all()
    shots = 20000
    counts = lq.StatevectorSimulator(seed=99, noise=noise).run(qc, shots).counts()
    exact = ref.dm_probabilities(qc, noise)
    for i, key in enumerate(["00", "01", "10", "11"]):
        assert abs(counts.get(key, 0) / shots - exact[i]) < 0.0125


@pytest.mark.parametrize("n", [3, 8, 14])
def test_expectation_values(port, n):
    init = W.gaussian_state(n, seed=n)
    sv = lq.Statevector.from_numpy(init)
    rng = np.random.default_rng(n)
    paulis = ["".join("IXYZ"[i] for i in rng.integers(0, 4, n)) for _ in range(40)]
    got = lq.algorithms.expectation_terms(sv, paulis)
    want = np.array([port.expectation_value(init, p) for p in paulis])
    assert np.max(np.abs(got - want)) < TOL
    h = [(float(rng.standard_normal()), p) for p in paulis]
    assert abs(lq.algorithms.expectation(sv, h) - port.expectation(init, h)) < 1e-11


def test_known_expectations():
    qc = lq.QuantumCircuit(2)
    qc.h(0).cx(0, 1)
    sv = lq.StatevectorSimulator().run_statevector(qc)
    assert abs(sv.expectation_value("ZZ") - 1) < TOL
    assert abs(sv.expectation_value("XX") - 1) < TOL
    assert abs(sv.expectation_value("YY") + 1) < TOL
    assert abs(sv.expectation_value("ZI")) < TOL


@pytest.mark.parametrize("n", [3, 9])
def test_collapse_reset_kraus(port, n):
    from oracle.oracle import _PortLib
    lib = _PortLib.get()
    init = W.gaussian_state(n, seed=21)
    for q in range(n):
        for u in (0.1, 0.9):
            a = init.copy()
            o_want = lib.orc_collapse_qubit(a.ctypes.data, a.size, q, u)
            sv = lq.Statevector.from_numpy(init)
            o_got = sv.collapse(q, u)
            assert o_got == o_want
            assert np.max(np.abs(sv.to_numpy() - a)) < TOL
            b = init.copy()
            lib.orc_reset_qubit(b.ctypes.data, b.size, q, u)
            sv = lq.Statevector.from_numpy(init)
            sv.reset_qubit(q, u)
            assert np.max(np.abs(sv.to_numpy() - b)) < TOL
        for ch in (lq.KrausChannel.depolarizing(0.3), lq.KrausChannel.amplitude_damping(0.4)):
            for k in ch.ops:
                kk = np.ascontiguousarray(np.asarray(k, dtype=np.complex128))
                want = lib.orc_kraus_probability(init.ctypes.data, init.size, q, kk.ctypes.data)
                got = lq.Statevector.from_numpy(init).kraus_probability(q, kk)
                assert abs(got - want) < TOL


@pytest.mark.parametrize("a,N,nc,nw", [(2, 209, 8, 8), (7, 187, 6, 8), (5, 21, 14, 5)])
def test_modular_exponentiation_vs_reference(ref, a, N, nc, nw):
    """algorithms::modular_exponentiation on the tile path (>= 12 qubits): singly controlled
    permutations of 5-8 work qubits between tile passes."""
    want = ref.modexp_statevector(a, N, nc, nw)
    qc = lq.QuantumCircuit(nc + nw)
    qc.x(nc)
    for j in range(nc):
        qc.h(j)
    qc.compose(lq.algorithms.modular_exponentiation(a, N, nc, nw))
    got = lq.StatevectorSimulator().run_statevector(qc).to_numpy()
    assert np.max(np.abs(got - want)) < TOL


@pytest.mark.parametrize("N,seed", [(39, 2), (51, 5), (65, 11), (119, 9), (143, 6)])
def test_shor_vs_reference(ref, N, seed):
    want = ref.shor(N, 64, 10, seed)
    got = lq.algorithms.shor(N, 64, 10, seed)
    for key in ("success", "factor1", "factor2", "a", "period", "attempts"):
        assert getattr(got, key) == want[key], key
    n = 2 * N.bit_length()
    assert got.counts == {format(k, "b").zfill(n): v for k, v in want["counts"].items()}


def test_parameter_shift_matches_reference(ref):
    pc, theta = W.random_pauli_ansatz(6, 20, seed=5)
    h = W.random_hamiltonian(6, 30, seed=6)
    want = ref.parameter_shift_gradient(h, pc, theta)
    got = np.array(lq.algorithms.parameter_shift_gradient(h, pc, theta))
    assert np.max(np.abs(got - want)) < 1e-9


@pytest.mark.parametrize("n", [3, 7])
def test_adjoint_matches_parameter_shift_and_fd(ref, n):
    pc, theta = W.random_pauli_ansatz(n, 16, seed=n, max_w=min(8, n))
    h = W.random_hamiltonian(n, 25, seed=n + 1)
    want = ref.parameter_shift_gradient(h, pc, theta)
    e, g = lq.algorithms.adjoint_gradient(h, pc, theta)
    assert np.max(np.abs(g - want)) < 1e-9
    e_ref = ref.expectation(ref.run_statevector(pc.bind(theta)), h)
    assert abs(e - e_ref) < 1e-11
    hstep = 1e-4
    for k in range(0, len(theta), 5):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += hstep
        tm[k] -= hstep
        ep = ref.expectation(ref.run_statevector(pc.bind(tp)), h)
        em = ref.expectation(ref.run_statevector(pc.bind(tm)), h)
        assert abs(g[k] - (ep - em) / (2 * hstep)) < 1e-6


@pytest.mark.parametrize("n", [12, 14])
def test_adjoint_hamiltonian_over_tiles(ref, n):
    """The Hamiltonian apply stages 2^11-amplitude source tiles grouped by the high bits of
    each term's X mask: energies and gradients at 12 and 14 qubits (2 and 8 groups) match the
    reference, batched (default resident count) as one set at a time."""
    pc, _ = W.random_pauli_ansatz(n, 12, seed=n + 20, max_w=8)
    h = W.random_hamiltonian(n, 60, seed=n + 21)
    sets = W.random_parameter_sets(pc.num_parameters(), 5, seed=n + 22)
    e_b, g_b = lq.algorithms.adjoint_gradient(h, pc, sets)
    for b in (0, 4):
        e_ref = ref.expectation(ref.run_statevector(pc.bind(sets[b])), h)
        assert abs(e_b[b] - e_ref) < 1e-11
        want = ref.parameter_shift_gradient(h, pc, sets[b])
        assert np.max(np.abs(g_b[b] - want)) < 1e-9
        e1, g1 = lq.algorithms.adjoint_gradient(h, pc, sets[b])
        assert abs(e1 - e_b[b]) < 1e-12 and np.max(np.abs(g1 - g_b[b])) < 1e-12


@pytest.mark.parametrize("n", [7, 13, 16])
def test_adjoint_rotation_tile_passes(ref, monkeypatch, n):
    """Runs of parameterised rotations go through shared-memory tile passes (forward and
    backward, gradients summed over tiles); fixed gates and rotations whose X bits do not fit
    a tile split the runs.  Energies and gradients agree with one launch per step and with
    the reference's parameter-shift gradient."""
    pc, _ = W.random_pauli_ansatz(n, 14, seed=n + 40, max_w=min(8, n))
    pc.h(0)
    pc.cx(1, n - 1)
    pc.rp("X" * n, list(range(n)))   # X bits on every qubit: wider than any tile when n > 12
    pc.ry(n - 1)
    pc.s(2)
    more, _ = W.random_pauli_ansatz(n, 9, seed=n + 41, max_w=min(8, n))
    for inst in more.template().instructions():
        pc.rp(inst.gate.pauli, list(inst.qubits))
    h = W.random_hamiltonian(n, 30, seed=n + 42)
    sets = W.random_parameter_sets(pc.num_parameters(), 6, seed=n + 43)
    e_t, g_t = lq.algorithms.adjoint_gradient(h, pc, sets)
    lq.algorithms.release_caches()
    monkeypatch.setenv("LQCS_ADJ_TILES", "0")
    e_s, g_s = lq.algorithms.adjoint_gradient(h, pc, sets)
    lq.algorithms.release_caches()
    assert np.max(np.abs(e_t - e_s)) < 1e-12
    assert np.max(np.abs(g_t - g_s)) < 1e-12
    want = ref.parameter_shift_gradient(h, pc, sets[2])
    assert np.max(np.abs(g_t[2] - want)) < 1e-9


def test_repeated_runs_reuse_compiled_programs(port, monkeypatch):
    """run_statevector / run keep the compiled programs of recent circuits: a repeated call
    gives the same amplitudes bit for bit, a changed tile setting compiles anew (and still
    matches the oracle), and release_caches drops them without changing results."""
    qc = W.brickwork(14, 6, seed=3)
    want = port.run_statevector(qc, fuse=False)
    sim = lq.StatevectorSimulator()
    a = sim.run_statevector(qc).to_numpy()
    b = sim.run_statevector(qc).to_numpy()
    assert np.array_equal(a, b) and np.max(np.abs(a - want)) < TOL
    monkeypatch.setenv("LQCS_TILE_BITS", "11")
    c = sim.run_statevector(qc).to_numpy()
    assert np.max(np.abs(c - want)) < TOL
    monkeypatch.delenv("LQCS_TILE_BITS")
    lq.algorithms.release_caches()
    assert np.array_equal(sim.run_statevector(qc).to_numpy(), a)
    m = W.brickwork(14, 6, seed=3, measure=True)
    r1 = lq.StatevectorSimulator(seed=4).run_registers(m, 500)
    r2 = lq.StatevectorSimulator(seed=4).run_registers(m, 500)
    assert np.array_equal(r1, r2)


def test_adjoint_batched_equals_single(ref):
    pc, _ = W.random_pauli_ansatz(8, 24, seed=8)
    h = W.random_hamiltonian(8, 40, seed=9)
    sets = W.random_parameter_sets(pc.num_parameters(), 10, seed=10)
    e_b, g_b = lq.algorithms.adjoint_gradient(h, pc, sets, max_resident=4)
    for b in range(sets.shape[0]):
        e1, g1 = lq.algorithms.adjoint_gradient(h, pc, sets[b])
        assert abs(e1 - e_b[b]) < 1e-12
        assert np.max(np.abs(g1 - g_b[b])) < 1e-12
    want = ref.parameter_shift_gradient(h, pc, sets[3])
    assert np.max(np.abs(g_b[3] - want)) < 1e-9


def test_errors_match_reference_types():
    sim = lq.StatevectorSimulator()
    qc = lq.QuantumCircuit(2)
    qc.h(0)
    with pytest.raises(ValueError, match="no measurements"):
        sim.run(qc, 10)
    qc.measure_all()
    with pytest.raises(ValueError, match="shots must be >= 1"):
        sim.run(qc, 0)
    r = lq.QuantumCircuit(1, 1)
    r.reset(0)
    with pytest.raises(ValueError, match="Reset is non-deterministic"):
        sim.run_statevector(r)
    noise = lq.NoiseModel()
    noise.add_all_qubit_channel(lq.KrausChannel.depolarizing(0.1))
    with pytest.raises(ValueError, match="stochastic"):
        lq.StatevectorSimulator(noise=noise).run_statevector(lq.QuantumCircuit(1).h(0))
    with pytest.raises(ValueError):
        lq.Statevector(60)
    sv = lq.Statevector(2)
    with pytest.raises(IndexError):
        _ = sv[4]
    with pytest.raises(ValueError, match="length must equal"):
        sv.expectation_value("ZZZ")


@pytest.mark.parametrize("width", [4, 5, 6])
@pytest.mark.parametrize("mma", ["1", "0"])
@pytest.mark.parametrize("n", [7, 14])
def test_wide_blocks_dmma_and_ffma(port, monkeypatch, width, mma, n):
    """Greedy 4..6-qubit blocks (controls included) on the FP64 tensor path
    (mma.sync.m8n8k4.f64, 64 groups per tile: partial tiles at 7 qubits) and on the FFMA
    kernel agree with the oracle."""
    monkeypatch.setenv("LQCS_DENSE_MMA", mma)
    init = W.gaussian_state(n, seed=width)
    qc = random_circuit(n, 80, seed=100 + width, max_controls=3, max_unitary=4)
    want = port.run_statevector(qc, fuse=False, state=init)
    sv = lq.Statevector.from_numpy(init)
    sv.apply(qc, fuse_gates=True, max_fusion_width=width, fusion_mode=1)
    assert np.max(np.abs(sv.to_numpy() - want)) < 1e-12


def test_adjoint_graph_replay_new_parameters(ref, monkeypatch):
    """The batched adjoint captures its launch sequence once per batch shape and replays it:
    replays with new parameters (fixed gates included) equal direct launches bit for bit and
    the reference's parameter-shift gradient."""
    n = 9
    pc = lq.ParametricCircuit(n)
    rng = np.random.default_rng(5)
    for q in range(n):
        pc.h(q)
    for i in range(14):
        a, b = (int(x) for x in rng.permutation(n)[:2])
        pc.cx(a, b)
        pc.ry(a)
        pc.rp("XZ" if i % 2 else "YY", [a, b])
        pc.t(b)
    h = W.random_hamiltonian(n, 30, seed=32)
    sets1 = W.random_parameter_sets(pc.num_parameters(), 6, seed=33)
    sets2 = W.random_parameter_sets(pc.num_parameters(), 6, seed=34)
    e1, g1 = lq.algorithms.adjoint_gradient(h, pc, sets1, max_resident=4)   # captures
    e2, g2 = lq.algorithms.adjoint_gradient(h, pc, sets2, max_resident=4)   # replays
    monkeypatch.setenv("LQCS_GRAPHS", "0")
    e2d, g2d = lq.algorithms.adjoint_gradient(h, pc, sets2, max_resident=4)
    assert np.array_equal(e2, e2d) and np.array_equal(g2, g2d)
    for b in (0, 5):
        want = ref.parameter_shift_gradient(h, pc, sets2[b])
        assert np.max(np.abs(g2[b] - want)) < 1e-9
    assert not np.allclose(g1, g2)


def test_adjoint_multi_ragged_problems(ref, monkeypatch):
    """Problems of 6, 9, 12 and 14 qubits (own ansatz, Hamiltonian and batch each) in one
    call — one captured graph, concurrent branches — equal the one-problem calls bit for
    bit, on the capture and on a replay with new parameters; small problems fall back to
    one-by-one and agree too."""
    probs = []
    for i, (n, b) in enumerate([(6, 3), (9, 5), (12, 2), (14, 4)]):
        pc, _ = W.random_pauli_ansatz(n, 10 + 3 * i, seed=50 + i, max_w=min(8, n))
        h = W.random_hamiltonian(n, 20 + i, seed=60 + i)
        probs.append((h, pc, b))
    for seed in (70, 71):   # capture, then replay
        sets = [W.random_parameter_sets(pc.num_parameters(), b, seed=seed + j)
                for j, (h, pc, b) in enumerate(probs)]
        got = lq.algorithms.adjoint_gradient_multi([(h, pc, s) for (h, pc, b), s in zip(probs, sets)])
        for (h, pc, b), s, (e, g) in zip(probs, sets, got):
            e1, g1 = lq.algorithms.adjoint_gradient(h, pc, s)
            assert np.array_equal(e, e1) and np.array_equal(g, g1)
    want = ref.parameter_shift_gradient(probs[1][0], probs[1][1], sets[1][2])
    assert np.max(np.abs(got[1][1][2] - want)) < 1e-9
    monkeypatch.setenv("LQCS_GRAPHS", "0")
    direct = lq.algorithms.adjoint_gradient_multi([(h, pc, s) for (h, pc, b), s in zip(probs, sets)])
    for (e, g), (e2, g2) in zip(got, direct):
        assert np.array_equal(e, e2) and np.array_equal(g, g2)
    small, _ = W.random_pauli_ansatz(3, 6, seed=9, max_w=3)
    hs = W.random_hamiltonian(3, 5, seed=8)
    ss = W.random_parameter_sets(small.num_parameters(), 2, seed=7)
    (e, g), _ = lq.algorithms.adjoint_gradient_multi([(hs, small, ss), probs[0][:2] + (sets[0],)])
    e1, g1 = lq.algorithms.adjoint_gradient(hs, small, ss)
    assert np.max(np.abs(g - g1)) < 1e-12 and np.max(np.abs(e - e1)) < 1e-12


def test_release_caches_frees_plan_memory(ref):
    import torch
    pc, _ = W.random_pauli_ansatz(16, 20, seed=3)
    h = W.random_hamiltonian(16, 10, seed=4)
    sets = W.random_parameter_sets(pc.num_parameters(), 64, seed=5)
    lq.algorithms.release_caches()
    free0 = torch.cuda.mem_get_info()[0]
    e1, g1 = lq.algorithms.adjoint_gradient(h, pc, sets, max_resident=64)
    held = free0 - torch.cuda.mem_get_info()[0]
    assert held >= 2 * 64 * (16 << 16)           # two resident batches of 64 states
    lq.algorithms.release_caches()
    assert torch.cuda.mem_get_info()[0] - free0 > -(16 << 20)
    e2, g2 = lq.algorithms.adjoint_gradient(h, pc, sets, max_resident=64)   # rebuilt
    assert np.array_equal(e1, e2) and np.array_equal(g1, g2)

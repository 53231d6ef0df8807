"""Batched trajectories (per-shot path with many shots resident on the device).

* Same seed, same uniforms: counts identical to the reference's per-shot semantics
  (oracle/_ref: StatevectorSimulator::run for a noise model, the reference-semantics
  driver for explicit Kraus placements).
* The config-3 cross-check: a 10-qubit noisy brickwork (depolarizing 1e-3 after U3,
  1e-2 on both qubits after CX, amplitude damping 1e-3 per qubit per layer), 1024
  trajectories, total-variation distance to the exact density-matrix distribution compared
  with the TVD of 1024 independent draws from that distribution (seeded bootstrap).
"""
import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import workloads as W

pytestmark = pytest.mark.gpu


def counts_of(regs):
    vals, cnt = np.unique(regs, return_counts=True)
    return {int(v): int(c) for v, c in zip(vals, cnt)}


@pytest.mark.parametrize("resident", [1, 7, 64])
def test_noise_model_counts_identical(ref, resident):
    noise = lq.NoiseModel()
    noise.add_all_qubit_channel(lq.KrausChannel.depolarizing(0.2))
    noise.add_all_qubit_channel(lq.KrausChannel.amplitude_damping(0.15))
    noise.add_all_qubit_channel(lq.KrausChannel.phase_flip(0.1))
    qc = lq.QuantumCircuit(5, 5)
    qc.h(0).cx(0, 1).ry(0.7, 2).cx(2, 3).t(3).cx(3, 4).measure(2, 2).h(2).reset(1).measure_all()
    want = ref.run(qc, 300, 17, noise=noise)
    got = counts_of(lq.StatevectorSimulator(seed=17, noise=noise, max_resident=resident)
                    .run_registers(qc, 300))
    assert got == want


def test_explicit_kraus_placements_identical(ref):
    qc = W.brickwork(6, 4, seed=3, measure=True, noise=(0.05, 0.1, 0.2))
    want = counts_of(ref.trajectories(qc, 256, 21))
    got = counts_of(lq.StatevectorSimulator(seed=21, max_resident=32).run_registers(qc, 256))
    assert got == want


def test_large_batch_trajectories_run():
    qc = W.brickwork(16, 3, seed=4, measure=True, noise=(1e-3, 1e-2, 1e-3))
    regs = lq.StatevectorSimulator(seed=5, max_resident=16).run_registers(qc, 40)
    assert regs.shape == (40,)
    regs2 = lq.StatevectorSimulator(seed=5, max_resident=40).run_registers(qc, 40)
    assert np.array_equal(regs, regs2)


def test_config3_cross_check_tvd(ref):
    n, shots = 10, 1024
    qc = W.brickwork(n, 20, seed=2026, measure=True, noise=(1e-3, 1e-2, 1e-3))
    exact = ref.dm_probabilities(qc)
    exact = exact / exact.sum()
    regs = lq.StatevectorSimulator(seed=99, max_resident=256).run_registers(qc, shots)
    freq = np.bincount(regs.astype(np.int64), minlength=1 << n) / shots
    tvd = 0.5 * np.abs(freq - exact).sum()
    rng = np.random.default_rng(12345)
    boot = []
    for _ in range(200):
        draw = rng.choice(1 << n, size=shots, p=exact)
        boot.append(0.5 * np.abs(np.bincount(draw, minlength=1 << n) / shots - exact).sum())
    assert tvd <= np.quantile(boot, 0.999)
    assert tvd >= np.quantile(boot, 0.001)


# ---- fused batches (n >= 9): fixed-branch noise fused into register tile passes


@pytest.mark.parametrize("resident", [5, 64])
def test_fused_explicit_kraus_counts_identical(ref, resident):
    """Heavy noise: many uncertain amplitude-damping events (cuts) and differing Pauli
    branches per state (noise slots); counts equal the reference's per-shot semantics."""
    qc = W.brickwork(10, 6, seed=8, measure=True, noise=(0.05, 0.1, 0.2))
    want = counts_of(ref.trajectories(qc, 128, 33))
    got = counts_of(lq.StatevectorSimulator(seed=33, max_resident=resident).run_registers(qc, 128))
    assert got == want


def test_fused_trajectories_with_swaps(ref):
    """SWAPs between noisy layers (relabelled inside register passes, per-state noise
    matrices in the same passes): counts equal the reference's per-shot semantics."""
    qc = lq.QuantumCircuit(10, 10)
    qc.compose(W.brickwork(10, 4, seed=9, noise=(0.05, 0.1, 0.2)))
    for i in range(5):
        qc.swap(i, 9 - i)
    qc.swap(0, 3)
    qc.compose(W.brickwork(10, 2, seed=10, noise=(0.05, 0.1, 0.2)))
    qc.measure_all()
    want = counts_of(ref.trajectories(qc, 96, 21))
    got = counts_of(lq.StatevectorSimulator(seed=21, max_resident=32).run_registers(qc, 96))
    assert got == want


def test_fused_trajectories_with_pauli_rotations(ref):
    """Pauli rotations of weight 2..8 between noisy layers run inside the register passes
    (flips on register bits and lanes, Z qubits in and out of the tile) beside the per-state
    noise matrices: counts equal the reference's per-shot semantics."""
    rng = np.random.default_rng(31)
    qc = lq.QuantumCircuit(12, 12)
    qc.compose(W.brickwork(12, 2, seed=11, noise=(0.05, 0.1, 0.2)))
    for _ in range(6):
        w = int(rng.integers(2, 9))
        q = [int(x) for x in rng.permutation(12)[:w]]
        qc.rp(float(rng.uniform(-np.pi, np.pi)),
              "".join("XYZ"[int(rng.integers(3))] for _ in range(w)), q)
    qc.compose(W.brickwork(12, 2, seed=12, noise=(0.05, 0.1, 0.2)))
    qc.measure_all()
    want = counts_of(ref.trajectories(qc, 96, 23))
    got = counts_of(lq.StatevectorSimulator(seed=23, max_resident=32).run_registers(qc, 96))
    assert got == want


def test_fused_noise_model_counts_identical(ref):
    noise = lq.NoiseModel()
    noise.add_all_qubit_channel(lq.KrausChannel.depolarizing(0.05))
    noise.add_all_qubit_channel(lq.KrausChannel.amplitude_damping(0.1))
    qc = W.brickwork(9, 4, seed=12, measure=True)
    want = ref.run(qc, 96, 5, noise=noise)
    got = counts_of(lq.StatevectorSimulator(seed=5, noise=noise, max_resident=32)
                    .run_registers(qc, 96))
    assert got == want


def test_fused_matches_unfused_at_config3_rates(monkeypatch):
    """Config-3 noise rates at 14 qubits: the fused driver and the gate-by-gate driver give
    the same registers for the same seed."""
    qc = W.brickwork(14, 8, seed=21, measure=True, noise=(1e-3, 1e-2, 1e-3))
    fused = lq.StatevectorSimulator(seed=7, max_resident=32).run_registers(qc, 96)
    monkeypatch.setenv("LQCS_TRAJ_FUSED", "0")
    plain = lq.StatevectorSimulator(seed=7, max_resident=32).run_registers(qc, 96)
    assert np.array_equal(fused, plain)


def test_fused_terminal_measures_any_order(ref):
    """Terminal measurements of a qubit subset in arbitrary order, into permuted clbits, after
    a mid-circuit measurement and reset: counts equal the reference's."""
    qc = W.brickwork(11, 3, seed=40, noise=(0.02, 0.05, 0.3))
    full = lq.QuantumCircuit(11, 6)
    full.compose(qc)
    full.measure(4, 5).reset(4).h(4).cx(4, 9)
    for q, c in ((7, 0), (2, 3), (9, 1), (0, 4), (10, 2)):
        full.measure(q, c)
    want = counts_of(ref.trajectories(full, 160, 71))
    got = counts_of(lq.StatevectorSimulator(seed=71, max_resident=40).run_registers(full, 160))
    assert got == want


@pytest.mark.parametrize("n", [6, 12])
def test_shot_ranges_concatenate_to_one_run(n):
    """Shots [0, 37) and [37, 100) run separately (shot_offset) give the registers of one
    100-shot run: what sharded_run_registers relies on (gate-by-gate driver at 6 qubits,
    fused driver at 12; sampling and density-matrix paths too)."""
    qc = W.brickwork(n, 4, seed=n, measure=True, noise=(0.02, 0.05, 0.2))
    sim = lq.StatevectorSimulator(seed=123, max_resident=16)
    full = sim.run_registers(qc, 100)
    parts = np.concatenate([sim.run_registers(qc, 37), sim.run_registers(qc, 63, shot_offset=37)])
    assert np.array_equal(full, parts)
    clean = W.brickwork(n, 4, seed=n, measure=True)
    full = sim.run_registers(clean, 100)
    parts = np.concatenate([sim.run_registers(clean, 50, shot_offset=0),
                            sim.run_registers(clean, 50, shot_offset=50)])
    assert np.array_equal(full, parts)
    dm = lq.DensityMatrixSimulator(seed=9)
    small = W.brickwork(6, 3, seed=1, measure=True, noise=(0.02, 0.05, 0.2))
    full = dm.run_registers(small, 80)
    parts = np.concatenate([dm.run_registers(small, 30), dm.run_registers(small, 50, shot_offset=30)])
    assert np.array_equal(full, parts)


@pytest.mark.parametrize("n", [6, 13])
def test_noiseless_per_shot_shares_one_state(ref, n):
    """Noiseless circuits that the reference runs per shot because its one-qubit fusion
    leaves gates between the final measurements (a Measure flushes only its own qubit):
    one state, one table of the measured qubits, per-shot walks — counts identical to the
    reference's, with measurements in any order and any clbit mapping, gates on unmeasured
    qubits after the measurements, and a unitary that has to stay between them."""
    rng = np.random.default_rng(n)
    for trial in range(4):
        qc = lq.QuantumCircuit(n, n)
        qc.compose(W.brickwork(n, 3, seed=50 + trial))
        for q in range(n):
            qc.u(*(float(x) for x in rng.uniform(0, 6.3, 3)), q)
        order = [int(x) for x in rng.permutation(n)]
        clbits = [int(x) for x in rng.permutation(n)]
        measured = order[: n - 2]
        for k, q in enumerate(measured):
            qc.measure(q, clbits[k])
            if trial == 3 and k == 1:
                qc.cx(measured[0], measured[2])   # touches a measured qubit: stays per-shot
        qc.h(order[-1])                           # after every measurement: no effect
        want = ref.run(qc, 500, 100 + trial)
        got = counts_of(lq.StatevectorSimulator(seed=100 + trial).run_registers(qc, 500))
        assert got == want

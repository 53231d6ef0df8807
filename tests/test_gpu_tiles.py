"""GPU parity of the tile passes (fusion_mode 4, the default from 12 qubits) — register
kernel and shared-memory kernel — and of the greedy dense-block path (fusion_mode 1)
against the oracle, for every gate type and several tile shapes."""
import os

import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import workloads as W

from helpers import random_circuit

pytestmark = pytest.mark.gpu
TOL = 1e-12
TILE = 4
GREEDY = 1


@pytest.fixture
def tile_env():
    keys = ("LQCS_TILE_BITS", "LQCS_TILE_LOW", "LQCS_TILE_INNER", "LQCS_TILE_REG", "LQCS_REG_MMA")
    saved = {k: os.environ.get(k) for k in keys}

    def set_cfg(m, low, inner, reg=1, mma=0):
        os.environ["LQCS_TILE_BITS"] = str(m)
        os.environ["LQCS_TILE_LOW"] = str(low)
        os.environ["LQCS_TILE_INNER"] = str(inner)
        os.environ["LQCS_TILE_REG"] = str(reg)
        os.environ["LQCS_REG_MMA"] = str(mma)

    yield set_cfg
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def run(qc, mode, init=None):
    if init is None:
        return lq.StatevectorSimulator(fusion_mode=mode).run_statevector(qc).to_numpy()
    sv = lq.Statevector.from_numpy(init)
    sv.apply(qc, fuse_gates=True, fusion_mode=mode)
    return sv.to_numpy()


def kernel_kinds(qc):
    """Profile kinds of a tile-mode program's device ops (6 shared-memory, 7 register pass)."""
    prog = lq.simulator.CompiledCircuit(qc, True, 0, TILE)
    sv = lq.Statevector(qc.num_qubits())
    return [r["kind"] for r in prog.profile(sv)]


@pytest.mark.parametrize("reg", [1, 0])
@pytest.mark.parametrize("n", [6, 8, 11, 13])
@pytest.mark.parametrize("cfg", [(12, 5, 2), (11, 5, 1), (13, 5, 3), (10, 6, 4), (12, 4, 2),
                                 (9, 5, 2)])
def test_tile_passes_every_gate_type(port, tile_env, n, cfg, reg):
    tile_env(*cfg, reg)
    init = W.gaussian_state(n, seed=n + cfg[0])
    qc = random_circuit(n, 90, seed=31 * n + cfg[2], max_controls=4, max_unitary=4)
    want = port.run_statevector(qc, fuse=False, state=init)
    got = run(qc, TILE, init)
    assert np.max(np.abs(got - want)) < TOL


@pytest.mark.parametrize("reg", [1, 0])
@pytest.mark.parametrize("inner", [1, 2, 3, 4])
def test_tile_brickwork_and_qft_vs_reference(ref, tile_env, inner, reg):
    tile_env(12, 5, inner, reg)
    qc = W.brickwork(18, 12, seed=77)
    want = ref.run_statevector(qc, fuse=True)
    assert np.max(np.abs(run(qc, TILE) - want)) < TOL
    init = W.gaussian_state(16, seed=4)
    q = lq.algorithms.qft(16)
    want = ref.evolve_from(q, init)
    assert np.max(np.abs(run(q, TILE, init) - want)) < TOL


@pytest.mark.parametrize("reg", [1, 0])
@pytest.mark.parametrize("n", [13, 16])
def test_diagonal_runs_and_gated_phases(port, tile_env, n, reg):
    """Runs of phases and diagonals between a few dense gates: merged into tables of up to 6
    tile bits, with phases controlled from outside the tile as per-tile terms (register
    passes) — results must not depend on the merge."""
    tile_env(12, 5, 2, reg)
    rng = np.random.default_rng(n + 10 * reg)
    qc = lq.QuantumCircuit(n)
    for step in range(260):
        a, b, c = (int(x) for x in rng.permutation(n)[:3])
        k = int(rng.integers(9))
        if step % 23 == 0 or k == 0:
            qc.h(a)
        elif k == 1:
            qc.cp(float(rng.uniform(0, 6.3)), a, b)
        elif k == 2:
            qc.rzz(float(rng.uniform(0, 6.3)), a, b)
        elif k == 3:
            qc.mcp(float(rng.uniform(0, 6.3)), [a, b], c)
        elif k == 4:
            qc.cz(a, b)
        elif k == 5:
            qc.crz(float(rng.uniform(0, 6.3)), a, b)
        elif k == 6:
            qc.t(a)
        elif k == 7:
            qc.rz(float(rng.uniform(0, 6.3)), a)
        else:
            qc.u(*(float(x) for x in rng.uniform(0, 6.3, 3)), a)
    init = W.gaussian_state(n, seed=n)
    want = port.run_statevector(qc, fuse=False, state=init)
    assert np.max(np.abs(run(qc, TILE, init) - want)) < TOL
    # the QFT's phase ladders: every pass holds long runs of gated phases
    q = lq.algorithms.qft(n)
    want = port.run_statevector(q, fuse=False, state=init)
    assert np.max(np.abs(run(q, TILE, init) - want)) < TOL


@pytest.mark.parametrize("n,k", [(24, 20), (24, 16), (22, 19)])
def test_partial_inverse_qft_on_larger_state(n, k):
    """The inverse QFT of k of n qubits through register tile passes equals gate-by-gate
    application (a missing barrier between tiles once made (24, 20) wrong by ~1e-3)."""
    init = W.gaussian_state(n, seed=n + k)
    qc = lq.QuantumCircuit(n)
    qc.compose(lq.algorithms.qft_inverse(k))
    a = lq.Statevector.from_numpy(init)
    a.apply(qc, fuse_gates=False)
    for _ in range(2):
        b = lq.Statevector.from_numpy(init)
        b.apply(qc, fuse_gates=True, fusion_mode=TILE)
        assert np.max(np.abs(a.to_numpy() - b.to_numpy())) < TOL


@pytest.mark.parametrize("n", [12, 15])
def test_relabelled_swaps(port, tile_env, n):
    """SWAPs of two tile qubits become relabellings in register passes (the store writes
    each tile bit to its qubit's new place): chains of swaps between low and high qubits,
    interleaved with dense and diagonal gates, and a full qubit reversal."""
    tile_env(12, 5, 2, 1)
    rng = np.random.default_rng(n)
    qc = lq.QuantumCircuit(n)
    for step in range(150):
        a, b = (int(x) for x in rng.permutation(n)[:2])
        k = int(rng.integers(5))
        if k < 2:
            qc.swap(a, b)
        elif k == 2:
            qc.u(*(float(x) for x in rng.uniform(0, 6.3, 3)), a)
        elif k == 3:
            qc.cx(a, b)
        else:
            qc.cp(float(rng.uniform(0, 6.3)), a, b)
    for i in range(n // 2):
        qc.swap(i, n - 1 - i)
    init = W.gaussian_state(n, seed=n + 1)
    want = port.run_statevector(qc, fuse=False, state=init)
    assert np.max(np.abs(run(qc, TILE, init) - want)) < TOL


@pytest.mark.parametrize("reg", [1, 0])
def test_tile_barrier_and_wide_gates(port, tile_env, reg):
    tile_env(12, 5, 2, reg)
    n = 14
    init = W.gaussian_state(n, seed=8)
    qc = random_circuit(n, 40, seed=5)
    qc.barrier()
    qc.rp(0.3, "XYZXYZX", [0, 3, 5, 7, 9, 11, 13])    # wider than a tile op: runs on its own
    qc.mcx([0, 1, 2, 3, 4, 5, 6, 7, 8], 13)             # too many controls for a tile op
    qc.permutation(list(np.random.default_rng(1).permutation(32)), [1, 6, 8, 10, 12])
    qc.compose(random_circuit(n, 40, seed=6))
    want = port.run_statevector(qc, fuse=False, state=init)
    assert np.max(np.abs(run(qc, TILE, init) - want)) < TOL


@pytest.mark.parametrize("n", [12, 15])
def test_greedy_blocks_at_tile_sizes(port, n):
    init = W.gaussian_state(n, seed=n)
    qc = random_circuit(n, 70, seed=n)
    want = port.run_statevector(qc, fuse=False, state=init)
    for width in (2, 4, 6):
        sv = lq.Statevector.from_numpy(init)
        sv.apply(qc, fuse_gates=True, max_fusion_width=width, fusion_mode=GREEDY)
        assert np.max(np.abs(sv.to_numpy() - want)) < TOL


@pytest.mark.parametrize("reg,mma", [(1, 0), (0, 0), (1, 1)])
def test_tile_batch_of_states(port, tile_env, reg, mma):
    """Tile passes walk a batch of states (gridDim.y), register passes on either path."""
    tile_env(12, 5, 2, reg, mma)
    from litequantumcomputingsimulator_b200 import _native as N
    import ctypes as C
    n, batch = 13, 3
    qc = random_circuit(n, 50, seed=9)
    inits = [W.gaussian_state(n, seed=s) for s in range(batch)]
    h = N.StatePtr()
    N.call("lqcs_state_create_batch", n, batch, None, C.byref(h))
    flat = np.ascontiguousarray(np.concatenate(inits))
    N.call("lqcs_state_load", h, flat.ctypes.data, flat.size)
    prog = lq.simulator.CompiledCircuit(qc, True, 0, TILE)
    N.call("lqcs_program_apply", h, prog._h)
    out = np.empty_like(flat)
    N.call("lqcs_state_store", h, out.ctypes.data, out.size)
    N.call("lqcs_state_destroy", h)
    for b in range(batch):
        want = port.run_statevector(qc, fuse=False, state=inits[b])
        assert np.max(np.abs(out[b << n:(b + 1) << n] - want)) < TOL


@pytest.mark.parametrize("m", [9, 10, 11, 12, 13])
def test_register_kernel_runs_the_passes(ref, tile_env, m):
    """With inner fusion <= 3 every pass of a brickwork fits the register kernel; with the
    register kernel off they all run in shared memory; both agree with the reference."""
    qc = W.brickwork(16, 10, seed=3)
    want = ref.run_statevector(qc, fuse=True)
    tile_env(m, 5, 2, 1)
    kinds = kernel_kinds(qc)
    assert kinds and all(k == 7 for k in kinds)
    assert np.max(np.abs(run(qc, TILE) - want)) < TOL
    tile_env(m, 5, 2, 0)
    assert all(k == 6 for k in kernel_kinds(qc))
    assert np.max(np.abs(run(qc, TILE) - want)) < TOL


def test_register_kernel_controls_phases_and_diagonals(port, tile_env):
    """Controls and phase bits on register bits, thread bits and out-of-tile qubits; diagonal
    blocks; X gates on register bits (swap path)."""
    tile_env(12, 5, 2, 1)
    n = 16
    rng = np.random.default_rng(12)
    qc = lq.QuantumCircuit(n)
    for _ in range(160):
        kind = int(rng.integers(7))
        q = [int(x) for x in rng.permutation(n)[:4]]
        if kind == 0:
            qc.u(*rng.uniform(0, 6.3, 3), q[0])
        elif kind == 1:
            qc.cx(q[0], q[1])
        elif kind == 2:
            qc.ccx(q[0], q[1], q[2])
        elif kind == 3:
            qc.cp(float(rng.uniform(0, 6.3)), q[0], q[1])
        elif kind == 4:
            qc.rzz(float(rng.uniform(0, 6.3)), q[0], q[1])
        elif kind == 5:
            qc.x(q[0])
        else:
            qc.cry(float(rng.uniform(0, 6.3)), q[0], q[1])
    init = W.gaussian_state(n, seed=2)
    want = port.run_statevector(qc, fuse=False, state=init)
    assert 7 in kernel_kinds(qc)
    assert np.max(np.abs(run(qc, TILE, init) - want)) < TOL


def test_autotune_picks_a_timed_plan_and_mode5_uses_it(port):
    """lqcs_autotune times every candidate plan; fusion_mode 5 compiles the fastest one and
    gives the oracle's amplitudes."""
    n = 16
    qc = W.brickwork(n, 6, seed=19)
    res = lq.simulator.autotune(qc)
    assert len(res) >= 5 and sum(r["chosen"] for r in res) == 1
    best = min(res, key=lambda r: r["ms"])
    assert best["chosen"] and all(r["ms"] > 0 for r in res)
    want = port.run_statevector(qc, fuse=False)
    prog = lq.simulator.CompiledCircuit(qc, True, 0, 5)
    sv = lq.Statevector(n)
    prog.apply(sv)
    assert np.max(np.abs(sv.to_numpy() - want)) < TOL
    assert prog.n_ops == best["n_ops"]


@pytest.mark.parametrize("m", [9, 11, 12, 13])
def test_register_passes_on_the_tensor_path(port, ref, tile_env, m):
    """LQCS_REG_MMA=1: one- and two-qubit blocks of register passes on mma.sync.m8n8k4.f64
    (their targets on lanes 0 and 1) — every gate type with controls, the brickwork against
    the reference, QFT on a Gaussian state, and a batch of states."""
    tile_env(m, 5, 2, 1, 1)
    for n, seed in ((13, 3), (16, 4)):
        init = W.gaussian_state(n, seed=seed)
        qc = random_circuit(n, 120, seed=seed, max_controls=4, max_unitary=3)
        want = port.run_statevector(qc, fuse=False, state=init)
        assert np.max(np.abs(run(qc, TILE, init) - want)) < TOL
    qc = W.brickwork(18, 12, seed=77)
    assert all(k == 7 for k in kernel_kinds(qc))
    assert np.max(np.abs(run(qc, TILE) - ref.run_statevector(qc, fuse=True))) < TOL
    init = W.gaussian_state(16, seed=5)
    q = lq.algorithms.qft(16)
    assert np.max(np.abs(run(q, TILE, init) - ref.evolve_from(q, init))) < TOL


def _pauli_circuit(n, n_gates, seed):
    rng = np.random.default_rng(seed)
    qc = lq.QuantumCircuit(n)
    for _ in range(n_gates):
        r = float(rng.uniform())
        q = [int(x) for x in rng.permutation(n)]
        if r < 0.4:
            qc.u(*(float(x) for x in rng.uniform(0, 2 * np.pi, 3)), q[0])
        elif r < 0.55:
            qc.cx(q[0], q[1])
        elif r < 0.6:
            qc.cp(float(rng.uniform(0, 6.3)), q[0], q[1])
        else:
            w = int(rng.integers(1, min(9, n + 1)))
            qc.rp(float(rng.uniform(-np.pi, np.pi)),
                  "".join("XYZ"[int(rng.integers(3))] for _ in range(w)), q[:w])
    return qc


@pytest.fixture
def pauli_env():
    saved = os.environ.get("LQCS_TILE_PAULI")
    yield lambda v: os.environ.__setitem__("LQCS_TILE_PAULI", str(v))
    if saved is None:
        os.environ.pop("LQCS_TILE_PAULI", None)
    else:
        os.environ["LQCS_TILE_PAULI"] = saved


@pytest.mark.parametrize("n", [13, 16, 20])
@pytest.mark.parametrize("cfg", [(12, 5, 2, 1, 0), (11, 5, 2, 1, 0), (12, 5, 2, 1, 1), (12, 5, 4, 1, 0)],
                         ids=["m12", "m11", "m12_tensor", "inner4_split"])
def test_native_pauli_rotations_in_register_passes(port, tile_env, pauli_env, n, cfg):
    """Pauli rotations of weight 1..8 whose X/Y qubits (at most four) are tile qubits run
    inside register passes — Z qubits inside or outside the tile act through parities; the
    others run on their own.  inner4_split: 4-qubit blocks keep passes off the register
    kernel, so the shared-memory passes split at each rotation.  Both against the oracle and
    against LQCS_TILE_PAULI=0 (rotations of at most four qubits as dense blocks)."""
    tile_env(*cfg)
    init = W.gaussian_state(n, seed=n + 1)
    qc = _pauli_circuit(n, 160, seed=3 * n + cfg[0])
    want = port.run_statevector(qc, fuse=False, state=init)
    pauli_env(1)
    got = run(qc, TILE, init)
    assert np.max(np.abs(got - want)) < TOL
    if cfg[2] <= 3:
        assert 7 in kernel_kinds(qc)
    pauli_env(0)
    assert np.max(np.abs(run(qc, TILE, init) - want)) < TOL


def test_random_mix_24q_native_rotations_equal_gate_by_gate():
    """The cost-model workload's gate mix (10 % Pauli rotations of weight 2..8) at 24 qubits,
    default path, against gate-by-gate application on the device."""
    qc = W.random_mix_circuit(24, 12, seed=5)
    init = W.gaussian_state(24, seed=24)
    a = lq.Statevector.from_numpy(init)
    lq.simulator.CompiledCircuit(qc, True, 0, 0).apply(a)
    b = lq.Statevector.from_numpy(init)
    lq.simulator.CompiledCircuit(qc, True, 0, 3).apply(b)
    assert float(np.max(np.abs(a.to_numpy() - b.to_numpy()))) < TOL


_SIGMA = {"I": np.eye(2), "X": np.array([[0, 1], [1, 0]], dtype=complex),
          "Y": np.array([[0, -1j], [1j, 0]]), "Z": np.diag([1.0, -1.0]).astype(complex)}


def _rotation_matrix(theta, pauli):
    """exp(-i theta/2 P), matrix bit j <-> qubits[j], P's character pauli[k-1-j] on it."""
    p = np.array([[1.0 + 0j]])
    for ch in pauli:          # leftmost character = most significant matrix bit
        p = np.kron(p, _SIGMA[ch])
    return np.cos(theta / 2) * np.eye(p.shape[0]) - 1j * np.sin(theta / 2) * p


def test_native_rotations_match_dense_matrices_and_named_gates():
    """Known answers of the reference's Pauli-rotation tests (tests/test_pauli_rotation.cpp:
    rp("XX"/"YY"/"ZZ") equal RXX/RYY/RZZ, the kernel equals the dense matrix for long
    strings) at 16 qubits, where the rotations run inside register passes: each circuit of
    rotations against the same circuit with the rotations as explicit unitaries or named
    gates, from one Gaussian state, within 1e-12."""
    n = 16
    rng = np.random.default_rng(41)
    init = W.gaussian_state(n, seed=41)
    rot = lq.QuantumCircuit(n)
    dense = lq.QuantumCircuit(n)
    for _ in range(40):
        w = int(rng.integers(1, 7))
        qs = [int(x) for x in rng.permutation(n)[:w]]
        pauli = "".join("XYZ"[int(rng.integers(3))] for _ in range(w))
        th = float(rng.uniform(-np.pi, np.pi))
        a = int(rng.integers(n))
        rot.h(a).rp(th, pauli, qs)
        dense.h(a).unitary(_rotation_matrix(th, pauli), qs)
    got = run(rot, TILE, init)
    assert 7 in kernel_kinds(rot)
    assert np.max(np.abs(got - run(dense, GREEDY, init))) < TOL
    named = lq.QuantumCircuit(n)
    as_rp = lq.QuantumCircuit(n)
    for i in range(30):
        a, b = (int(x) for x in rng.permutation(n)[:2])
        th = float(rng.uniform(-np.pi, np.pi))
        kind = i % 3
        named.h(a)
        as_rp.h(a)
        getattr(named, ("rxx", "ryy", "rzz")[kind])(th, a, b)
        as_rp.rp(th, ("XX", "YY", "ZZ")[kind], [a, b])
    assert np.max(np.abs(run(as_rp, TILE, init) - run(named, TILE, init))) < TOL

"""Host emulation of the register tile kernel (lqcs_debug_emulate_register_passes): the
records the planner lowers a circuit into are executed thread by thread on the CPU, as
k_regtile and its double-buffered form execute them, and every shared-memory access is
checked against the CUDA barrier model.  No GPU.

* Values: brickwork, QFT, partial inverse QFT and random circuits of the gate types that
  run inside register passes match the oracle within 1e-12, out of place, with every
  amplitude stored exactly once by the tile that loaded it — with two-qubit blocks on the
  FP64 tensor path (the lane pair, emulated as the warp's mma.sync computes them) and on
  register bits (LQCS_REG_MMA=0).
* Races: none in the kernels as launched (a barrier between tiles only in passes whose last
  layout has other warp bits than the first — elsewhere each warp keeps its own
  shared-memory slots across the tile boundary; the double-buffered kernel), and many when
  that barrier is dropped from passes that need it — the check is sensitive.
* In place: a pass that relabels tile bits (SWAPs of two tile qubits) stores amplitudes to
  places other warps load.  Without a barrier between the tile's loads and its stores a fast
  warp can overwrite an amplitude before a slow warp has read it; this made QFT(n >= 24)
  wrong by ~1e-4..1e-3 on the device when two CTAs shared an SM.  The kernel adds that
  barrier where no remap or table barrier provides it; the check finds the hazard without it.
"""
import ctypes as C

import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import _native as N
from litequantumcomputingsimulator_b200 import workloads as W

TOL = 1e-12
BARRIER, NONE, PLANNED, PIPE = 1, 0, 2, 3   # PLANNED: the barriers k_regtile runs with
NO_LOAD_BARRIER = 8


def emulate(qc, mode, state=None, grid=296, race_ctas=4):
    arr, cnt, _keep = qc.c_instructions()
    passes, races = C.c_uint64(0), C.c_uint64(0)
    report = C.create_string_buffer(512)
    st = None if state is None else np.ascontiguousarray(np.array(state, dtype=np.complex128))
    N.call("lqcs_debug_emulate_register_passes", qc.num_qubits(), arr, cnt, grid, mode,
           st.ctypes.data if st is not None else None, race_ctas, C.byref(passes), C.byref(races),
           report, 512)
    return st, passes.value, races.value, report.value.decode()


def tile_circuit(n, n_gates, seed):
    rng = np.random.default_rng(seed)
    qc = lq.QuantumCircuit(n)
    for _ in range(n_gates):
        a, b, c = (int(x) for x in rng.permutation(n)[:3])
        ang = float(rng.uniform(-np.pi, np.pi))
        k = int(rng.integers(12))
        if k == 0:
            qc.h(a)
        elif k == 1:
            qc.u(ang, 0.3 * ang, -ang, a)
        elif k == 2:
            qc.cx(a, b)
        elif k == 3:
            qc.cp(ang, a, b)
        elif k == 4:
            qc.rzz(ang, a, b)
        elif k == 5:
            qc.swap(a, b)
        elif k == 6:
            qc.ccx(a, b, c)
        elif k == 7:
            qc.mcp(ang, [a, b], c)
        elif k == 8:
            qc.t(a)
        elif k == 9:
            qc.crx(ang, a, b)
        elif k == 10:
            qc.iswap(a, b)
        else:
            qc.rxx(ang, a, b)
    return qc


def pauli_circuit(n, n_gates, seed, max_flips=4):
    """U3, CX and Pauli rotations of weight 2..8 on random qubits (X/Y/Z uniform, at most
    max_flips X/Y)."""
    rng = np.random.default_rng(seed)
    qc = lq.QuantumCircuit(n)
    for _ in range(n_gates):
        r = float(rng.uniform())
        q = [int(x) for x in rng.permutation(n)]
        if r < 0.4:
            qc.u(*(float(x) for x in rng.uniform(0, 2 * np.pi, 3)), q[0])
        elif r < 0.6:
            qc.cx(q[0], q[1])
        else:
            w = int(rng.integers(2, 9))
            chars = ["XYZ"[int(rng.integers(3))] for _ in range(w)]
            flips = [i for i, ch in enumerate(chars) if ch != "Z"]
            for i in flips[max_flips:]:
                chars[i] = "Z"
            qc.rp(float(rng.uniform(-np.pi, np.pi)), "".join(chars), q[:w])
    return qc


def circuits():
    yield "brickwork14", W.brickwork(14, 8, seed=3)
    yield "brickwork17", W.brickwork(17, 6, seed=4)
    q = lq.QuantumCircuit(16)
    q.compose(lq.algorithms.qft_inverse(14))
    yield "iqft16of14", q
    yield "qft15", lq.algorithms.qft(15)
    yield "random13", tile_circuit(13, 150, seed=5)
    yield "random16", tile_circuit(16, 200, seed=6)
    yield "pauli14", pauli_circuit(14, 120, seed=7)
    yield "pauli18", pauli_circuit(18, 150, seed=8)
    yield "pauli16_lanes", pauli_circuit(16, 150, seed=9, max_flips=8)


@pytest.mark.parametrize("mma", ["1", "0"], ids=["tensor_path", "fma_path"])
@pytest.mark.parametrize("mode", [PLANNED, BARRIER, PIPE])
@pytest.mark.parametrize("name,qc", list(circuits()), ids=[c[0] for c in circuits()])
def test_emulated_passes_match_oracle(port, monkeypatch, name, qc, mode, mma):
    monkeypatch.setenv("LQCS_REG_MMA", mma)
    n = qc.num_qubits()
    init = W.gaussian_state(n, seed=n)
    got, passes, races, report = emulate(qc, mode, init)
    want = port.run_statevector(qc, fuse=False, state=init)
    assert passes >= 1
    assert races == 0, report
    assert np.max(np.abs(got - want)) < TOL


@pytest.mark.parametrize("tile_bits", ["11", "12"])
def test_double_buffered_tile_sizes(port, monkeypatch, tile_bits):
    monkeypatch.setenv("LQCS_TILE_BITS", tile_bits)
    qc = W.brickwork(15, 8, seed=9)
    init = W.gaussian_state(15, seed=2)
    got, _passes, races, report = emulate(qc, PIPE, init, grid=444)
    assert races == 0, report
    assert np.max(np.abs(got - port.run_statevector(qc, fuse=False, state=init))) < TOL


@pytest.mark.parametrize("n,k", [(24, 20), (24, 16), (22, 19)])
def test_partial_inverse_qft_barrier_model(n, k):
    """The passes of the inverse QFT of k of n qubits (no remap changes the warp bits) are
    race-free even without a barrier between tiles."""
    qc = lq.QuantumCircuit(n)
    qc.compose(lq.algorithms.qft_inverse(k))
    for mode in (BARRIER, PLANNED, PIPE):
        _st, _p, races, report = emulate(qc, mode, race_ctas=8)
        assert races == 0, (mode, report)


@pytest.mark.parametrize("mma,n,seed", [("1", 23, 11), ("0", 22, 2025)],
                         ids=["tensor_path", "fma_path"])
def test_race_check_is_sensitive(monkeypatch, mma, n, seed):
    """Passes whose last layout has other warp bits than the first need the barrier between
    tiles: without it the check must report races; with it (or as planned), none.  Both
    planners: two-qubit blocks on the lane pair (tensor path) and on register bits."""
    monkeypatch.setenv("LQCS_REG_MMA", mma)
    qc = W.brickwork(n, 10, seed=seed)
    _st, _p, races, report = emulate(qc, NONE, race_ctas=2)
    assert races > 0 and "races with" in report
    for mode in (PLANNED, BARRIER, PIPE):
        assert emulate(qc, mode, race_ctas=2)[2] == 0


@pytest.mark.parametrize("n", [18, 20])
def test_relabelled_store_needs_the_load_barrier(port, n):
    """QFT(n) ends with qubit-reversal SWAPs, relabelled in its last pass: with the pass's
    load barrier no store can overtake another thread's load; without it the check reports
    the hazard (values of the out-of-place emulation are right either way)."""
    qc = lq.algorithms.qft(n)
    init = W.gaussian_state(n, seed=n + 3)
    want = port.run_statevector(qc, fuse=False, state=init)
    got, _p, races, report = emulate(qc, PLANNED, init)
    assert races == 0, report
    assert np.max(np.abs(got - want)) < TOL
    _got, _p, races, report = emulate(qc, PLANNED + NO_LOAD_BARRIER, init)
    assert races > 0 and "may overtake its load" in report

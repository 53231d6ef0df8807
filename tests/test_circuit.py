"""Circuit IR: build-time validation with the reference's rules, messages and exception
types (src/circuit/quantum_circuit.cpp, src/circuit/parametric_circuit.cpp), and the
pylqcs fluent API (tests/python/test_bindings.py of the reference project)."""
import math

import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq


def test_fluent_chain_depth_repr():
    qc = lq.QuantumCircuit(2, 2)
    qc.h(0).cx(0, 1).measure_all()
    assert qc.num_qubits() == 2 and qc.num_clbits() == 2
    assert qc.depth() == 3
    assert "instructions=4" in repr(qc)


def test_validation_errors():
    with pytest.raises(ValueError, match="num_qubits must be >= 1"):
        lq.QuantumCircuit(0)
    qc = lq.QuantumCircuit(2)
    with pytest.raises(IndexError, match="qubit index 5 out of range"):
        qc.h(5)
    with pytest.raises(ValueError, match="duplicate qubit"):
        qc.cx(1, 1)
    with pytest.raises(ValueError, match="not unitary"):
        qc.unitary(np.array([[1, 1], [0, 1]], dtype=complex), [0])
    with pytest.raises(ValueError, match="matrix size"):
        qc.unitary(np.eye(4), [0])
    with pytest.raises(ValueError, match="not a bijection"):
        qc.permutation([0, 0, 1, 2], [0, 1])
    with pytest.raises(ValueError, match="table size"):
        qc.permutation([0, 1], [0, 1])
    with pytest.raises(ValueError, match="only I/X/Y/Z"):
        qc.rp(0.1, "XA", [0, 1])
    with pytest.raises(ValueError, match="non-empty"):
        qc.rp(0.1, "X", [0, 1])
    with pytest.raises(IndexError, match="clbit index"):
        qc.measure(0, 0)
    with pytest.raises(ValueError, match="at least one control"):
        qc.mcx([], 0)


def test_measure_all_extends_clbits():
    qc = lq.QuantumCircuit(3, 1)
    qc.measure_all()
    assert qc.num_clbits() == 3 and qc.num_instructions() == 3


def test_compose_inverse_power():
    a = lq.QuantumCircuit(2)
    a.h(0).s(1).u(0.1, 0.2, 0.3, 0).iswap(0, 1).sx(1)
    inv = a.inverse()
    assert [i.gate.name() for i in inv.instructions()] == ["unitary", "unitary", "u", "sdg", "h"]
    assert inv.instructions()[2].gate.params == [-0.1, -0.3, -0.2]
    big = lq.QuantumCircuit(4)
    big.compose(a, [3, 1])
    assert [i.qubits for i in big.instructions()][0] == [3]
    assert a.power(3).num_instructions() == 15
    assert a.power(-1).num_instructions() == 5
    m = lq.QuantumCircuit(1, 1)
    m.measure(0, 0)
    with pytest.raises(ValueError, match="non-unitary"):
        m.inverse()


def test_gate_names_and_matrices():
    assert lq.Gate(lq.GateType.X, [], 1).name() == "cx"
    assert lq.Gate(lq.GateType.X, [], 2).name() == "ccx"
    assert lq.Gate(lq.GateType.X, [], 3).name() == "mcx"
    cx = lq.Gate(lq.GateType.X, [], 1).matrix()
    # controls in the low local bit: |c=1,t=0> = 1 <-> |c=1,t=1> = 3
    assert np.array_equal(cx.real, np.array([[1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0], [0, 1, 0, 0]]))
    for t in (lq.GateType.H, lq.GateType.SX, lq.GateType.T):
        m = lq.Gate(t).base_matrix()
        assert np.allclose(m @ m.conj().T, np.eye(2), atol=1e-12)
    u = lq.Gate(lq.GateType.U, [0.4, 1.5, 2.6])
    assert np.allclose(u.base_matrix() @ u.inverse().base_matrix(), np.eye(2), atol=1e-12)


def test_parametric_circuit_bind():
    pc = lq.ParametricCircuit(2)
    pc.x(0)
    assert pc.ry(1) == 0
    pc.cx(1, 0)
    assert pc.rp("XZ", [0, 1]) == 1
    assert pc.num_parameters() == 2
    qc = pc.bind([0.3, -0.2])
    assert qc.instructions()[1].gate.params == [0.3]
    assert qc.instructions()[3].gate.params == [-0.2]
    assert qc.instructions()[3].gate.pauli == "XZ"
    with pytest.raises(ValueError, match="number of values"):
        pc.bind([0.1])


def test_kraus_channels_completeness():
    for ch in (lq.KrausChannel.depolarizing(0.1), lq.KrausChannel.amplitude_damping(0.3),
               lq.KrausChannel.phase_damping(0.2), lq.KrausChannel.bit_flip(0.4),
               lq.KrausChannel.phase_flip(0.5)):
        s = sum(np.conj(k.T) @ k for k in ch.as_array())
        assert np.allclose(s, np.eye(2), atol=1e-12)
    with pytest.raises(ValueError, match="completeness"):
        lq.KrausChannel([np.eye(2) * 0.5])
    with pytest.raises(ValueError, match="probability"):
        lq.KrausChannel.depolarizing(1.5)
    nm = lq.NoiseModel()
    assert nm.empty()
    assert nm.add_all_qubit_channel(lq.KrausChannel.bit_flip(0.1)) is nm
    assert not nm.empty()

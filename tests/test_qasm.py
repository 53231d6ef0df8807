"""OpenQASM 2.0 reader and writer (the pylqcs io surface): round trips equal the reference's
io::to_qasm(io::from_qasm(...)) byte for byte, errors carry the reference's messages.
Host logic only (no GPU)."""
import math

import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import io as qio

SOURCES = [
    """OPENQASM 2.0;
include "qelib1.inc";
qreg q[4];
creg c[4];
h q[0];
cx q[0],q[1];
u3(pi/2, -pi/4, 0.125) q[2];
u2(0.5, pi) q[3];
u1(-(pi+1)/3) q[1];
rz(2*pi/7) q[0]; // comment
crz(0.3) q[1],q[2];
cu1(1e-3) q[0],q[3];
ccx q[0],q[1],q[2];
cswap q[3],q[0],q[1];
barrier q[0],q[1];
reset q[2];
measure q -> c;
""",
    """OPENQASM 2.0;
qreg r[3];
creg m[2];
id r[0]; x r[1]; y r[2]; z r[0]; s r[1]; sdg r[2]; t r[0]; tdg r[1]; sx r[2];
rx(0.1) r[0]; ry(-0.2) r[1]; p(3) r[2]; u(1,2,3) r[0];
cy r[0],r[1]; cz r[1],r[2]; ch r[2],r[0]; cp(0.7) r[0],r[2]; crx(0.1) r[1],r[0];
cry(0.2) r[2],r[1]; swap r[0],r[2];
measure r[2] -> m[0];
measure r[0] -> m[1];
""",
]


@pytest.mark.parametrize("src", SOURCES)
def test_round_trip_equals_reference(ref, src):
    assert qio.to_qasm(qio.from_qasm(src)) == ref.qasm_roundtrip(src)


def test_builder_circuit_round_trip(ref):
    qc = lq.QuantumCircuit(3, 3)
    qc.h(0).cx(0, 1).u(0.1, 0.2, 0.3, 2).cp(math.pi / 3, 2, 0).swap(0, 1).measure_all()
    text = qio.to_qasm(qc)
    assert qio.to_qasm(qio.from_qasm(text)) == text == ref.qasm_roundtrip(text)


@pytest.mark.parametrize("src", [
    "OPENQASM 3.0; qreg q[1];",
    "OPENQASM 2.0; h q[0];",
    "OPENQASM 2.0; qreg q[2]; qreg r[1];",
    "OPENQASM 2.0; qreg q[2]; h q[0]; creg c[2];",
    "OPENQASM 2.0; qreg q[2]; foo q[0];",
    "OPENQASM 2.0; qreg q[2]; rx q[0];",
    "OPENQASM 2.0; qreg q[2]; h q;",
    "OPENQASM 2.0; qreg q[2]; rx(tau) q[0];",
    "OPENQASM 2.0; qreg q[2]; creg c[1]; measure q -> c;",
    "OPENQASM 2.0; qreg q[2]; creg c[2]; measure q[0] -> c;",
    "OPENQASM 2.0; qreg q[2]; reset q;",
    "OPENQASM 2.0; qreg q[2]; h p[0];",
    "OPENQASM 2.0;",
])
def test_errors_match_reference(ref, src):
    with pytest.raises(ValueError) as mine:
        qio.from_qasm(src)
    with pytest.raises(ValueError) as theirs:
        ref.qasm_roundtrip(src)
    assert str(mine.value).split(" near position")[0] == str(theirs.value).split(" near position")[0]


def test_writer_rejects_gates_outside_qelib1():
    qc = lq.QuantumCircuit(2)
    qc.rzz(0.3, 0, 1)
    with pytest.raises(ValueError, match="not representable in the OpenQASM 2.0 qelib1 gate set"):
        qio.to_qasm(qc)

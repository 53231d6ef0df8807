"""Circuit IR mirroring lqcs's QuantumCircuit / ParametricCircuit / Gate / GateType.

Pure host-side data: a circuit records instructions (controls first, then targets, as
``include/lqcs/circuit/instruction.hpp:9-13``) and validates them at build time with the
reference's rules and messages (``src/circuit/quantum_circuit.cpp``).  Method names,
argument order and the exceptions raised match the ``pylqcs`` bindings
(``python/src/bindings.cpp:34-147, 304-340``): ``std::invalid_argument`` surfaces as
``ValueError`` and ``std::out_of_range`` as ``IndexError``.

Gate matrices are computed by the engine's C++ host code (``lqcs_gate_matrix``), the
same code the device path uses.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _native as N


class GateType(enum.IntEnum):
    """Same names and numbering as lqcs::GateType (include/lqcs/circuit/gate.hpp:14-28)."""

    I = 0
    X = 1
    Y = 2
    Z = 3
    H = 4
    S = 5
    Sdg = 6
    T = 7
    Tdg = 8
    SX = 9
    RX = 10
    RY = 11
    RZ = 12
    P = 13
    U = 14
    SWAP = 15
    iSWAP = 16
    RXX = 17
    RYY = 18
    RZZ = 19
    PauliRotation = 20
    Unitary = 21
    Permutation = 22
    Measure = 23
    Reset = 24
    Barrier = 25
    # engine extension: an explicit one-qubit Kraus channel in the instruction stream
    Kraus = 64


_NAMES = {
    GateType.I: "id", GateType.X: "x", GateType.Y: "y", GateType.Z: "z", GateType.H: "h",
    GateType.S: "s", GateType.Sdg: "sdg", GateType.T: "t", GateType.Tdg: "tdg",
    GateType.SX: "sx", GateType.RX: "rx", GateType.RY: "ry", GateType.RZ: "rz",
    GateType.P: "p", GateType.U: "u", GateType.SWAP: "swap", GateType.iSWAP: "iswap",
    GateType.RXX: "rxx", GateType.RYY: "ryy", GateType.RZZ: "rzz",
    GateType.Unitary: "unitary", GateType.Permutation: "perm", GateType.Measure: "measure",
    GateType.Reset: "reset", GateType.Barrier: "barrier", GateType.Kraus: "kraus",
}

_TWO_QUBIT = {GateType.SWAP, GateType.iSWAP, GateType.RXX, GateType.RYY, GateType.RZZ}


@dataclass
class Gate:
    """lqcs::Gate (include/lqcs/circuit/gate.hpp:30-68)."""

    type: GateType
    params: list = field(default_factory=list)
    n_controls: int = 0
    mat: list = field(default_factory=list)      # Unitary: row-major complex
    perm: list = field(default_factory=list)     # Permutation
    pauli: str = ""                              # PauliRotation
    kraus: list = field(default_factory=list)    # Kraus: list of 4-tuples of complex

    def __post_init__(self):
        self.type = GateType(self.type)
        self.params = [float(p) for p in self.params]

    def base_qubits(self) -> int:
        t = self.type
        if t in _TWO_QUBIT:
            return 2
        if t == GateType.Unitary:
            dim = int(round(math.sqrt(len(self.mat))))
            return dim.bit_length() - 1
        if t == GateType.Permutation:
            return len(self.perm).bit_length() - 1
        if t == GateType.PauliRotation:
            return len(self.pauli)
        if t == GateType.Barrier:
            return 0
        return 1

    def num_qubits(self) -> int:
        return self.n_controls + self.base_qubits()

    def is_unitary(self) -> bool:
        return self.type not in (GateType.Measure, GateType.Reset, GateType.Barrier,
                                 GateType.Kraus)

    def is_diagonal(self) -> bool:
        if self.type in (GateType.I, GateType.Z, GateType.S, GateType.Sdg, GateType.T,
                         GateType.Tdg, GateType.RZ, GateType.P, GateType.RZZ):
            return True
        if self.type == GateType.PauliRotation:
            return all(c in "IZ" for c in self.pauli)
        return False

    def name(self) -> str:
        base = "rp(" + self.pauli + ")" if self.type == GateType.PauliRotation else _NAMES[self.type]
        if self.n_controls == 0:
            return base
        if self.n_controls == 1:
            return "c" + base
        if self.n_controls == 2:
            return "cc" + base
        return "mc" + base

    def _matrix(self, with_controls: bool) -> np.ndarray:
        if not self.is_unitary():
            raise RuntimeError(f"Gate::base_matrix: {self.name()} has no matrix")
        qubits = list(range(self.num_qubits()))
        inst = Instruction(self, qubits, [])
        arr, keep = _to_c([inst])
        dim = C.c_uint64(0)
        N.call("lqcs_gate_matrix", arr, int(with_controls), None, 0, C.byref(dim))
        out = np.zeros((dim.value, dim.value), dtype=np.complex128)
        N.call("lqcs_gate_matrix", arr, int(with_controls), out.ctypes.data, 2 * out.size,
               C.byref(dim))
        return out

    def base_matrix(self) -> np.ndarray:
        """Gate::base_matrix (src/circuit/gate.cpp:94-201)."""
        return self._matrix(False)

    def matrix(self) -> np.ndarray:
        """Gate::matrix (src/circuit/gate.cpp:203-226): controls in the low local bits."""
        return self._matrix(True)

    def inverse(self) -> "Gate":
        """Gate::inverse (src/circuit/gate.cpp:228-281)."""
        if not self.is_unitary():
            raise RuntimeError(f"Gate::inverse: {self.name()} is not invertible")
        t = self.type
        g = Gate(t, list(self.params), self.n_controls, list(self.mat), list(self.perm),
                 self.pauli)
        if t in (GateType.I, GateType.X, GateType.Y, GateType.Z, GateType.H, GateType.SWAP):
            return g
        if t in (GateType.RX, GateType.RY, GateType.RZ, GateType.P, GateType.RXX, GateType.RYY,
                 GateType.RZZ, GateType.PauliRotation):
            g.params[0] = -g.params[0]
            return g
        swap = {GateType.S: GateType.Sdg, GateType.Sdg: GateType.S, GateType.T: GateType.Tdg,
                GateType.Tdg: GateType.T}
        if t in swap:
            g.type = swap[t]
            return g
        if t == GateType.U:
            g.params = [-self.params[0], -self.params[2], -self.params[1]]
            return g
        if t in (GateType.SX, GateType.iSWAP, GateType.Unitary):
            m = self.base_matrix()
            g.type = GateType.Unitary
            g.mat = list(np.conj(m.T).reshape(-1))
            g.params = []
            return g
        if t == GateType.Permutation:
            inv = [0] * len(self.perm)
            for l, v in enumerate(self.perm):
                inv[v] = l
            g.perm = inv
            return g
        raise RuntimeError("Gate::inverse: unhandled gate type")

    def __repr__(self) -> str:
        return f"<Gate {self.name()}>"


@dataclass
class Instruction:
    """lqcs::Instruction: gate, qubits (controls first), clbits (Measure only)."""

    gate: Gate
    qubits: list
    clbits: list = field(default_factory=list)


def _to_c(instructions: Sequence[Instruction]):
    """Flatten instructions into a ctypes array of lqcs_instruction.

    Returns (array, keepalive): the keepalive list owns every buffer the records point to.
    """
    n = len(instructions)
    arr = (N.Instruction * max(n, 1))()
    keep = [arr]
    for i, inst in enumerate(instructions):
        g = inst.gate
        rec = arr[i]
        rec.gate_type = int(g.type)
        rec.n_controls = g.n_controls
        rec.n_qubits = len(inst.qubits)
        rec.n_params = len(g.params)
        for k, p in enumerate(g.params[:3]):
            rec.params[k] = p
        if inst.clbits:
            rec.clbit = inst.clbits[0]
        if inst.qubits:
            q = (C.c_uint32 * len(inst.qubits))(*inst.qubits)
            keep.append(q)
            rec.qubits = C.cast(q, C.POINTER(C.c_uint32))
        if g.type == GateType.Unitary:
            m = np.ascontiguousarray(np.asarray(g.mat, dtype=np.complex128)).view(np.float64)
            keep.append(m)
            rec.matrix = m.ctypes.data_as(C.POINTER(C.c_double))
        elif g.type == GateType.Kraus:
            m = np.ascontiguousarray(np.asarray(g.kraus, dtype=np.complex128).reshape(-1)).view(np.float64)
            keep.append(m)
            rec.matrix = m.ctypes.data_as(C.POINTER(C.c_double))
            rec.n_kraus = len(g.kraus)
        if g.type == GateType.Permutation:
            p = np.ascontiguousarray(np.asarray(g.perm, dtype=np.uint64))
            keep.append(p)
            rec.perm = p.ctypes.data_as(C.POINTER(C.c_uint64))
        if g.type == GateType.PauliRotation:
            b = g.pauli.encode()
            keep.append(b)
            rec.pauli = b
    return arr, keep


def _validate_unitary(m: np.ndarray) -> None:
    # U * U^dagger == I within 1e-10 (src/circuit/quantum_circuit.cpp:14-29)
    prod = m @ np.conj(m.T)
    if np.max(np.abs(prod - np.eye(m.shape[0]))) > 1e-10:
        raise ValueError("unitary: matrix is not unitary (U*Udag != I)")


class QuantumCircuit:
    """Fluent circuit builder: lqcs::QuantumCircuit (include/lqcs/circuit/quantum_circuit.hpp)."""

    def __init__(self, num_qubits: int, num_clbits: int = 0):
        if num_qubits == 0:
            raise ValueError("QuantumCircuit: num_qubits must be >= 1")
        self._n = int(num_qubits)
        self._nc = int(num_clbits)
        self._insts: list[Instruction] = []
        self._c_cache = None

    # ------------------------------------------------------------------ validation
    def _check_qubit(self, q: int) -> None:
        if q < 0 or q >= self._n:
            raise IndexError(f"qubit index {q} out of range (num_qubits = {self._n})")

    def _check_clbit(self, c: int) -> None:
        if c < 0 or c >= self._nc:
            raise IndexError(f"clbit index {c} out of range (num_clbits = {self._nc})")

    def _add(self, gate: Gate, qubits: Sequence[int]) -> "QuantumCircuit":
        qubits = [int(q) for q in qubits]
        if len(qubits) != gate.num_qubits():
            raise ValueError(f"{gate.name()}: expects {gate.num_qubits()} qubits, got {len(qubits)}")
        seen = set()
        for q in qubits:
            self._check_qubit(q)
            if q in seen:
                raise ValueError(f"{gate.name()}: duplicate qubit {q}")
            seen.add(q)
        self._insts.append(Instruction(gate, qubits, []))
        self._c_cache = None
        return self

    # ------------------------------------------------------------------ one-qubit gates
    def i(self, q): return self._add(Gate(GateType.I), [q])
    def x(self, q): return self._add(Gate(GateType.X), [q])
    def y(self, q): return self._add(Gate(GateType.Y), [q])
    def z(self, q): return self._add(Gate(GateType.Z), [q])
    def h(self, q): return self._add(Gate(GateType.H), [q])
    def s(self, q): return self._add(Gate(GateType.S), [q])
    def sdg(self, q): return self._add(Gate(GateType.Sdg), [q])
    def t(self, q): return self._add(Gate(GateType.T), [q])
    def tdg(self, q): return self._add(Gate(GateType.Tdg), [q])
    def sx(self, q): return self._add(Gate(GateType.SX), [q])
    def rx(self, theta, q): return self._add(Gate(GateType.RX, [theta]), [q])
    def ry(self, theta, q): return self._add(Gate(GateType.RY, [theta]), [q])
    def rz(self, theta, q): return self._add(Gate(GateType.RZ, [theta]), [q])
    def p(self, lam, q): return self._add(Gate(GateType.P, [lam]), [q])
    def u(self, theta, phi, lam, q): return self._add(Gate(GateType.U, [theta, phi, lam]), [q])

    # ------------------------------------------------------------------ controlled gates
    def cx(self, c, t): return self._add(Gate(GateType.X, [], 1), [c, t])
    def cy(self, c, t): return self._add(Gate(GateType.Y, [], 1), [c, t])
    def cz(self, c, t): return self._add(Gate(GateType.Z, [], 1), [c, t])
    def ch(self, c, t): return self._add(Gate(GateType.H, [], 1), [c, t])
    def cp(self, lam, c, t): return self._add(Gate(GateType.P, [lam], 1), [c, t])
    def crx(self, theta, c, t): return self._add(Gate(GateType.RX, [theta], 1), [c, t])
    def cry(self, theta, c, t): return self._add(Gate(GateType.RY, [theta], 1), [c, t])
    def crz(self, theta, c, t): return self._add(Gate(GateType.RZ, [theta], 1), [c, t])
    def ccx(self, c1, c2, t): return self._add(Gate(GateType.X, [], 2), [c1, c2, t])
    def cswap(self, c, a, b): return self._add(Gate(GateType.SWAP, [], 1), [c, a, b])

    def mcx(self, controls: Sequence[int], target: int):
        if len(controls) == 0:
            raise ValueError("mcx: needs at least one control qubit")
        return self._add(Gate(GateType.X, [], len(controls)), list(controls) + [target])

    def mcp(self, lam: float, controls: Sequence[int], target: int):
        if len(controls) == 0:
            raise ValueError("mcp: needs at least one control qubit")
        return self._add(Gate(GateType.P, [lam], len(controls)), list(controls) + [target])

    # ------------------------------------------------------------------ two-qubit gates
    def swap(self, a, b): return self._add(Gate(GateType.SWAP), [a, b])
    def iswap(self, a, b): return self._add(Gate(GateType.iSWAP), [a, b])
    def rxx(self, theta, a, b): return self._add(Gate(GateType.RXX, [theta]), [a, b])
    def ryy(self, theta, a, b): return self._add(Gate(GateType.RYY, [theta]), [a, b])
    def rzz(self, theta, a, b): return self._add(Gate(GateType.RZZ, [theta]), [a, b])

    def rp(self, theta: float, pauli: str, qubits: Sequence[int]):
        """exp(-i theta/2 P); the rightmost character of pauli acts on qubits[0]."""
        if len(pauli) == 0 or len(pauli) != len(qubits):
            raise ValueError("rp: pauli length must equal qubit count and be non-empty")
        if any(c not in "IXYZ" for c in pauli):
            raise ValueError("rp: pauli must contain only I/X/Y/Z")
        return self._add(Gate(GateType.PauliRotation, [theta], 0, pauli=pauli), list(qubits))

    # ------------------------------------------------------------------ custom operators
    def unitary(self, matrix, qubits: Sequence[int]):
        qubits = list(qubits)
        dim = 1 << len(qubits)
        m = np.asarray(matrix, dtype=np.complex128)
        if m.size != dim * dim:
            raise ValueError("unitary: matrix size must be 2^k x 2^k for k qubits")
        m = m.reshape(dim, dim)
        _validate_unitary(m)
        return self._add(Gate(GateType.Unitary, [], 0, list(m.reshape(-1))), qubits)

    def permutation(self, table: Sequence[int], qubits: Sequence[int]):
        qubits = list(qubits)
        dim = 1 << len(qubits)
        table = [int(v) for v in table]
        if len(table) != dim:
            raise ValueError("permutation: table size must be 2^k for k qubits")
        hit = [False] * dim
        for v in table:
            if v < 0 or v >= dim or hit[v]:
                raise ValueError("permutation: table is not a bijection")
            hit[v] = True
        return self._add(Gate(GateType.Permutation, [], 0, [], table), qubits)

    def kraus(self, ops, q: int):
        """Engine extension: a one-qubit Kraus channel applied at this point of every
        trajectory (ops: list of 2x2 matrices with sum K^dagger K = I)."""
        from .noise import KrausChannel
        ch = ops if isinstance(ops, KrausChannel) else KrausChannel(ops)
        self._check_qubit(q)
        self._insts.append(Instruction(Gate(GateType.Kraus, kraus=[tuple(k) for k in ch.ops]), [int(q)], []))
        self._c_cache = None
        return self

    # ------------------------------------------------------------------ non-unitary
    def measure(self, q: int, c: int):
        self._check_qubit(q)
        self._check_clbit(c)
        self._insts.append(Instruction(Gate(GateType.Measure), [int(q)], [int(c)]))
        self._c_cache = None
        return self

    def measure_all(self):
        self._nc = max(self._nc, self._n)
        for q in range(self._n):
            self.measure(q, q)
        return self

    def reset(self, q: int):
        self._check_qubit(q)
        self._insts.append(Instruction(Gate(GateType.Reset), [int(q)], []))
        self._c_cache = None
        return self

    def barrier(self):
        self._insts.append(Instruction(Gate(GateType.Barrier), [], []))
        self._c_cache = None
        return self

    def append(self, inst: Instruction):
        if inst.gate.type == GateType.Measure:
            if len(inst.qubits) != 1 or len(inst.clbits) != 1:
                raise ValueError("append: malformed measure instruction")
            self._check_clbit(inst.clbits[0])
            self._check_qubit(inst.qubits[0])
            self._insts.append(Instruction(inst.gate, list(inst.qubits), list(inst.clbits)))
            self._c_cache = None
            return self
        if inst.gate.type in (GateType.Reset, GateType.Barrier, GateType.Kraus):
            for q in inst.qubits:
                self._check_qubit(q)
            self._insts.append(Instruction(inst.gate, list(inst.qubits), []))
            self._c_cache = None
            return self
        return self._add(inst.gate, inst.qubits)

    # ------------------------------------------------------------------ composition
    def compose(self, other: "QuantumCircuit", qubit_map: Sequence[int] = ()):
        m = list(qubit_map)
        if not m:
            if other.num_qubits() > self._n:
                raise ValueError("compose: sub-circuit has more qubits")
            m = list(range(other.num_qubits()))
        if len(m) != other.num_qubits():
            raise ValueError("compose: qubit_map size must equal sub-circuit qubit count")
        seen = set()
        for q in m:
            self._check_qubit(q)
            if q in seen:
                raise ValueError("compose: duplicate qubit in map")
            seen.add(q)
        if other.num_clbits() > self._nc:
            raise ValueError("compose: sub-circuit has more clbits")
        for inst in other.instructions():
            self._insts.append(Instruction(inst.gate, [m[q] for q in inst.qubits], list(inst.clbits)))
        self._c_cache = None
        return self

    def inverse(self) -> "QuantumCircuit":
        inv = QuantumCircuit(self._n, self._nc)
        for inst in reversed(self._insts):
            if inst.gate.type == GateType.Barrier:
                inv.barrier()
                continue
            if not inst.gate.is_unitary():
                raise ValueError(
                    f"inverse: circuit contains non-unitary operation '{inst.gate.name()}'")
            inv._insts.append(Instruction(inst.gate.inverse(), list(inst.qubits), []))
        return inv

    def power(self, n: int) -> "QuantumCircuit":
        out = QuantumCircuit(self._n, self._nc)
        base = self.inverse() if n < 0 else self
        for _ in range(abs(n)):
            out.compose(base)
        return out

    # ------------------------------------------------------------------ accessors
    def num_qubits(self) -> int:
        return self._n

    def num_clbits(self) -> int:
        return self._nc

    def num_instructions(self) -> int:
        return len(self._insts)

    def instructions(self) -> list:
        return list(self._insts)

    def depth(self) -> int:
        level = [0] * self._n
        for inst in self._insts:
            if inst.gate.type == GateType.Barrier:
                continue
            d = max((level[q] for q in inst.qubits), default=0) + 1
            for q in inst.qubits:
                level[q] = d
        return max(level) if level else 0

    def c_instructions(self):
        """(ctypes array, count, keepalive) of the flattened instructions (cached)."""
        if self._c_cache is None:
            arr, keep = _to_c(self._insts)
            self._c_cache = (arr, len(self._insts), keep)
        return self._c_cache

    def __repr__(self) -> str:
        return (f"<QuantumCircuit qubits={self._n} clbits={self._nc} "
                f"instructions={len(self._insts)}>")


class ParametricCircuit:
    """lqcs::ParametricCircuit (include/lqcs/circuit/parametric_circuit.hpp:20-63):
    fixed gates plus parameterised rotations, one parameter per rotation in order."""

    def __init__(self, num_qubits: int, num_clbits: int = 0):
        self._t = QuantumCircuit(num_qubits, num_clbits)
        self._param_inst: list[int] = []

    def x(self, q): self._t.x(q); return self
    def y(self, q): self._t.y(q); return self
    def z(self, q): self._t.z(q); return self
    def h(self, q): self._t.h(q); return self
    def s(self, q): self._t.s(q); return self
    def sdg(self, q): self._t.sdg(q); return self
    def t(self, q): self._t.t(q); return self
    def sx(self, q): self._t.sx(q); return self
    def cx(self, c, t): self._t.cx(c, t); return self
    def cy(self, c, t): self._t.cy(c, t); return self
    def cz(self, c, t): self._t.cz(c, t); return self
    def swap(self, a, b): self._t.swap(a, b); return self
    def ccx(self, c1, c2, t): self._t.ccx(c1, c2, t); return self
    def barrier(self): self._t.barrier(); return self

    def _param(self, gate: Gate, qubits) -> int:
        idx = self._t.num_instructions()
        self._t.append(Instruction(gate, list(qubits), []))
        self._param_inst.append(idx)
        return len(self._param_inst) - 1

    def rx(self, qubit: int) -> int: return self._param(Gate(GateType.RX, [0.0]), [qubit])
    def ry(self, qubit: int) -> int: return self._param(Gate(GateType.RY, [0.0]), [qubit])
    def rz(self, qubit: int) -> int: return self._param(Gate(GateType.RZ, [0.0]), [qubit])

    def rp(self, pauli: str, qubits: Sequence[int]) -> int:
        if len(pauli) == 0 or len(pauli) != len(qubits):
            raise ValueError("ParametricCircuit::rp: pauli length must equal qubit count")
        if any(c not in "IXYZ" for c in pauli):
            raise ValueError("rp: pauli must contain only I/X/Y/Z")
        return self._param(Gate(GateType.PauliRotation, [0.0], 0, pauli=pauli), qubits)

    def bind(self, values: Sequence[float]) -> QuantumCircuit:
        """ParametricCircuit::bind (src/circuit/parametric_circuit.cpp:73-96)."""
        values = list(values)
        if len(values) != self.num_parameters():
            raise ValueError("bind: number of values must equal num_parameters()")
        param_of = {inst: p for p, inst in enumerate(self._param_inst)}
        out = QuantumCircuit(self._t.num_qubits(), self._t.num_clbits())
        for i, inst in enumerate(self._t.instructions()):
            g = inst.gate
            if i in param_of:
                g = Gate(g.type, [values[param_of[i]]] + g.params[1:], g.n_controls, g.mat,
                         g.perm, g.pauli)
            out._insts.append(Instruction(g, list(inst.qubits), list(inst.clbits)))
        return out

    def num_parameters(self) -> int: return len(self._param_inst)
    def num_qubits(self) -> int: return self._t.num_qubits()
    def num_clbits(self) -> int: return self._t.num_clbits()
    def template(self) -> QuantumCircuit: return self._t
    def param_instructions(self) -> list: return list(self._param_inst)

    def c_struct(self):
        """(lqcs_parametric_circuit, keepalive)."""
        arr, n, keep = self._t.c_instructions()
        pinst = (C.c_uint64 * max(1, len(self._param_inst)))(*self._param_inst)
        pc = N.ParametricCircuitC()
        pc.n_qubits = self._t.num_qubits()
        pc.n_insts = n
        pc.insts = C.cast(arr, C.POINTER(N.Instruction))
        pc.n_params = len(self._param_inst)
        pc.param_inst = C.cast(pinst, C.POINTER(C.c_uint64))
        return pc, [arr, keep, pinst]

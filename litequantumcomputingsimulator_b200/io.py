"""OpenQASM 2.0 in and out — the ``pylqcs.io`` surface (``from_qasm``, ``to_qasm``).

Behaviour follows the reference's reader and writer (src/io/qasm.cpp, include/lqcs/io/qasm.hpp):
the accepted subset is the writer's own output plus the usual qelib1 exports — one ``qreg``,
at most one ``creg`` (declared before any gate), ``include`` lines ignored, ``measure``
indexed or whole-register, ``barrier`` (its operands ignored: a full barrier), indexed
``reset``, the qelib1 gates listed in ``_READ`` and parameter expressions over numbers and
``pi`` with ``+ - * /``, unary minus and parentheses.  Errors raise ``ValueError`` with the
reference's ``from_qasm:`` / ``to_qasm:`` messages.
"""
from __future__ import annotations

import math
import re

from .circuit import GateType, QuantumCircuit

__all__ = ["from_qasm", "to_qasm"]

# ------------------------------------------------------------------ writer

# (gate type, number of controls) -> qelib1 name
_WRITE = {
    (GateType.I, 0): "id", (GateType.X, 0): "x", (GateType.X, 1): "cx", (GateType.X, 2): "ccx",
    (GateType.Y, 0): "y", (GateType.Y, 1): "cy", (GateType.Z, 0): "z", (GateType.Z, 1): "cz",
    (GateType.H, 0): "h", (GateType.H, 1): "ch", (GateType.S, 0): "s", (GateType.Sdg, 0): "sdg",
    (GateType.T, 0): "t", (GateType.Tdg, 0): "tdg", (GateType.SX, 0): "sx",
    (GateType.RX, 0): "rx", (GateType.RX, 1): "crx", (GateType.RY, 0): "ry",
    (GateType.RY, 1): "cry", (GateType.RZ, 0): "rz", (GateType.RZ, 1): "crz",
    (GateType.P, 0): "u1", (GateType.P, 1): "cu1", (GateType.U, 0): "u3",
    (GateType.SWAP, 0): "swap", (GateType.SWAP, 1): "cswap",
}


def _num(v: float) -> str:
    """printf %.17g."""
    return "%.17g" % v


def to_qasm(circuit: QuantumCircuit) -> str:
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{circuit.num_qubits()}];"]
    if circuit.num_clbits() > 0:
        lines.append(f"creg c[{circuit.num_clbits()}];")
    for inst in circuit.instructions():
        g = inst.gate
        if g.type == GateType.Barrier:
            lines.append("barrier q;")
        elif g.type == GateType.Measure:
            lines.append(f"measure q[{inst.qubits[0]}] -> c[{inst.clbits[0]}];")
        elif g.type == GateType.Reset:
            lines.append(f"reset q[{inst.qubits[0]}];")
        else:
            name = _WRITE.get((g.type, g.n_controls))
            if name is None:
                raise ValueError(f"to_qasm: gate '{g.name()}' is not representable in the "
                                 "OpenQASM 2.0 qelib1 gate set")
            par = "(" + ",".join(_num(p) for p in g.params) + ")" if g.params else ""
            lines.append(name + par + " " + ",".join(f"q[{q}]" for q in inst.qubits) + ";")
    return "\n".join(lines) + "\n"


# ------------------------------------------------------------------ reader

# qelib1 name -> (number of parameters, number of qubits, builder)
_READ = {
    "id": (0, 1, lambda qc, p, q: qc.i(*q)),
    "x": (0, 1, lambda qc, p, q: qc.x(*q)),
    "y": (0, 1, lambda qc, p, q: qc.y(*q)),
    "z": (0, 1, lambda qc, p, q: qc.z(*q)),
    "h": (0, 1, lambda qc, p, q: qc.h(*q)),
    "s": (0, 1, lambda qc, p, q: qc.s(*q)),
    "sdg": (0, 1, lambda qc, p, q: qc.sdg(*q)),
    "t": (0, 1, lambda qc, p, q: qc.t(*q)),
    "tdg": (0, 1, lambda qc, p, q: qc.tdg(*q)),
    "sx": (0, 1, lambda qc, p, q: qc.sx(*q)),
    "rx": (1, 1, lambda qc, p, q: qc.rx(p[0], *q)),
    "ry": (1, 1, lambda qc, p, q: qc.ry(p[0], *q)),
    "rz": (1, 1, lambda qc, p, q: qc.rz(p[0], *q)),
    "p": (1, 1, lambda qc, p, q: qc.p(p[0], *q)),
    "u1": (1, 1, lambda qc, p, q: qc.p(p[0], *q)),
    "u2": (2, 1, lambda qc, p, q: qc.u(math.pi / 2, p[0], p[1], *q)),
    "u": (3, 1, lambda qc, p, q: qc.u(p[0], p[1], p[2], *q)),
    "u3": (3, 1, lambda qc, p, q: qc.u(p[0], p[1], p[2], *q)),
    "cx": (0, 2, lambda qc, p, q: qc.cx(*q)),
    "cy": (0, 2, lambda qc, p, q: qc.cy(*q)),
    "cz": (0, 2, lambda qc, p, q: qc.cz(*q)),
    "ch": (0, 2, lambda qc, p, q: qc.ch(*q)),
    "cp": (1, 2, lambda qc, p, q: qc.cp(p[0], *q)),
    "cu1": (1, 2, lambda qc, p, q: qc.cp(p[0], *q)),
    "crx": (1, 2, lambda qc, p, q: qc.crx(p[0], *q)),
    "cry": (1, 2, lambda qc, p, q: qc.cry(p[0], *q)),
    "crz": (1, 2, lambda qc, p, q: qc.crz(p[0], *q)),
    "swap": (0, 2, lambda qc, p, q: qc.swap(*q)),
    "ccx": (0, 3, lambda qc, p, q: qc.ccx(*q)),
    "cswap": (0, 3, lambda qc, p, q: qc.cswap(*q)),
}

_TOKEN = re.compile(r"\s*(?:(//[^\n]*)|(\d+\.\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?|"
                    r"\d+(?:[eE][+-]?\d+)?)|([A-Za-z_][A-Za-z0-9_]*)|(\"[^\"]*\")|(->)|(\S))")


class _Reader:
    """Token stream with one-token lookahead; positions are character offsets."""

    def __init__(self, src: str):
        self.toks = []   # (kind, text, pos)
        pos = 0
        while pos < len(src):
            m = _TOKEN.match(src, pos)
            if m is None or m.end() == pos:
                break
            start = m.start(m.lastindex) if m.lastindex else m.end()
            kinds = (None, "comment", "num", "id", "str", "arrow", "sym")
            if m.lastindex and kinds[m.lastindex] != "comment":
                self.toks.append((kinds[m.lastindex], m.group(m.lastindex), start))
            pos = m.end()
        self.i = 0
        self.end = len(src)

    def fail(self, msg: str):
        pos = self.toks[self.i][2] if self.i < len(self.toks) else self.end
        raise ValueError(f"from_qasm: {msg} near position {pos}")

    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else (None, "", self.end)

    def take(self):
        t = self.peek()
        if t[0] is None:
            self.fail("unexpected end of input")
        self.i += 1
        return t

    def accept(self, text: str) -> bool:
        if self.peek()[1] == text:
            self.i += 1
            return True
        return False

    def expect(self, text: str):
        if not self.accept(text):
            self.fail(f"expected '{text}'")

    def ident(self) -> str:
        kind, text, _ = self.peek()
        if kind != "id":
            self.fail("expected identifier")
        self.i += 1
        return text

    # expressions: sum of products of signed factors
    def expr(self) -> float:
        v = self.product()
        while True:
            if self.accept("+"):
                v += self.product()
            elif self.accept("-"):
                v -= self.product()
            else:
                return v

    def product(self) -> float:
        v = self.factor()
        while True:
            if self.accept("*"):
                v *= self.factor()
            elif self.accept("/"):
                v /= self.factor()
            else:
                return v

    def factor(self) -> float:
        if self.accept("-"):
            return -self.factor()
        if self.accept("("):
            v = self.expr()
            self.expect(")")
            return v
        kind, text, _ = self.peek()
        if kind == "id":
            self.i += 1
            if text != "pi":
                self.i -= 1
                self.fail("unknown symbol in expression")
            return math.pi
        if kind == "num":
            self.i += 1
            return float(text)
        self.fail("expected number")


def from_qasm(source: str) -> QuantumCircuit:
    r = _Reader(source)
    if r.ident() != "OPENQASM":
        r.i -= 1
        r.fail("expected 'OPENQASM'")
    if r.peek()[1] != "2.0":
        r.fail("expected '2.0'")
    r.i += 1
    r.expect(";")
    qc = None
    qname = cname = ""
    nq = nc = 0

    def ref(reg: str):
        name = r.ident()
        if name != reg:
            r.i -= 1
            r.fail(f"unknown register '{name}'")
        if not r.accept("["):
            return None   # whole register
        idx = int(r.expr())
        r.expect("]")
        return idx

    while r.peek()[0] is not None:
        head = r.ident()
        if head == "include":
            if r.peek()[0] != "str":
                r.fail("expected '\"'")
            r.i += 1
            r.expect(";")
            continue
        if head in ("qreg", "creg"):
            name = r.ident()
            r.expect("[")
            size = int(r.expr())
            r.expect("]")
            r.expect(";")
            if head == "qreg":
                if qc is not None:
                    r.fail("only one qreg is supported")
                qname, nq = name, size
            else:
                if nc > 0:
                    r.fail("only one creg is supported")
                if qc is not None and qc.num_instructions() > 0:
                    r.fail("creg must be declared before any gate")
                cname, nc = name, size
            qc = QuantumCircuit(nq, nc) if nq > 0 else None
            continue
        if qc is None:
            r.fail("statement before qreg declaration")
        if head == "measure":
            q = ref(qname)
            if not r.accept("->"):
                r.fail("expected '->'")
            c = ref(cname)
            r.expect(";")
            if q is not None and c is not None:
                qc.measure(q, c)
            elif q is None and c is None:
                if nq != nc:
                    r.fail("whole-register measure needs equal register sizes")
                for i in range(nq):
                    qc.measure(i, i)
            else:
                r.fail("mixed whole-register and indexed measure")
            continue
        if head == "barrier":
            while r.peek()[0] is not None and r.peek()[1] != ";":
                r.i += 1
            r.expect(";")
            qc.barrier()
            continue
        if head == "reset":
            q = ref(qname)
            r.expect(";")
            if q is None:
                r.fail("reset requires an indexed qubit")
            qc.reset(q)
            continue
        params = []
        if r.accept("("):
            params.append(r.expr())
            while r.accept(","):
                params.append(r.expr())
            r.expect(")")
        qubits = []
        while True:
            q = ref(qname)
            if q is None:
                r.fail("gate operands must be indexed qubits")
            qubits.append(q)
            if not r.accept(","):
                break
        r.expect(";")
        spec = _READ.get(head)
        if spec is None or spec[0] != len(params) or spec[1] != len(qubits):
            r.fail(f"unsupported gate '{head}' with {len(params)} params / {len(qubits)} qubits")
        spec[2](qc, params, qubits)
    if qc is None:
        raise ValueError("from_qasm: missing qreg declaration")
    return qc

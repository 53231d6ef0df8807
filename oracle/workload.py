"""ORACLE — test infrastructure only; never imported by the product path.

The seeded brickwork circuit as the reference's CPU arm builds it, without the engine's
package: records in the ``lqcs_instruction`` layout (include/lqcs_b200.h), angles drawn
from the reference's own ``lqcs::Rng`` (src/util/random.hpp:10-23) through
``oracle/_ref/liblqcs_ref.so`` (``lqcsref_uniforms``) or, where that library is absent,
from the C restatement of mt19937_64 (``MT64``).

Generator (the reference ships none; the engine's workloads.brickwork draws the same
sequence): per layer, U(theta, phi, lambda) on every qubit with each angle 2*pi*u, then
CX on a perfect matching from a Fisher-Yates shuffle of 0..n-1 (index j = min(floor(u*(i+1)),
i) for i = n-1 .. 1), pairs (p0, p1), (p2, p3), ...; the first of a pair is the control.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import List, Sequence, Tuple

import numpy as np

X_GATE, U_GATE = 1, 14   # lqcs::GateType::X, lqcs::GateType::U (gate.hpp:14-28)


class InstructionC(C.Structure):
    """lqcs_instruction of include/lqcs_b200.h."""
    _fields_ = [
        ("gate_type", C.c_int32),
        ("n_controls", C.c_uint32),
        ("n_qubits", C.c_uint32),
        ("n_params", C.c_uint32),
        ("params", C.c_double * 3),
        ("clbit", C.c_uint32),
        ("n_kraus", C.c_uint32),
        ("qubits", C.POINTER(C.c_uint32)),
        ("matrix", C.POINTER(C.c_double)),
        ("perm", C.POINTER(C.c_uint64)),
        ("pauli", C.c_char_p),
    ]


class GateList:
    """A list of U and CX records on n qubits; duck-types the circuit argument of
    ``oracle.oracle.Ref`` (``num_qubits()``, ``c_instructions()``)."""

    def __init__(self, n: int, records: Sequence[Tuple[int, int, tuple, tuple]] = ()):
        self.n = n
        self.records: List[Tuple[int, int, tuple, tuple]] = list(records)   # (type, n_ctrl, qubits, params)
        self._c = None

    def num_qubits(self) -> int:
        return self.n

    def num_clbits(self) -> int:
        return 0

    def u(self, theta: float, phi: float, lam: float, q: int) -> None:
        self.records.append((U_GATE, 0, (q,), (theta, phi, lam)))
        self._c = None

    def cx(self, c: int, t: int) -> None:
        self.records.append((X_GATE, 1, (c, t), ()))
        self._c = None

    def slice(self, lo: int, hi: int) -> "GateList":
        return GateList(self.n, self.records[lo:hi])

    def __len__(self) -> int:
        return len(self.records)

    def c_instructions(self):
        if self._c is None:
            arr = (InstructionC * max(1, len(self.records)))()
            keep = [arr]
            for i, (gt, nc, qs, ps) in enumerate(self.records):
                r = arr[i]
                r.gate_type = gt
                r.n_controls = nc
                r.n_qubits = len(qs)
                r.n_params = len(ps)
                for k, p in enumerate(ps):
                    r.params[k] = p
                q = (C.c_uint32 * len(qs))(*qs)
                keep.append(q)
                r.qubits = C.cast(q, C.POINTER(C.c_uint32))
            self._c = (arr, len(self.records), keep)
        return self._c

    def alg_bytes(self) -> float:
        """32 * 2^n * f per gate: f = 1 for U, 1/2 for CX (one control)."""
        total = 0.0
        for _gt, nc, _qs, _ps in self.records:
            total += 32.0 * (1 << self.n) * 2.0 ** (-nc)
        return total


class _Uniforms:
    """Sequential uniforms of lqcs::Rng(seed)."""

    def __init__(self, seed: int, draw):
        self.seed, self.draw = seed, draw
        self.buf = np.zeros(0)
        self.pos = 0

    def next(self) -> float:
        if self.pos >= self.buf.size:
            self.buf = self.draw(self.seed, max(2 * self.buf.size, 4096))
        v = float(self.buf[self.pos])
        self.pos += 1
        return v


def _reference_draw():
    from .oracle import Ref, MT64
    if Ref.available():
        ref = Ref()
        return ref.uniforms

    def draw(seed: int, count: int) -> np.ndarray:
        return MT64(seed).uniforms(count)
    return draw


def brickwork(n: int, depth: int, seed: int) -> GateList:
    """The seeded brickwork circuit (n U gates then n // 2 CX per layer)."""
    rng = _Uniforms(seed, _reference_draw())
    qc = GateList(n)
    two_pi = 2.0 * math.pi
    for _ in range(depth):
        for q in range(n):
            th, ph, la = (two_pi * rng.next() for _ in range(3))
            qc.u(th, ph, la, q)
        order = list(range(n))
        for i in range(n - 1, 0, -1):
            j = min(int(rng.next() * (i + 1)), i)
            order[i], order[j] = order[j], order[i]
        for k in range(0, n - 1, 2):
            qc.cx(order[k], order[k + 1])
    return qc


def layer_size(n: int) -> int:
    """Gates per brickwork layer."""
    return n + n // 2

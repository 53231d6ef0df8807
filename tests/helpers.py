"""Random circuit generators for the parity tests (every gate type of lqcs::GateType, any
control count, any target placement), seeded with numpy."""
from __future__ import annotations

import math

import numpy as np

import litequantumcomputingsimulator_b200 as lq


def random_unitary(k: int, rng: np.random.Generator) -> np.ndarray:
    dim = 1 << k
    z = (rng.standard_normal((dim, dim)) + 1j * rng.standard_normal((dim, dim))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))


def random_circuit(n: int, n_gates: int, seed: int, kinds=None, max_controls: int = 3,
                   max_unitary: int = 3) -> lq.QuantumCircuit:
    rng = np.random.default_rng(seed)
    qc = lq.QuantumCircuit(n)
    all_kinds = ["1q", "1qp", "u", "c1q", "mc", "swap", "cswap", "2q", "rp", "unitary", "perm",
                 "cperm", "ccx", "cp", "mcp"]
    kinds = kinds or all_kinds
    fixed1 = ["i", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx"]
    rot1 = ["rx", "ry", "rz", "p"]
    for _ in range(n_gates):
        kind = kinds[rng.integers(len(kinds))]
        q = rng.permutation(n).tolist()
        ang = float(rng.uniform(-math.pi, math.pi))
        if kind == "1q":
            getattr(qc, fixed1[rng.integers(len(fixed1))])(q[0])
        elif kind == "1qp":
            getattr(qc, rot1[rng.integers(len(rot1))])(ang, q[0])
        elif kind == "u":
            qc.u(*rng.uniform(0, 2 * math.pi, 3), q[0])
        elif kind == "c1q" and n >= 2:
            name = ["cx", "cy", "cz", "ch"][rng.integers(4)]
            getattr(qc, name)(q[0], q[1])
            if rng.integers(2):
                getattr(qc, ["crx", "cry", "crz"][rng.integers(3)])(ang, q[0], q[1])
        elif kind == "mc" and n >= 3:
            c = int(rng.integers(2, min(max_controls, n - 1) + 1))
            qc.mcx(q[:c], q[c])
        elif kind == "mcp" and n >= 3:
            c = int(rng.integers(2, min(max_controls, n - 1) + 1))
            qc.mcp(ang, q[:c], q[c])
        elif kind == "ccx" and n >= 3:
            qc.ccx(q[0], q[1], q[2])
        elif kind == "cp" and n >= 2:
            qc.cp(ang, q[0], q[1])
        elif kind == "swap" and n >= 2:
            qc.swap(q[0], q[1])
        elif kind == "cswap" and n >= 3:
            qc.cswap(q[0], q[1], q[2])
        elif kind == "2q" and n >= 2:
            name = ["iswap", "rxx", "ryy", "rzz"][rng.integers(4)]
            if name == "iswap":
                qc.iswap(q[0], q[1])
            else:
                getattr(qc, name)(ang, q[0], q[1])
        elif kind == "rp":
            w = int(rng.integers(1, min(n, 6) + 1))
            pauli = "".join("IXYZ"[i] for i in rng.integers(0, 4, w))
            qc.rp(ang, pauli, q[:w])
        elif kind == "unitary":
            k = int(rng.integers(1, min(n, max_unitary) + 1))
            qc.unitary(random_unitary(k, rng), q[:k])
        elif kind == "perm":
            k = int(rng.integers(1, min(n, 3) + 1))
            qc.permutation(rng.permutation(1 << k).tolist(), q[:k])
        elif kind == "cperm" and n >= 3:
            k = int(rng.integers(1, min(n - 1, 3) + 1))
            table = rng.permutation(1 << k).tolist()
            g = lq.Gate(lq.GateType.Permutation, [], 1, [], table)
            qc.append(lq.Instruction(g, [q[k]] + q[:k], []))
    return qc

"""Seeded synthetic workloads (the reference ships no circuit generators; these define them).

Every random draw comes from lqcs::Rng(seed) — std::mt19937_64 with
uniform_real_distribution<double>(0, 1) — through ``lqcs_rng_uniforms``, so the C++ side
of the reference can regenerate the same circuits from the same seed.

* brickwork(n, depth, seed): per layer, U3 on every qubit (theta, phi, lambda iid
  U[0, 2 pi)), then CX on a random perfect matching of the qubits (Fisher-Yates shuffle;
  pairs (p0, p1), (p2, p3), ...; the first of a pair is the control).
* random_pauli_ansatz(n, n_gates, seed): ParametricCircuit of rp gates on random supports
  of weight U{2..8}, Paulis iid from {X, Y, Z}; plus angles U[-pi, pi).
* random_hamiltonian(n, n_terms, seed): coefficients N(0, 1) (Box-Muller), each qubit iid
  from {I, X, Y, Z}, an all-identity string is redrawn.
* gaussian_state(n, seed): iid complex Gaussian amplitudes normalised to 1.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N
from .circuit import ParametricCircuit, QuantumCircuit


class UniformStream:
    """Sequential uniforms of lqcs::Rng(seed), fetched from the engine in blocks."""

    def __init__(self, seed: int, block: int = 1 << 16):
        self.seed = int(seed)
        self.block = block
        self.pos = 0
        self.buf = np.zeros(0)
        self.base = 0

    def _fill(self, upto: int) -> None:
        need = max(upto, self.base + self.buf.size + self.block)
        out = np.empty(need, dtype=np.float64)
        N.call("lqcs_rng_uniforms", self.seed, need, out.ctypes.data)
        self.buf = out
        self.base = 0

    def next(self) -> float:
        if self.pos >= self.base + self.buf.size:
            self._fill(self.pos + 1)
        v = float(self.buf[self.pos - self.base])
        self.pos += 1
        return v

    def take(self, k: int) -> np.ndarray:
        if self.pos + k > self.base + self.buf.size:
            self._fill(self.pos + k)
        v = self.buf[self.pos - self.base: self.pos - self.base + k].copy()
        self.pos += k
        return v

    def randint(self, hi: int) -> int:
        """Integer in [0, hi)."""
        return min(int(self.next() * hi), hi - 1)


def _shuffle(order: list, rng: UniformStream) -> list:
    for i in range(len(order) - 1, 0, -1):
        j = rng.randint(i + 1)
        order[i], order[j] = order[j], order[i]
    return order


def brickwork(n: int, depth: int, seed: int, measure: bool = False,
              noise=None) -> QuantumCircuit:
    """Random brickwork circuit.  With ``noise=(p1, p2, gamma)`` explicit Kraus
    instructions follow the gates: depolarizing p1 on the qubit after each U3,
    depolarizing p2 on each qubit after each CX, amplitude damping gamma on every qubit at
    the end of each layer."""
    from .noise import KrausChannel
    rng = UniformStream(seed)
    qc = QuantumCircuit(n, n if measure else 0)
    two_pi = 2.0 * math.pi
    if noise is not None:
        dep1 = KrausChannel.depolarizing(noise[0])
        dep2 = KrausChannel.depolarizing(noise[1])
        ad = KrausChannel.amplitude_damping(noise[2])
    for _ in range(depth):
        for q in range(n):
            th, ph, la = (two_pi * v for v in rng.take(3))
            qc.u(th, ph, la, q)
            if noise is not None:
                qc.kraus(dep1, q)
        order = _shuffle(list(range(n)), rng)
        for k in range(0, n - 1, 2):
            c, t = order[k], order[k + 1]
            qc.cx(c, t)
            if noise is not None:
                qc.kraus(dep2, c)
                qc.kraus(dep2, t)
        if noise is not None:
            for q in range(n):
                qc.kraus(ad, q)
    if measure:
        qc.measure_all()
    return qc


def random_pauli_ansatz(n: int, n_gates: int, seed: int, min_w: int = 2, max_w: int = 8):
    """(ParametricCircuit, params) with n_gates rp rotations."""
    rng = UniformStream(seed)
    pc = ParametricCircuit(n)
    for _ in range(n_gates):
        w = min_w + rng.randint(min(max_w, n) - min_w + 1)
        support = _shuffle(list(range(n)), rng)[:w]
        pauli = "".join("XYZ"[rng.randint(3)] for _ in range(w))
        pc.rp(pauli, support)
    params = (rng.take(n_gates) * 2.0 - 1.0) * math.pi
    return pc, params


def random_parameter_sets(n_params: int, n_sets: int, seed: int) -> np.ndarray:
    rng = UniformStream(seed)
    return ((rng.take(n_params * n_sets) * 2.0 - 1.0) * math.pi).reshape(n_sets, n_params)


def random_hamiltonian(n: int, n_terms: int, seed: int) -> list:
    rng = UniformStream(seed)
    terms = []
    while len(terms) < n_terms:
        u1, u2 = rng.next(), rng.next()
        coeff = math.sqrt(-2.0 * math.log(max(u1, 1e-300))) * math.cos(2.0 * math.pi * u2)
        while True:
            s = "".join("IXYZ"[rng.randint(4)] for _ in range(n))
            if any(ch != "I" for ch in s):
                break
        terms.append((coeff, s))
    return terms


def gaussian_state(n: int, seed: int) -> np.ndarray:
    """iid complex Gaussian amplitudes (Box-Muller on lqcs::Rng uniforms), normalised."""
    rng = UniformStream(seed, block=min(1 << 22, 2 << n))
    size = 1 << n
    out = np.empty(size, dtype=np.complex128)
    chunk = 1 << 20
    for s in range(0, size, chunk):
        m = min(chunk, size - s)
        u = rng.take(2 * m).reshape(m, 2)
        r = np.sqrt(-2.0 * np.log(np.maximum(u[:, 0], 1e-300)))
        out[s:s + m] = r * np.cos(2 * np.pi * u[:, 1]) + 1j * r * np.sin(2 * np.pi * u[:, 1])
    out /= math.sqrt(float(np.vdot(out, out).real))
    return out


def random_mix_circuit(n: int, depth: int, seed: int) -> QuantumCircuit:
    """Gate mix of the cost-model workload: per layer, about n gates drawn 50 % U3,
    30 % CX or CZ (random pair), 10 % RZZ (random pair, random angle), 10 % Pauli
    rotation of weight 2..8 on random qubits."""
    rng = UniformStream(seed)
    qc = QuantumCircuit(n)
    two_pi = 2.0 * math.pi
    for _ in range(depth):
        for _ in range(n):
            r = rng.next()
            if r < 0.5:
                q = rng.randint(n)
                th, ph, la = (two_pi * v for v in rng.take(3))
                qc.u(th, ph, la, q)
            elif r < 0.8:
                a, b = _shuffle(list(range(n)), rng)[:2]
                if rng.next() < 0.5:
                    qc.cx(a, b)
                else:
                    qc.cz(a, b)
            elif r < 0.9:
                a, b = _shuffle(list(range(n)), rng)[:2]
                qc.rzz(two_pi * rng.next(), a, b)
            else:
                w = 2 + rng.randint(min(8, n) - 1)
                support = _shuffle(list(range(n)), rng)[:w]
                pauli = "".join("XYZ"[rng.randint(3)] for _ in range(w))
                qc.rp(two_pi * rng.next() - math.pi, pauli, support)
    return qc


def alg_bytes(circuit: QuantumCircuit) -> float:
    """Algorithmic bytes of a circuit's gates on its register: sum over gates of
    32 * 2^n * f, f = the fraction of amplitudes the gate can change (dense and fused
    gates 1; diagonal gates with one entry equal to 1: 1/2; c controls: 2^-c; SWAP: 1/2)."""
    from .circuit import GateType
    n = circuit.num_qubits()
    total = 0.0
    for inst in circuit.instructions():
        g = inst.gate
        if not g.is_unitary():
            continue
        f = 2.0 ** (-g.n_controls)
        if g.type == GateType.SWAP:
            f *= 0.5
        elif g.type in (GateType.Z, GateType.S, GateType.Sdg, GateType.T, GateType.Tdg, GateType.P):
            f *= 0.5
        total += 32.0 * (1 << n) * f
    return total

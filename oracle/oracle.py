"""ORACLE — test infrastructure only; never imported by the product path.

Two checkers for the engine, both on the CPU:

* ``Port`` — a restatement of the reference's statevector semantics: the instruction
  dispatch of ``StatevectorSimulator`` (src/backend/statevector_simulator.cpp:22-85),
  gate matrices (src/circuit/gate.cpp:94-201), single-qubit fusion
  (src/transpiler/gate_fusion.cpp:32-67), end-of-circuit sampling and per-shot
  trajectories (src/backend/statevector_simulator.cpp:88-265), expectations
  (src/backend/statevector.cpp:39-78) and the parameter-shift gradient
  (src/algorithms/vqe.cpp:68-94).  The amplitude loops run in oracle/lqcs_oracle.c
  (``liblqcs_oracle.so``), the rest is plain Python.
* ``Ref`` — the reference itself, compiled from its own sources into
  ``oracle/_ref/liblqcs_ref.so`` (oracle/Makefile) and reached through oracle/ref_shim.cpp.
  Available wherever that library was built; it travels with the repository snapshot.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "liblqcs_oracle.so"
REF_LIB = HERE / "_ref" / "liblqcs_ref.so"

# gate type numbers (same order as lqcs::GateType, include/lqcs/circuit/gate.hpp:14-28)
I, X, Y, Z, H, S, SDG, T, TDG, SX, RX, RY, RZ, P, U, SWAP, ISWAP, RXX, RYY, RZZ, \
    PAULI_ROTATION, UNITARY, PERMUTATION, MEASURE, RESET, BARRIER = range(26)
KRAUS = 64

_dp = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class _PortLib:
    _lib = None

    @classmethod
    def get(cls):
        if cls._lib is None:
            if not PORT_LIB.exists():
                raise RuntimeError(f"{PORT_LIB} missing: run `make -C oracle port`")
            lib = C.CDLL(str(PORT_LIB))
            u32, u64, d = C.c_uint32, C.c_uint64, C.c_double
            vp = C.c_void_p
            sig = {
                "orc_apply_single_qubit": (None, [vp, u64, u32, vp]),
                "orc_apply_diagonal": (None, [vp, u64, u32, vp]),
                "orc_apply_controlled_single": (None, [vp, u64, u32, u32, vp]),
                "orc_apply_swap": (None, [vp, u64, u32, u32]),
                "orc_apply_two_qubit": (None, [vp, u64, u32, u32, vp]),
                "orc_apply_controlled_unitary": (None, [vp, u64, vp, u32, vp, u32, vp]),
                "orc_apply_controlled_permutation": (None, [vp, u64, vp, u32, vp, u32, vp]),
                "orc_apply_pauli_rotation": (None, [vp, u64, u64, u64, u32, d, d]),
                "orc_collapse_qubit": (C.c_int, [vp, u64, u32, d]),
                "orc_reset_qubit": (None, [vp, u64, u32, d]),
                "orc_kraus_probability": (d, [vp, u64, u32, vp]),
                "orc_expectation": (d, [vp, u64, u64, u64, u32]),
                "orc_cumulative": (None, [vp, u64, vp]),
                "orc_upper_bound": (u64, [vp, u64, d]),
                "orc_norm": (d, [vp, u64]),
                "orc_mt64_seed": (None, [vp, u64]),
                "orc_mt64_next": (u64, [vp]),
                "orc_mt64_uniform": (d, [vp]),
                "orc_mt64_sizeof": (C.c_size_t, []),
                "orc_mt64_uniforms": (None, [vp, u64, vp]),
            }
            for name, (res, args) in sig.items():
                f = getattr(lib, name)
                f.restype = res
                f.argtypes = args
            cls._lib = lib
        return cls._lib


class MT64:
    """std::mt19937_64 + uniform_real_distribution<double>(0,1), as lqcs::Rng draws it."""

    def __init__(self, seed: int = 5489):
        lib = _PortLib.get()
        self._buf = C.create_string_buffer(lib.orc_mt64_sizeof())
        lib.orc_mt64_seed(self._buf, seed & 0xFFFFFFFFFFFFFFFF)

    def next_u64(self) -> int:
        return _PortLib.get().orc_mt64_next(self._buf)

    def uniform(self) -> float:
        return _PortLib.get().orc_mt64_uniform(self._buf)

    def uniforms(self, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        _PortLib.get().orc_mt64_uniforms(self._buf, n, out.ctypes.data)
        return out


# ------------------------------------------------------------------ gate matrices
def _expi(t: float) -> complex:
    return complex(math.cos(t), math.sin(t))


def base_matrix(gtype: int, params, mat=None, perm=None, pauli: str = "") -> np.ndarray:
    """Gate::base_matrix (src/circuit/gate.cpp:94-201) with libm cos/sin."""
    s2 = math.sqrt(2.0) / 2.0
    kI = 1j
    t = gtype
    if t == I: m = [1, 0, 0, 1]
    elif t == X: m = [0, 1, 1, 0]
    elif t == Y: m = [0, -kI, kI, 0]
    elif t == Z: m = [1, 0, 0, -1]
    elif t == H: m = [s2, s2, s2, -s2]
    elif t == S: m = [1, 0, 0, kI]
    elif t == SDG: m = [1, 0, 0, -kI]
    elif t == T: m = [1, 0, 0, _expi(math.pi / 4)]
    elif t == TDG: m = [1, 0, 0, _expi(-math.pi / 4)]
    elif t == SX: m = [0.5 + 0.5j, 0.5 - 0.5j, 0.5 - 0.5j, 0.5 + 0.5j]
    elif t == RX:
        h = params[0] / 2
        m = [math.cos(h), -kI * math.sin(h), -kI * math.sin(h), math.cos(h)]
    elif t == RY:
        h = params[0] / 2
        m = [math.cos(h), -math.sin(h), math.sin(h), math.cos(h)]
    elif t == RZ:
        h = params[0] / 2
        m = [_expi(-h), 0, 0, _expi(h)]
    elif t == P: m = [1, 0, 0, _expi(params[0])]
    elif t == U:
        h = params[0] / 2
        phi, lam = params[1], params[2]
        m = [math.cos(h), -_expi(lam) * math.sin(h), _expi(phi) * math.sin(h),
             _expi(phi + lam) * math.cos(h)]
    elif t == SWAP: m = [1, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 1]
    elif t == ISWAP: m = [1, 0, 0, 0, 0, 0, kI, 0, 0, kI, 0, 0, 0, 0, 0, 1]
    elif t == RXX:
        h = params[0] / 2
        c, i_s = math.cos(h), kI * math.sin(h)
        m = [c, 0, 0, -i_s, 0, c, -i_s, 0, 0, -i_s, c, 0, -i_s, 0, 0, c]
    elif t == RYY:
        h = params[0] / 2
        c, i_s = math.cos(h), kI * math.sin(h)
        m = [c, 0, 0, i_s, 0, c, -i_s, 0, 0, -i_s, c, 0, i_s, 0, 0, c]
    elif t == RZZ:
        h = params[0] / 2
        m = [_expi(-h), 0, 0, 0, 0, _expi(h), 0, 0, 0, 0, _expi(h), 0, 0, 0, 0, _expi(-h)]
    elif t == PAULI_ROTATION:
        k = len(pauli)
        dim = 1 << k
        x, zy, ny = pauli_local_masks(pauli)
        h = params[0] / 2
        out = np.zeros((dim, dim), dtype=np.complex128)
        yph = [1, 1j, -1, -1j][ny % 4]
        mis = complex(0.0, -math.sin(h))
        for col in range(dim):
            out[col, col] += math.cos(h)
            sign = 1.0 if bin(col & zy).count("1") % 2 == 0 else -1.0
            out[col ^ x, col] += mis * yph * sign
        return out
    elif t == UNITARY:
        dim = int(round(math.sqrt(len(mat))))
        return np.asarray(mat, dtype=np.complex128).reshape(dim, dim)
    elif t == PERMUTATION:
        dim = len(perm)
        out = np.zeros((dim, dim), dtype=np.complex128)
        for l, v in enumerate(perm):
            out[v, l] = 1
        return out
    else:
        raise ValueError("no matrix for this gate type")
    dim = 2 if len(m) == 4 else 4
    return np.asarray(m, dtype=np.complex128).reshape(dim, dim)


def pauli_local_masks(pauli: str):
    """Gate::pauli_masks (src/circuit/gate.cpp:51-68): local bit j <-> pauli[k-1-j]."""
    x = zy = ny = 0
    k = len(pauli)
    for j in range(k):
        c = pauli[k - 1 - j]
        b = 1 << j
        if c == "X": x |= b
        elif c == "Y": x |= b; zy |= b; ny += 1
        elif c == "Z": zy |= b
    return x, zy, ny


def pauli_global_masks(pauli: str, n: int):
    """Statevector::expectation_value masks (src/backend/statevector.cpp:44-60)."""
    x = zy = ny = 0
    for j, c in enumerate(pauli):
        b = 1 << (n - 1 - j)
        if c == "X": x |= b
        elif c == "Z": zy |= b
        elif c == "Y": x |= b; zy |= b; ny += 1
    return x, zy, ny


def is_diagonal_type(gtype: int, pauli: str = "") -> bool:
    # Gate::is_diagonal (src/circuit/gate.cpp:75-92)
    if gtype in (I, Z, S, SDG, T, TDG, RZ, P, RZZ):
        return True
    if gtype == PAULI_ROTATION:
        return pauli_local_masks(pauli)[0] == 0
    return False


def _base_qubits(g) -> int:
    t = int(g.type)
    if t in (SWAP, ISWAP, RXX, RYY, RZZ): return 2
    if t == UNITARY: return int(round(math.sqrt(len(g.mat)))).bit_length() - 1
    if t == PERMUTATION: return len(g.perm).bit_length() - 1
    if t == PAULI_ROTATION: return len(g.pauli)
    if t == BARRIER: return 0
    return 1


def _is_unitary(g) -> bool:
    return int(g.type) not in (MEASURE, RESET, BARRIER, KRAUS)


def _gate_matrix(g) -> np.ndarray:
    return base_matrix(int(g.type), g.params, g.mat, g.perm, g.pauli)


# ------------------------------------------------------------------ the port
class Port:
    """CPU restatement of the reference's statevector backend (see module docstring)."""

    def __init__(self):
        self.lib = _PortLib.get()

    # ---- amplitude-level dispatch: apply_instruction (statevector_simulator.cpp:22-85)
    def apply_instruction(self, st: np.ndarray, inst) -> None:
        lib = self.lib
        g = inst.gate
        t = int(g.type)
        nc = g.n_controls
        k = _base_qubits(g)
        qs = [int(q) for q in inst.qubits]
        controls, targets = qs[:nc], qs[nc:]
        n_amps = st.size
        buf = st.ctypes.data
        cu = (C.c_uint32 * max(1, nc))(*controls)
        tu = (C.c_uint32 * max(1, k))(*targets)
        if t == PERMUTATION:
            perm = np.ascontiguousarray(g.perm, dtype=np.uint64)
            lib.orc_apply_controlled_permutation(buf, n_amps, cu, nc, tu, k, perm.ctypes.data)
            return
        if t == PAULI_ROTATION and nc == 0:
            lx, lzy, ny = pauli_local_masks(g.pauli)
            xg = zyg = 0
            for j in range(k):
                if lx >> j & 1: xg |= 1 << targets[j]
                if lzy >> j & 1: zyg |= 1 << targets[j]
            h = g.params[0] / 2
            lib.orc_apply_pauli_rotation(buf, n_amps, xg, zyg, ny, math.cos(h), math.sin(h))
            return
        m = np.ascontiguousarray(_gate_matrix(g), dtype=np.complex128)
        if nc == 0 and k == 1:
            if is_diagonal_type(t, g.pauli):
                d = np.array([m[0, 0], m[1, 1]], dtype=np.complex128)
                lib.orc_apply_diagonal(buf, n_amps, targets[0], d.ctypes.data)
            else:
                lib.orc_apply_single_qubit(buf, n_amps, targets[0], m.ctypes.data)
            return
        if nc == 0 and t == SWAP:
            lib.orc_apply_swap(buf, n_amps, targets[0], targets[1])
            return
        if nc == 0 and k == 2:
            lib.orc_apply_two_qubit(buf, n_amps, targets[0], targets[1], m.ctypes.data)
            return
        if nc == 1 and k == 1:
            lib.orc_apply_controlled_single(buf, n_amps, controls[0], targets[0], m.ctypes.data)
            return
        lib.orc_apply_controlled_unitary(buf, n_amps, cu, nc, tu, k, m.ctypes.data)

    # ---- SingleQubitGateFusion (src/transpiler/gate_fusion.cpp:32-67)
    def fuse_1q(self, instructions, n: int) -> list:
        from types import SimpleNamespace as NS
        out = []
        pending: list[Optional[np.ndarray]] = [None] * n

        def is_identity(m):
            tol = 1e-12
            return (abs(m[0, 0] - 1) < tol and abs(m[0, 1]) < tol and abs(m[1, 0]) < tol
                    and abs(m[1, 1] - 1) < tol)

        def mm(a, b):  # 2x2 product with the reference's summation order
            return np.array([[a[0, 0] * b[0, 0] + a[0, 1] * b[1, 0], a[0, 0] * b[0, 1] + a[0, 1] * b[1, 1]],
                             [a[1, 0] * b[0, 0] + a[1, 1] * b[1, 0], a[1, 0] * b[0, 1] + a[1, 1] * b[1, 1]]])

        def flush(q):
            if pending[q] is None:
                return
            if not is_identity(pending[q]):
                gate = NS(type=UNITARY, params=[], n_controls=0, mat=list(pending[q].reshape(-1)),
                          perm=[], pauli="")
                out.append(NS(gate=gate, qubits=[q], clbits=[]))
            pending[q] = None

        for inst in instructions:
            g = inst.gate
            if _is_unitary(g) and g.n_controls == 0 and _base_qubits(g) == 1:
                q = int(inst.qubits[0])
                m = _gate_matrix(g)
                pending[q] = m if pending[q] is None else mm(m, pending[q])
                continue
            if int(g.type) == BARRIER:
                for q in range(n):
                    flush(q)
            else:
                for q in inst.qubits:
                    flush(int(q))
            out.append(inst)
        for q in range(n):
            flush(q)
        return out

    # ---- evolve (statevector_simulator.cpp:197-207)
    def evolve(self, instructions, n: int, state: Optional[np.ndarray] = None) -> np.ndarray:
        st = np.zeros(1 << n, dtype=np.complex128) if state is None else np.array(state, dtype=np.complex128)
        if state is None:
            st[0] = 1.0
        for inst in instructions:
            if int(inst.gate.type) == RESET:
                raise ValueError("run_statevector: Reset is non-deterministic; use run() instead")
            if _is_unitary(inst.gate):
                self.apply_instruction(st, inst)
        return st

    def run_statevector(self, circuit, fuse: bool = True, state=None) -> np.ndarray:
        insts = circuit.instructions()
        if fuse:
            insts = self.fuse_1q(insts, circuit.num_qubits())
        return self.evolve(insts, circuit.num_qubits(), state)

    # ---- run (statevector_simulator.cpp:232-265)
    def run(self, circuit, shots: int, seed: int, fuse: bool = True, channels=()) -> dict:
        """Counts {register int: count} with the reference's path selection and RNG order."""
        if shots == 0:
            raise ValueError("run: shots must be >= 1")
        n = circuit.num_qubits()
        noisy = len(channels) > 0
        insts = circuit.instructions() if noisy or not fuse else self.fuse_1q(circuit.instructions(), n)
        seen, per_shot = False, noisy
        for inst in insts:
            t = int(inst.gate.type)
            if t == MEASURE:
                seen = True
            elif t in (RESET, KRAUS):
                per_shot = True
            elif seen and _is_unitary(inst.gate):
                per_shot = True
        if not seen:
            raise ValueError("run: circuit has no measurements")
        rng = MT64(seed)
        if per_shot:
            return self._run_per_shot(insts, n, shots, rng, channels)
        st = self.evolve(insts, n)
        src = {}
        for inst in insts:
            if int(inst.gate.type) == MEASURE:
                src[int(inst.clbits[0])] = int(inst.qubits[0])
        cum = np.empty(st.size, dtype=np.float64)
        self.lib.orc_cumulative(st.ctypes.data, st.size, cum.ctypes.data)
        total = cum[-1]
        counts: dict[int, int] = {}
        for _ in range(shots):
            r = rng.uniform() * total
            idx = self.lib.orc_upper_bound(cum.ctypes.data, cum.size, r)
            reg = 0
            for c, q in src.items():
                if idx >> q & 1:
                    reg |= 1 << c
            counts[reg] = counts.get(reg, 0) + 1
        return counts

    def _branch(self, st, ops, q, rng):
        # sample_kraus_branch (statevector_simulator.cpp:122-144)
        r = rng.uniform()
        cum = 0.0
        chosen, chosen_p = None, 0.0
        for k in ops:
            kk = np.ascontiguousarray(np.asarray(k, dtype=np.complex128).reshape(4))
            p = self.lib.orc_kraus_probability(st.ctypes.data, st.size, q, kk.ctypes.data)
            if p <= 0.0:
                continue
            chosen, chosen_p = kk, p
            cum += p
            if r < cum:
                break
        if chosen is None:
            return
        inv = 1.0 / math.sqrt(chosen_p)
        m = np.ascontiguousarray(chosen * inv)
        self.lib.orc_apply_single_qubit(st.ctypes.data, st.size, q, m.ctypes.data)

    def _run_per_shot(self, insts, n, shots, rng, channels) -> dict:
        counts: dict[int, int] = {}
        for _ in range(shots):
            st = np.zeros(1 << n, dtype=np.complex128)
            st[0] = 1.0
            creg = 0
            for inst in insts:
                t = int(inst.gate.type)
                if t == MEASURE:
                    o = self.lib.orc_collapse_qubit(st.ctypes.data, st.size, int(inst.qubits[0]), rng.uniform())
                    c = int(inst.clbits[0])
                    creg = (creg | (1 << c)) if o else (creg & ~(1 << c))
                elif t == RESET:
                    self.lib.orc_reset_qubit(st.ctypes.data, st.size, int(inst.qubits[0]), rng.uniform())
                elif t == BARRIER:
                    pass
                elif t == KRAUS:
                    self._branch(st, inst.gate.kraus, int(inst.qubits[0]), rng)
                else:
                    self.apply_instruction(st, inst)
                    for ch in channels:
                        for q in inst.qubits:
                            self._branch(st, ch, int(q), rng)
            counts[creg] = counts.get(creg, 0) + 1
        return counts

    # ---- expectations (statevector.cpp:39-78, vqe.cpp:11-17)
    def expectation_value(self, st: np.ndarray, pauli: str) -> float:
        n = st.size.bit_length() - 1
        x, zy, ny = pauli_global_masks(pauli, n)
        return self.lib.orc_expectation(st.ctypes.data, st.size, x, zy, ny)

    def expectation(self, st: np.ndarray, hamiltonian) -> float:
        e = 0.0
        for c, p in hamiltonian:
            e += c * self.expectation_value(st, p)
        return e

    def parameter_shift_gradient(self, hamiltonian, pc, params) -> np.ndarray:
        """algorithms::parameter_shift_gradient (src/algorithms/vqe.cpp:68-94)."""
        theta = [float(v) for v in params]
        grad = np.zeros(len(theta))
        for k in range(len(theta)):
            saved = theta[k]
            theta[k] = saved + math.pi / 2
            ep = self.expectation(self.run_statevector(pc.bind(theta)), hamiltonian)
            theta[k] = saved - math.pi / 2
            em = self.expectation(self.run_statevector(pc.bind(theta)), hamiltonian)
            theta[k] = saved
            grad[k] = 0.5 * (ep - em)
        return grad


def dm_probabilities_numpy(instructions, n: int, channels=()) -> np.ndarray:
    """Exact outcome distribution of a noisy circuit by density-matrix evolution
    (DensityMatrixSimulator semantics, src/backend/density_matrix_simulator.cpp:8-24; the
    channels of the noise model follow every unitary on each touched qubit, explicit Kraus
    instructions apply where they stand).  Dense numpy, small n only."""
    dim = 1 << n
    rho = np.zeros((dim, dim), dtype=np.complex128)
    rho[0, 0] = 1.0

    def embed(m, qubits):
        # full 2^n operator of a gate on `qubits` (local bit j <-> qubits[j])
        k = len(qubits)
        full = np.zeros((dim, dim), dtype=np.complex128)
        others = [q for q in range(n) if q not in qubits]
        for col in range(dim):
            lc = sum(((col >> q) & 1) << j for j, q in enumerate(qubits))
            base = col & ~sum(1 << q for q in qubits)
            for lr in range(1 << k):
                row = base | sum(((lr >> j) & 1) << q for j, q in enumerate(qubits))
                full[row, col] += m[lr, lc]
        del others
        return full

    def channel(ops, q):
        nonlocal rho
        acc = np.zeros_like(rho)
        for k in ops:
            kk = embed(np.asarray(k, dtype=np.complex128).reshape(2, 2), [q])
            acc += kk @ rho @ kk.conj().T
        rho = acc

    for inst in instructions:
        g = inst.gate
        t = int(g.type)
        if t in (MEASURE, BARRIER):
            continue
        if t == KRAUS:
            channel(g.kraus, int(inst.qubits[0]))
            continue
        nc = g.n_controls
        base = _gate_matrix(g)
        k = base.shape[0].bit_length() - 1
        # controls in the low local bits (Gate::matrix, src/circuit/gate.cpp:203-226)
        dimf = 1 << (nc + k)
        cm = (1 << nc) - 1
        full_local = np.zeros((dimf, dimf), dtype=np.complex128)
        for col in range(dimf):
            if col & cm != cm:
                full_local[col, col] = 1
                continue
            tc = col >> nc
            for tr in range(1 << k):
                full_local[(tr << nc) | cm, col] = base[tr, tc]
        u = embed(full_local, [int(q) for q in inst.qubits])
        rho = u @ rho @ u.conj().T
        for ch in channels:
            for q in inst.qubits:
                channel(ch, int(q))
    return np.real(np.diag(rho)).copy()


class Ref:
    """The reference library built from its own sources (oracle/_ref/liblqcs_ref.so)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return REF_LIB.exists()

    def __init__(self):
        if Ref._lib is None:
            if not REF_LIB.exists():
                raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle ref`")
            lib = C.CDLL(str(REF_LIB))
            vp, u32, u64, d, i = C.c_void_p, C.c_uint32, C.c_uint64, C.c_double, C.c_int
            sig = {
                "lqcsref_last_error": (C.c_char_p, []),
                "lqcsref_set_threads": (None, [i]),
                "lqcsref_max_threads": (i, []),
                "lqcsref_run_statevector": (i, [u32, vp, u64, i, vp]),
                "lqcsref_run": (i, [u32, u32, vp, u64, u64, i, u64, i, u64, vp, vp, vp, u64, vp]),
                "lqcsref_dm_run": (i, [u32, u32, vp, u64, u64, i, u64, u64, vp, vp, vp, u64, vp]),
                "lqcsref_qasm_roundtrip": (i, [C.c_char_p, vp, u64]),
                "lqcsref_evolve_from": (i, [u32, vp, vp, u64, vp]),
                "lqcsref_time_apply": (i, [u32, vp, u64, u32, vp]),
                "lqcsref_expectation": (i, [u32, vp, C.c_char_p, vp]),
                "lqcsref_hamiltonian": (i, [u32, vp, u64, vp, vp, vp]),
                "lqcsref_parameter_shift": (i, [u32, vp, u64, vp, u64, u64, vp, vp, vp, vp]),
                "lqcsref_dm_probabilities": (i, [u32, vp, u64, u64, vp, vp]),
                "lqcsref_trajectories": (i, [u32, u32, vp, u64, u64, u64, u64, vp, vp]),
                "lqcsref_uniforms": (None, [u64, u64, vp]),
                "lqcsref_modexp_statevector": (i, [u64, u64, u32, u32, vp]),
                "lqcsref_shor": (i, [u64, u64, u64, i, u64, vp, vp, vp, u64, vp]),
            }
            for name, (res, args) in sig.items():
                f = getattr(lib, name)
                f.restype = res
                f.argtypes = args
            Ref._lib = lib
        self.lib = Ref._lib

    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = self.lib.lqcsref_last_error().decode()
            raise {1: ValueError, 2: IndexError}.get(rc, RuntimeError)(msg)

    def set_threads(self, n: int) -> None:
        self.lib.lqcsref_set_threads(n)

    def max_threads(self) -> int:
        return self.lib.lqcsref_max_threads()

    def run_statevector(self, circuit, fuse: bool = True) -> np.ndarray:
        arr, n, _k = circuit.c_instructions()
        out = np.empty(1 << circuit.num_qubits(), dtype=np.complex128)
        self._check(self.lib.lqcsref_run_statevector(circuit.num_qubits(), C.cast(arr, C.c_void_p),
                                                     n, int(fuse), out.ctypes.data))
        return out

    def run(self, circuit, shots: int, seed: Optional[int], fuse: bool = True, noise=None) -> dict:
        arr, n, _k = circuit.c_instructions()
        chp, nch, keep = (noise.c_channels() if noise is not None else (None, 0, []))
        cap = 1 << 20
        keys = np.zeros(min(cap, max(shots, 1)), dtype=np.uint64)
        counts = np.zeros_like(keys)
        nout = C.c_uint64(0)
        self._check(self.lib.lqcsref_run(circuit.num_qubits(), circuit.num_clbits(),
                                         C.cast(arr, C.c_void_p), n, shots,
                                         0 if seed is None else 1, 0 if seed is None else seed,
                                         int(fuse), nch, C.cast(chp, C.c_void_p) if chp else None,
                                         keys.ctypes.data, counts.ctypes.data, keys.size,
                                         C.byref(nout)))
        return {int(k): int(c) for k, c in zip(keys[: nout.value], counts[: nout.value])}

    def dm_run(self, circuit, shots: int, seed: Optional[int], noise=None) -> dict:
        """DensityMatrixSimulator::run counts {register int: count}."""
        arr, n, _k = circuit.c_instructions()
        chp, nch, keep = (noise.c_channels() if noise is not None else (None, 0, []))
        cap = 1 << 20
        keys = np.zeros(min(cap, max(shots, 1)), dtype=np.uint64)
        counts = np.zeros_like(keys)
        nout = C.c_uint64(0)
        self._check(self.lib.lqcsref_dm_run(circuit.num_qubits(), circuit.num_clbits(),
                                            C.cast(arr, C.c_void_p), n, shots,
                                            0 if seed is None else 1, 0 if seed is None else seed,
                                            nch, C.cast(chp, C.c_void_p) if chp else None,
                                            keys.ctypes.data, counts.ctypes.data, keys.size,
                                            C.byref(nout)))
        return {int(k): int(c) for k, c in zip(keys[: nout.value], counts[: nout.value])}

    def qasm_roundtrip(self, source: str) -> str:
        """io::to_qasm(io::from_qasm(source)) of the reference."""
        buf = C.create_string_buffer(1 << 22)
        self._check(self.lib.lqcsref_qasm_roundtrip(source.encode(), C.cast(buf, C.c_void_p),
                                                    len(buf)))
        return buf.value.decode()

    def evolve_from(self, circuit, state: np.ndarray) -> np.ndarray:
        arr, n, _k = circuit.c_instructions()
        src = np.ascontiguousarray(state, dtype=np.complex128)
        out = np.empty_like(src)
        self._check(self.lib.lqcsref_evolve_from(circuit.num_qubits(), src.ctypes.data,
                                                 C.cast(arr, C.c_void_p), n, out.ctypes.data))
        return out

    def time_apply(self, circuit, reps: int = 1) -> float:
        arr, n, _k = circuit.c_instructions()
        sec = C.c_double(0.0)
        self._check(self.lib.lqcsref_time_apply(circuit.num_qubits(), C.cast(arr, C.c_void_p), n,
                                                reps, C.byref(sec)))
        return sec.value

    def expectation_value(self, state: np.ndarray, pauli: str) -> float:
        n = state.size.bit_length() - 1
        out = C.c_double(0.0)
        src = np.ascontiguousarray(state, dtype=np.complex128)
        self._check(self.lib.lqcsref_expectation(n, src.ctypes.data, pauli.encode(), C.byref(out)))
        return out.value

    def expectation(self, state: np.ndarray, hamiltonian) -> float:
        n = state.size.bit_length() - 1
        coeffs = np.ascontiguousarray([c for c, _ in hamiltonian], dtype=np.float64)
        strs = [p.encode() for _, p in hamiltonian]
        arr = (C.c_char_p * max(1, len(strs)))(*strs)
        out = C.c_double(0.0)
        src = np.ascontiguousarray(state, dtype=np.complex128)
        self._check(self.lib.lqcsref_hamiltonian(n, src.ctypes.data, len(strs), coeffs.ctypes.data,
                                                 C.cast(arr, C.c_void_p), C.byref(out)))
        return out.value

    def parameter_shift_gradient(self, hamiltonian, pc, params) -> np.ndarray:
        arr, n, _k = pc.template().c_instructions()
        pinst = np.ascontiguousarray(pc.param_instructions(), dtype=np.uint64)
        coeffs = np.ascontiguousarray([c for c, _ in hamiltonian], dtype=np.float64)
        strs = [p.encode() for _, p in hamiltonian]
        parr = (C.c_char_p * max(1, len(strs)))(*strs)
        th = np.ascontiguousarray(params, dtype=np.float64)
        grad = np.zeros(max(1, th.size))
        self._check(self.lib.lqcsref_parameter_shift(pc.num_qubits(), C.cast(arr, C.c_void_p), n,
                                                     pinst.ctypes.data, pinst.size, len(strs),
                                                     coeffs.ctypes.data, C.cast(parr, C.c_void_p),
                                                     th.ctypes.data, grad.ctypes.data))
        return grad[: th.size]

    def dm_probabilities(self, circuit, noise=None) -> np.ndarray:
        arr, n, _k = circuit.c_instructions()
        chp, nch, keep = (noise.c_channels() if noise is not None else (None, 0, []))
        out = np.empty(1 << circuit.num_qubits())
        self._check(self.lib.lqcsref_dm_probabilities(circuit.num_qubits(), C.cast(arr, C.c_void_p), n,
                                                      nch, C.cast(chp, C.c_void_p) if chp else None,
                                                      out.ctypes.data))
        return out

    def trajectories(self, circuit, shots: int, seed: int, noise=None) -> np.ndarray:
        arr, n, _k = circuit.c_instructions()
        chp, nch, keep = (noise.c_channels() if noise is not None else (None, 0, []))
        regs = np.zeros(max(1, shots), dtype=np.uint64)
        self._check(self.lib.lqcsref_trajectories(circuit.num_qubits(), circuit.num_clbits(),
                                                  C.cast(arr, C.c_void_p), n, shots, seed, nch,
                                                  C.cast(chp, C.c_void_p) if chp else None,
                                                  regs.ctypes.data))
        return regs[:shots]

    def uniforms(self, seed: int, count: int) -> np.ndarray:
        out = np.empty(count)
        self.lib.lqcsref_uniforms(seed, count, out.ctypes.data)
        return out

    def modexp_statevector(self, a: int, N: int, n_count: int, n_work: int) -> np.ndarray:
        """run_statevector of X(work 0), H on the counting qubits and
        algorithms::modular_exponentiation(a, N, n_count, n_work)."""
        out = np.empty(1 << (n_count + n_work), dtype=np.complex128)
        self._check(self.lib.lqcsref_modexp_statevector(a, N, n_count, n_work, out.ctypes.data))
        return out

    def shor(self, N: int, shots: int = 64, max_attempts: int = 10,
             seed: Optional[int] = None) -> dict:
        """algorithms::shor: {success, factor1, factor2, a, period, attempts, counts}."""
        info = np.zeros(6, dtype=np.uint64)
        keys = np.zeros(max(shots, 1), dtype=np.uint64)
        counts = np.zeros_like(keys)
        nout = C.c_uint64(0)
        self._check(self.lib.lqcsref_shor(N, shots, max_attempts, 0 if seed is None else 1,
                                          0 if seed is None else seed, info.ctypes.data,
                                          keys.ctypes.data, counts.ctypes.data, keys.size,
                                          C.byref(nout)))
        return {"success": bool(info[0]), "factor1": int(info[1]), "factor2": int(info[2]),
                "a": int(info[3]), "period": int(info[4]), "attempts": int(info[5]),
                "counts": {int(k): int(c) for k, c in zip(keys[: nout.value], counts[: nout.value])}}

"""Statevector, Result and StatevectorSimulator — the drop-in of lqcs's statevector backend
(include/lqcs/backend/statevector_simulator.hpp:17-42, python/src/bindings.cpp:149-222),
with the state held in device memory and every computation done by the engine's CUDA
kernels through the C ABI.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _native as N
from .circuit import QuantumCircuit
from .noise import NoiseModel


class Statevector:
    """A 2^n complex128 state resident on the current CUDA device (lqcs::Statevector,
    include/lqcs/backend/statevector.hpp:12-37).  ``to_numpy()`` copies to the host; the
    device buffer itself is exposed through ``__cuda_array_interface__`` / ``to_torch()``
    for zero-copy use."""

    def __init__(self, num_qubits: int = 0, *, _handle=None):
        if _handle is not None:
            self._h = _handle
        else:
            if num_qubits == 0:
                raise ValueError("Statevector: num_qubits must be >= 1")
            h = N.StatePtr()
            N.call("lqcs_state_create", int(num_qubits), None, C.byref(h))
            self._h = h
        n = C.c_uint32(0)
        N.call("lqcs_state_num_qubits", self._h, C.byref(n))
        self._n = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and N._lib is not None:
            N._lib.lqcs_state_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def num_qubits(self) -> int:
        return self._n

    def __len__(self) -> int:
        return 1 << self._n

    def size(self) -> int:
        return 1 << self._n

    def __getitem__(self, i: int) -> complex:
        i = int(i)
        if i < 0 or i >= len(self):
            raise IndexError("statevector index out of range")
        buf = np.zeros(1, dtype=np.complex128)
        N.call("lqcs_state_read_range", self._h, i, 1, buf.ctypes.data)
        return complex(buf[0])

    def norm(self) -> float:
        out = C.c_double(0.0)
        N.call("lqcs_state_norm", self._h, C.byref(out))
        return out.value

    def probabilities(self) -> np.ndarray:
        out = np.empty(len(self), dtype=np.float64)
        N.call("lqcs_state_probabilities", self._h, out.ctypes.data)
        return out

    def expectation_value(self, pauli: str) -> float:
        out = C.c_double(0.0)
        N.call("lqcs_state_expectation_pauli", self._h, pauli.encode(), C.byref(out))
        return out.value

    def to_numpy(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(len(self), dtype=np.complex128)
        if out.dtype != np.complex128 or out.size != len(self) or not out.flags.c_contiguous:
            raise ValueError("to_numpy: out must be a contiguous complex128 array of 2^n entries")
        N.call("lqcs_state_store", self._h, out.ctypes.data, len(self))
        return out

    def load(self, amps) -> "Statevector":
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128).reshape(-1))
        N.call("lqcs_state_load", self._h, a.ctypes.data, a.size)
        return self

    @classmethod
    def from_numpy(cls, amps) -> "Statevector":
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128).reshape(-1))
        n = a.size.bit_length() - 1
        if a.size != (1 << n) or n == 0:
            raise ValueError("from_numpy: length must be a power of two >= 2")
        sv = cls(n)
        return sv.load(a)

    def device_ptr(self) -> int:
        p = C.c_void_p()
        N.call("lqcs_state_device_ptr", self._h, C.byref(p))
        return int(p.value or 0)

    @property
    def __cuda_array_interface__(self):
        return {"shape": (len(self),), "typestr": "<c16", "data": (self.device_ptr(), False),
                "version": 3, "strides": None}

    def to_torch(self):
        """Zero-copy torch view of the device amplitudes (complex128)."""
        import torch
        return torch.as_tensor(self, device="cuda")

    def apply(self, circuit: QuantumCircuit, fuse_gates: bool = True, max_fusion_width: int = 0,
              fusion_mode: int = 0) -> "Statevector":
        """Evolve this state in place by the unitary instructions of `circuit`."""
        if circuit.num_qubits() != self._n:
            raise ValueError("apply: circuit and state have different qubit counts")
        arr, n, _keep = circuit.c_instructions()
        N.call("lqcs_state_apply", self._h, arr, n, int(fuse_gates), int(max_fusion_width),
               int(fusion_mode))
        return self

    def collapse(self, qubit: int, uniform: float) -> int:
        out = C.c_int32(0)
        N.call("lqcs_state_collapse", self._h, int(qubit), float(uniform), C.byref(out))
        return out.value

    def reset_qubit(self, qubit: int, uniform: float) -> None:
        N.call("lqcs_state_reset_qubit", self._h, int(qubit), float(uniform))

    def kraus_probability(self, qubit: int, k) -> float:
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.complex128).reshape(4)).view(np.float64)
        out = C.c_double(0.0)
        N.call("lqcs_state_kraus_probability", self._h, int(qubit), kk.ctypes.data, C.byref(out))
        return out.value

    def sample(self, uniforms) -> tuple[np.ndarray, float]:
        """Basis indices upper_bound(cumsum(|a|^2), u * total) for each uniform, and the
        smallest relative distance of a scaled uniform from a bin edge."""
        u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64))
        idx = np.empty(u.size, dtype=np.uint64)
        margin = C.c_double(0.0)
        N.call("lqcs_state_sample", self._h, u.ctypes.data, u.size, idx.ctypes.data,
               C.byref(margin))
        return idx, margin.value


class CompiledCircuit:
    """A circuit fused and lowered once (``lqcs_program_create``); ``apply`` then costs only
    kernel launches.  fusion_mode: 0 default, 1 greedy, 2 learned, 3 gate by gate, 4 tile
    passes, 5 autotuned (see autotune)."""

    def __init__(self, circuit: QuantumCircuit, fuse_gates: bool = True, max_fusion_width: int = 0,
                 fusion_mode: int = 0):
        arr, n, _keep = circuit.c_instructions()
        h = N.ProgramPtr()
        N.call("lqcs_program_create", circuit.num_qubits(), arr, n, int(fuse_gates),
               int(max_fusion_width), int(fusion_mode), C.byref(h))
        self._h = h
        self.num_qubits = circuit.num_qubits()
        ops, gates = C.c_uint64(0), C.c_uint64(0)
        N.call("lqcs_program_info", self._h, C.byref(ops), C.byref(gates))
        self.n_ops = ops.value
        self.n_gates = gates.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and N._lib is not None:
            N._lib.lqcs_program_destroy(h)
            self._h = None

    def apply(self, sv: "Statevector") -> "Statevector":
        N.call("lqcs_program_apply", sv.handle, self._h)
        return sv

    def profile(self, sv: "Statevector") -> list:
        """Apply once with CUDA-event timing per operation: list of dicts."""
        cap = max(1, self.n_ops)
        arr = (N.OpProfile * cap)()
        n = C.c_uint64(0)
        N.call("lqcs_program_apply_profiled", sv.handle, self._h, cap, arr, C.byref(n))
        out = []
        for i in range(min(n.value, cap)):
            r = arr[i]
            name = N.OP_KIND_NAMES.get(r.kind, str(r.kind))
            if r.kind in (2, 3):
                name += f"<{r.n_targets}>"
            out.append({"kernel": name, "kind": r.kind, "width": r.n_targets, "gates": r.n_gates,
                        "min_target": r.min_target, "max_target": r.max_target,
                        "controls": r.n_controls, "ms": r.device_ms, "alg_bytes": r.alg_bytes,
                        "alg_flops": r.alg_flops})
        return out


class Result:
    """lqcs::Result (include/lqcs/result/result.hpp:12-28): counts keyed by bit strings with
    the highest classical bit leftmost."""

    def __init__(self, counts: dict, shots: int):
        self._counts = dict(sorted(counts.items()))
        self._shots = int(shots)

    def counts(self) -> dict:
        return dict(self._counts)

    def shots(self) -> int:
        return self._shots

    def probabilities(self) -> dict:
        if self._shots == 0:
            return {}
        return {k: v / self._shots for k, v in self._counts.items()}

    def __repr__(self) -> str:
        body = ", ".join(f"'{k}': {v}" for k, v in self._counts.items())
        return f"<Result shots={self._shots} {{{body}}}>"


_PLANNERS = {0: "register tile passes", 1: "shared-memory tile passes", 2: "greedy blocks"}


def autotune(circuit) -> list:
    """Time every candidate fusion plan of the circuit's unitary part on a scratch state
    (lqcs_autotune) and remember the fastest: ``fusion_mode=5`` then uses it.  One dict per
    candidate; empty when no scratch state fits in device memory."""
    arr, n, _keep = circuit.c_instructions()
    cap = 32
    out = (N.TuneEntry * cap)()
    cnt = C.c_uint64(0)
    N.call("lqcs_autotune", circuit.num_qubits(), arr, n, cap, out, C.byref(cnt))
    res = []
    for i in range(min(cnt.value, cap)):
        e = out[i]
        res.append({"planner": _PLANNERS.get(e.planner, str(e.planner)), "tile_bits": e.tile_bits,
                    "tile_low": e.tile_low, "inner": e.inner, "width": e.width,
                    "chosen": bool(e.chosen), "n_ops": e.n_ops, "ms": e.device_ms})
    return res


def registers_to_counts(regs: np.ndarray, n_clbits: int) -> dict:
    """Count per-shot classical registers as the reference's MSB-left key strings."""
    vals, cnt = np.unique(regs, return_counts=True)
    if n_clbits == 0:
        return {"": int(cnt.sum())} if vals.size else {}
    # all keys at once: the bits as ASCII digits, MSB first, cut into n_clbits-wide strings
    shifts = np.arange(n_clbits - 1, -1, -1, dtype=np.uint64)
    digits = ((vals.astype(np.uint64)[:, None] >> shifts) & np.uint64(1)).astype(np.uint8) + 48
    text = digits.tobytes().decode()
    keys = [text[i:i + n_clbits] for i in range(0, len(text), n_clbits)]
    return dict(zip(keys, cnt.tolist()))


class StatevectorSimulator:
    """Drop-in for lqcs::StatevectorSimulator with the pylqcs keyword arguments
    (seed, fuse_gates, num_threads, noise).  Extra engine knobs: max_fusion_width,
    fusion_mode (0 default, 1 greedy, 2 learned cost model, 3 gate by gate, 4 tile passes,
    5 autotuned)."""

    def __init__(self, seed: Optional[int] = None, fuse_gates: bool = True, num_threads: int = 0,
                 noise: Optional[NoiseModel] = None, *, max_fusion_width: int = 0,
                 fusion_mode: int = 0, max_resident: int = 0):
        self.seed = seed
        self.fuse_gates = bool(fuse_gates)
        self.num_threads = int(num_threads)
        self.noise = noise if noise is not None else NoiseModel()
        self.max_fusion_width = int(max_fusion_width)
        self.fusion_mode = int(fusion_mode)
        self.max_resident = int(max_resident)

    def name(self) -> str:
        return "statevector_simulator"

    def _options(self, shot_offset: int = 0):
        o = N.SimOptions()
        o.shot_offset = int(shot_offset)
        o.has_seed = 0 if self.seed is None else 1
        o.seed = 0 if self.seed is None else int(self.seed) & 0xFFFFFFFFFFFFFFFF
        o.fuse_gates = int(self.fuse_gates)
        o.num_threads = self.num_threads
        o.max_fusion_width = self.max_fusion_width
        o.fusion_mode = self.fusion_mode
        o.max_resident = self.max_resident
        ptr, n, keep = self.noise.c_channels()
        o.n_channels = n
        if ptr is not None:
            o.channels = ptr
        return o, keep

    def run_statevector(self, circuit: QuantumCircuit) -> Statevector:
        opts, keep = self._options()
        arr, n, _k = circuit.c_instructions()
        h = N.StatePtr()
        N.call("lqcs_run_statevector", circuit.num_qubits(), arr, n, C.byref(opts), None,
               C.byref(h))
        return Statevector(_handle=h)

    def run(self, circuit: QuantumCircuit, shots: int = 1024) -> Result:
        opts, keep = self._options()
        arr, n, _k = circuit.c_instructions()
        regs = np.zeros(max(int(shots), 1), dtype=np.uint64)
        N.call("lqcs_run", circuit.num_qubits(), circuit.num_clbits(), arr, n, int(shots),
               C.byref(opts), regs.ctypes.data)
        return Result(registers_to_counts(regs[:shots], circuit.num_clbits()), shots)

    def run_registers(self, circuit: QuantumCircuit, shots: int = 1024,
                      shot_offset: int = 0) -> np.ndarray:
        """Per-shot classical registers (clbit c -> bit c) in shot order.  With shot_offset,
        these are shots shot_offset .. shot_offset + shots - 1 of the seeded run (the
        uniforms of the earlier shots are skipped): consecutive ranges concatenate to one
        run, which is how sharding.sharded_run_registers splits shots over ranks."""
        opts, keep = self._options(shot_offset)
        arr, n, _k = circuit.c_instructions()
        regs = np.zeros(max(int(shots), 1), dtype=np.uint64)
        N.call("lqcs_run", circuit.num_qubits(), circuit.num_clbits(), arr, n, int(shots),
               C.byref(opts), regs.ctypes.data)
        return regs[:shots]


class DensityMatrix:
    """lqcs::DensityMatrix (include/lqcs/backend/density_matrix.hpp) held on the device as a
    2n-qubit vector: element rho_{rc} at index (c << n) | r."""

    def __init__(self, state: Statevector, num_qubits: int):
        self._sv = state
        self._n = int(num_qubits)

    def num_qubits(self) -> int:
        return self._n

    def dim(self) -> int:
        return 1 << self._n

    def probabilities(self) -> np.ndarray:
        out = np.empty(self.dim(), dtype=np.float64)
        N.call("lqcs_dm_probabilities", self._sv.handle, out.ctypes.data)
        return out

    def to_numpy(self) -> np.ndarray:
        """rho as a dim x dim host matrix."""
        d = self.dim()
        return self._sv.to_numpy().reshape(d, d).T.copy()

    def element(self, row: int, col: int) -> complex:
        d = self.dim()
        if not (0 <= row < d and 0 <= col < d):
            raise IndexError("DensityMatrix::element: index out of range")
        return complex(self._sv[(col << self._n) | row])

    def trace(self) -> float:
        return float(self.probabilities().sum())

    def purity(self) -> float:
        """Tr(rho^2) = sum |rho_rc|^2 (rho Hermitian)."""
        return float(self._sv.norm() ** 2)


class DensityMatrixSimulator:
    """Drop-in for lqcs::DensityMatrixSimulator (seed, noise): run() samples the final
    diagonal (terminal measurements only), run_density_matrix() returns rho."""

    def __init__(self, seed: Optional[int] = None, noise: Optional[NoiseModel] = None):
        self._sim = StatevectorSimulator(seed=seed, noise=noise)

    def name(self) -> str:
        return "density_matrix_simulator"

    def run_density_matrix(self, circuit: QuantumCircuit) -> DensityMatrix:
        opts, keep = self._sim._options()
        arr, n, _k = circuit.c_instructions()
        h = N.StatePtr()
        N.call("lqcs_dm_create", circuit.num_qubits(), arr, n, C.byref(opts), C.byref(h))
        return DensityMatrix(Statevector(_handle=h), circuit.num_qubits())

    def run_registers(self, circuit: QuantumCircuit, shots: int = 1024,
                      shot_offset: int = 0) -> np.ndarray:
        opts, keep = self._sim._options(shot_offset)
        arr, n, _k = circuit.c_instructions()
        regs = np.zeros(max(int(shots), 1), dtype=np.uint64)
        N.call("lqcs_dm_run", circuit.num_qubits(), circuit.num_clbits(), arr, n, int(shots),
               C.byref(opts), regs.ctypes.data)
        return regs[:shots]

    def run(self, circuit: QuantumCircuit, shots: int = 1024) -> Result:
        return Result(registers_to_counts(self.run_registers(circuit, shots), circuit.num_clbits()),
                      shots)

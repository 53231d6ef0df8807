"""Algorithms on the hot path: expectation values, gradients and the QFT circuit builder
(lqcs::algorithms, src/algorithms/vqe.cpp and src/algorithms/qft.cpp)."""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence

import numpy as np

from . import _native as N
from .circuit import ParametricCircuit, QuantumCircuit
from .simulator import Statevector, StatevectorSimulator


def _hamiltonian(terms):
    """[(coeff, pauli), ...] -> (lqcs_hamiltonian, keepalive)."""
    terms = list(terms)
    coeffs = np.ascontiguousarray([float(c) for c, _ in terms], dtype=np.float64)
    strs = [p.encode() for _, p in terms]
    arr = (C.c_char_p * max(1, len(strs)))(*strs)
    h = N.HamiltonianC()
    h.n_terms = len(terms)
    h.coeffs = coeffs.ctypes.data_as(C.POINTER(C.c_double))
    h.paulis = C.cast(arr, C.POINTER(C.c_char_p))
    return h, [coeffs, strs, arr]


def expectation(statevector: Statevector, hamiltonian) -> float:
    """<psi|H|psi>, hamiltonian = [(coeff, pauli_str), ...] (src/algorithms/vqe.cpp:11-17)."""
    terms = list(hamiltonian)
    if not terms:
        return 0.0
    coeffs = np.ascontiguousarray([float(c) for c, _ in terms], dtype=np.float64)
    strs = [p.encode() for _, p in terms]
    arr = (C.c_char_p * len(strs))(*strs)
    total = C.c_double(0.0)
    N.call("lqcs_state_expectation_terms", statevector.handle, arr, coeffs.ctypes.data,
           len(terms), None, C.byref(total))
    return total.value


def expectation_terms(statevector: Statevector, paulis: Sequence[str]) -> np.ndarray:
    """<psi|P_t|psi> for every Pauli string."""
    strs = [p.encode() for p in paulis]
    if not strs:
        return np.zeros(0)
    arr = (C.c_char_p * len(strs))(*strs)
    coeffs = np.zeros(len(strs))
    out = np.zeros(len(strs))
    N.call("lqcs_state_expectation_terms", statevector.handle, arr, coeffs.ctypes.data,
           len(strs), out.ctypes.data, None)
    return out


def parameter_shift_gradient(hamiltonian, ansatz: ParametricCircuit, params) -> list:
    """Analytic dE/dtheta by the parameter-shift rule, evaluated circuit by circuit on the
    GPU (the algorithm of src/algorithms/vqe.cpp:68-94)."""
    params = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
    if params.size != ansatz.num_parameters():
        raise ValueError("parameter_shift_gradient: params size must equal num_parameters")
    h, keep_h = _hamiltonian(hamiltonian)
    pc, keep_p = ansatz.c_struct()
    grad = np.zeros(max(1, params.size))
    N.call("lqcs_parameter_shift_gradient", C.byref(pc), C.byref(h), params.ctypes.data,
           grad.ctypes.data)
    return grad[: params.size].tolist()


def _parameter_sets(params, n_params: int):
    """params as (B, P) float64 and whether a single (P,) set was given; an ansatz without
    parameters takes (0,) for one set or (B, 0) for B sets."""
    p = np.asarray(params, dtype=np.float64)
    single = p.ndim <= 1
    if n_params == 0:
        sets = 1 if single else p.shape[0]
        return np.zeros((sets, 0)), single
    return np.ascontiguousarray(p.reshape(-1, n_params)), single


def adjoint_gradient(hamiltonian, ansatz: ParametricCircuit, params, max_resident: int = 0):
    """Batched adjoint-state gradients.  params: (P,) or (B, P).  Returns
    (energies (B,), gradients (B, P)) as numpy arrays (squeezed for a single set)."""
    p, single = _parameter_sets(params, ansatz.num_parameters())
    if p.shape[1] != ansatz.num_parameters():
        raise ValueError("adjoint_gradient: params size must equal num_parameters")
    b = p.shape[0]
    h, keep_h = _hamiltonian(hamiltonian)
    pc, keep_p = ansatz.c_struct()
    energies = np.zeros(b)
    grads = np.zeros((b, ansatz.num_parameters()))
    N.call("lqcs_adjoint_gradient", C.byref(pc), C.byref(h), p.ctypes.data, b, int(max_resident),
           energies.ctypes.data, grads.ctypes.data)
    if single:
        return float(energies[0]), grads[0]
    return energies, grads


def adjoint_gradient_multi(problems) -> list:
    """Adjoint gradients of several problems of different qubit counts in one call.
    problems: [(hamiltonian, ansatz, params (B, P) or (P,)), ...].  All problems run as one
    captured CUDA graph, replayed on later calls with the same problems (new parameter values
    allowed).  Returns [(energies (B,), gradients (B, P)), ...] in problem order."""
    keep, pcs, hs, ps, outs_e, outs_g = [], [], [], [], [], []
    batches = np.zeros(len(problems), dtype=np.uint64)
    for i, (ham, ansatz, params) in enumerate(problems):
        p, _ = _parameter_sets(params, ansatz.num_parameters())
        h, kh = _hamiltonian(ham)
        pc, kp = ansatz.c_struct()
        e = np.zeros(p.shape[0])
        g = np.zeros((p.shape[0], ansatz.num_parameters()))
        keep += [p, h, kh, pc, kp, e, g]
        pcs.append(C.addressof(pc))
        hs.append(C.addressof(h))
        ps.append(p.ctypes.data)
        outs_e.append(e)
        outs_g.append(g)
        batches[i] = p.shape[0]
    n = len(problems)
    arr = lambda xs: (C.c_void_p * max(n, 1))(*xs)   # noqa: E731
    a_pc, a_h, a_p = arr(pcs), arr(hs), arr(ps)
    a_e = arr([e.ctypes.data for e in outs_e])
    a_g = arr([g.ctypes.data if g.size else None for g in outs_g])
    N.call("lqcs_adjoint_gradient_multi", n, a_pc, a_h, a_p, batches.ctypes.data, a_e, a_g)
    return list(zip(outs_e, outs_g))


def release_caches() -> None:
    """Free the device memory kept between gradient calls (cached plans and graphs) and the
    autotuner's remembered choices."""
    N.call("lqcs_release_caches")


def batched_energy(hamiltonian, ansatz: ParametricCircuit, params, max_resident: int = 0):
    """Energies of B parameter sets (the forward pass of adjoint_gradient)."""
    p, _ = _parameter_sets(params, ansatz.num_parameters())
    h, keep_h = _hamiltonian(hamiltonian)
    pc, keep_p = ansatz.c_struct()
    energies = np.zeros(p.shape[0])
    N.call("lqcs_batched_energy", C.byref(pc), C.byref(h), p.ctypes.data, p.shape[0],
           int(max_resident), energies.ctypes.data)
    return energies


def qft(n: int, do_swaps: bool = True) -> QuantumCircuit:
    """QFT(n) circuit: H and controlled-phase ladder from the highest qubit down, then the
    reversal swaps (src/algorithms/qft.cpp:7-23)."""
    qc = QuantumCircuit(n)
    for i in range(n - 1, -1, -1):
        qc.h(i)
        for j in range(i - 1, -1, -1):
            qc.cp(math.pi / float(1 << (i - j)), j, i)
    if do_swaps:
        for i in range(n // 2):
            qc.swap(i, n - 1 - i)
    return qc


def qft_inverse(n: int, do_swaps: bool = True) -> QuantumCircuit:
    return qft(n, do_swaps).inverse()


def vqe_gradient_descent(hamiltonian, ansatz: ParametricCircuit, max_iterations: int = 200,
                         learning_rate: float = 0.1, tol: float = 1e-9,
                         initial_parameters: Sequence[float] = ()):
    """Gradient-descent VQE (src/algorithms/vqe.cpp:96-133) with GPU adjoint gradients."""
    n = ansatz.num_parameters()
    if n == 0:
        raise ValueError("vqe_gradient_descent: ansatz has no parameters")
    theta = np.array(initial_parameters, dtype=np.float64) if len(initial_parameters) else np.zeros(n)
    if theta.size != n:
        raise ValueError("vqe_gradient_descent: initial_parameters size must equal num_parameters")
    history = []
    iterations = 0
    for it in range(max_iterations):
        _, g = adjoint_gradient(hamiltonian, ansatz, theta)
        theta = theta - learning_rate * g
        e, _ = adjoint_gradient(hamiltonian, ansatz, theta)
        history.append(e)
        iterations = it + 1
        if math.sqrt(float(np.dot(g, g))) < tol:
            break
    energy = history[-1] if history else adjoint_gradient(hamiltonian, ansatz, theta)[0]
    return {"energy": energy, "parameters": theta.tolist(), "iterations": iterations,
            "history": history}

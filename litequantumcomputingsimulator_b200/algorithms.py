"""Algorithms on the hot path: expectation values, gradients, the QFT circuit builder and
Shor's period finding over controlled permutations (lqcs::algorithms,
src/algorithms/vqe.cpp, qft.cpp, arithmetic.cpp, number_theory.cpp, shor.cpp)."""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence

import numpy as np

from dataclasses import dataclass, field
from typing import Optional

from . import _native as N
from .circuit import Gate, GateType, Instruction, ParametricCircuit, QuantumCircuit
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


# ---------------------------------------------------------------- number theory
# lqcs::algorithms::number_theory (src/algorithms/number_theory.cpp): exact integer forms.

def gcd(a: int, b: int) -> int:
    return math.gcd(int(a), int(b))


def pow_mod(base: int, exp: int, mod: int) -> int:
    return pow(int(base), int(exp), int(mod))


def is_prime(n: int) -> bool:
    """Trial division by odd numbers up to sqrt(n) (src/algorithms/number_theory.cpp:44-51)."""
    if n < 2:
        return False
    if n % 2 == 0:
        return n == 2
    d = 3
    while d * d <= n:
        if n % d == 0:
            return False
        d += 2
    return True


def perfect_power_base(n: int) -> int:
    """b if n = b^k for some k >= 2 (the smallest such k), else 0
    (src/algorithms/number_theory.cpp:53-70: k from 2 while 2^k <= n; the reference rounds a
    floating k-th root and checks its neighbours, which for n < 2^53 finds the same b as the
    exact integer root used here)."""
    if n < 4:
        return 0
    k = 2
    while (1 << k) <= n:
        b = _iroot(n, k)
        for cand in (b, b + 1):
            if cand >= 2 and cand ** k == n:
                return cand
        k += 1
    return 0


def _iroot(n: int, k: int) -> int:
    """floor(n^(1/k)) by Newton's method on integers."""
    if n < 2:
        return n
    x = 1 << ((n.bit_length() + k - 1) // k)
    while True:
        y = ((k - 1) * x + n // x ** (k - 1)) // k
        if y >= x:
            return x
        x = y


def continued_fraction_denominators(num: int, den: int, max_denominator: int) -> list:
    """Denominators q_i = a_i q_{i-1} + q_{i-2} (q_{-1} = 0, q_{-2} = 1) of the convergents
    of num/den, stopping before the first one above max_denominator
    (src/algorithms/number_theory.cpp:72-89)."""
    out = []
    km1, km2 = 0, 1
    while den != 0:
        a, rem = divmod(num, den)
        num, den = den, rem
        k = a * km1 + km2
        if k > max_denominator:
            break
        out.append(k)
        km2, km1 = km1, k
    return out


# ---------------------------------------------------------------- modular exponentiation

def modular_exponentiation(a: int, N: int, n_counting: int, n_work: int) -> QuantumCircuit:
    """|c>|y> -> |c>|a^c y mod N> on counting register [0, n_counting) and work register
    [n_counting, n_counting + n_work) (src/algorithms/arithmetic.cpp:10-43): one singly
    controlled permutation per counting qubit j, y -> a^(2^j) y mod N for y < N and the
    identity on y >= N.  The engine applies each as a controlled permutation of the work
    register (cycles in shared memory)."""
    a, N = int(a), int(N)
    if N < 2 or (1 << n_work) < N:
        raise ValueError("modular_exponentiation: work register too small for N")
    if math.gcd(a % N, N) != 1:
        raise ValueError("modular_exponentiation: gcd(a, N) must be 1 (else not a bijection)")
    qc = QuantumCircuit(n_counting + n_work)
    work = [n_counting + w for w in range(n_work)]
    dim = 1 << n_work
    for j in range(n_counting):
        factor = pow(a, 1 << j, N)
        table = [(factor * y) % N if y < N else y for y in range(dim)]
        qc.append(Instruction(Gate(GateType.Permutation, [], 1, [], table), [j] + work))
    return qc


# ---------------------------------------------------------------- Shor

class _Mt64Stream:
    """Sequential raw draws of std::mt19937_64(seed), the engine of lqcs::Rng."""

    def __init__(self, seed: int):
        self.seed = int(seed) & ((1 << 64) - 1)
        self.pos = 0
        self.buf = np.zeros(0, dtype=np.uint64)
        self.base = 0

    def __call__(self) -> int:
        if self.pos >= self.base + self.buf.size:
            self.base = self.pos
            self.buf = np.empty(64, dtype=np.uint64)
            N.call("lqcs_rng_u64", self.seed, self.base, self.buf.size, self.buf.ctypes.data)
        v = int(self.buf[self.pos - self.base])
        self.pos += 1
        return v

    def uniform_int(self, lo: int, hi: int) -> int:
        """std::uniform_int_distribution<uint64_t>(lo, hi) over this 64-bit engine, as
        libstdc++ 13 computes it: Lemire's multiply-and-reject downscaling (D. Lemire, "Fast
        Random Integer Generation in an Interval", ACM TOMACS 29(1), 2019) on range
        hi - lo + 1, one or more draws."""
        rng = hi - lo + 1
        mask = (1 << 64) - 1
        product = self() * rng
        low = product & mask
        if low < rng:
            threshold = ((1 << 64) - rng) % rng
            while low < threshold:
                product = self() * rng
                low = product & mask
        return lo + (product >> 64)


@dataclass
class ShorResult:
    """lqcs::algorithms::ShorResult (include/lqcs/algorithms/shor.hpp)."""
    success: bool = False
    N: int = 0
    factor1: int = 0
    factor2: int = 0
    a: int = 0
    period: int = 0
    attempts: int = 0
    counts: dict = field(default_factory=dict)
    circuit: Optional[QuantumCircuit] = None


def _try_period(N: int, a: int, r: int, res: ShorResult) -> bool:
    """Factors from a candidate period r (src/algorithms/shor.cpp:22-39)."""
    if r == 0 or r >= N or pow(a, r, N) != 1 or r % 2 != 0:
        return False
    x = pow(a, r // 2, N)
    if x == N - 1:
        return False
    for f in (math.gcd(x - 1, N), math.gcd(x + 1, N)):
        if f != 1 and f != N:
            res.factor1, res.factor2 = min(f, N // f), max(f, N // f)
            res.period = r
            return True
    return False


def shor(N: int, shots: int = 64, max_attempts: int = 10,
         seed: Optional[int] = None) -> ShorResult:
    """Shor's factoring (src/algorithms/shor.cpp:43-129): classical shortcuts (even N, prime
    N, perfect powers, a lucky gcd), then per attempt a base a drawn from lqcs::Rng(seed),
    period finding on the GPU (H on 2w counting qubits, the controlled modular
    multiplications, inverse QFT, `shots` measurements with a simulator seeded by the next
    raw draw), and continued-fraction post-processing of the outcomes by decreasing count,
    trying multiples 1..4 of each convergent's denominator.  With a seed, every field equals
    the reference's."""
    N = int(N)
    res = ShorResult(N=N)
    if N < 4:
        raise ValueError("shor: N must be >= 4")
    if N % 2 == 0:
        res.success, res.factor1, res.factor2 = True, 2, N // 2
        return res
    if is_prime(N):
        return res
    b = perfect_power_base(N)
    if b:
        res.success, res.factor1, res.factor2 = True, min(b, N // b), max(b, N // b)
        return res
    n_work = N.bit_length()
    n_count = 2 * n_work   # 3 * bit_length(N) qubits: up to N < 2^11 (33 qubits) on one B200
    count_dim = 1 << n_count
    rng = _Mt64Stream(seed if seed is not None else int.from_bytes(np.random.bytes(8), "little"))
    for attempt in range(max_attempts):
        res.attempts = attempt + 1
        a = rng.uniform_int(2, N - 2)
        res.a = a
        g = math.gcd(a, N)
        if g != 1:
            res.success, res.factor1, res.factor2 = True, min(g, N // g), max(g, N // g)
            res.period = 0
            return res
        qc = QuantumCircuit(n_count + n_work, n_count)
        qc.x(n_count)
        for j in range(n_count):
            qc.h(j)
        qc.compose(modular_exponentiation(a, N, n_count, n_work))
        qc.compose(qft_inverse(n_count))
        for j in range(n_count):
            qc.measure(j, j)
        counts = StatevectorSimulator(seed=rng()).run(qc, shots).counts()
        outcomes = sorted(((c, int(k, 2)) for k, c in counts.items()), reverse=True)
        for _, m in outcomes:
            if m == 0:
                continue
            for r_base in continued_fraction_denominators(m, count_dim, N):
                for k in range(1, 5):
                    if _try_period(N, a, k * r_base, res):
                        res.success = True
                        res.counts = counts
                        res.circuit = qc
                        return res
    return res

"""The allocation-free expectation entry point (lqcs_expectation_terms_noalloc).

It exists for callers that cannot allocate device memory — code inside a pool or arena that
owns the whole device, an embedding that forbids cudaMalloc after start-up — and keeps its
partial sums in a static device array of the library.  It is an ordinary host call (it waits
for its stream), never one made inside stream capture or a CUDA host function.  Its
results must equal those of the regular entry point (lqcs_state_expectation_terms) within
the expectation tolerance of the other tests, on consecutive calls that reuse the array.
This file is collected last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import _native as N
from litequantumcomputingsimulator_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _strings(paulis):
    enc = [p.encode() for p in paulis]
    return (C.c_char_p * max(1, len(enc)))(*enc), enc


def regular(sv, paulis):
    arr, _keep = _strings(paulis)
    out = np.zeros(len(paulis))
    coeffs = np.zeros(len(paulis))
    N.call("lqcs_state_expectation_terms", sv.handle, arr, coeffs.ctypes.data, len(paulis),
           out.ctypes.data, None)
    return out


def noalloc(sv, paulis):
    arr, _keep = _strings(paulis)
    out = np.full(len(paulis), np.nan)
    N.call("lqcs_expectation_terms_noalloc", C.c_void_p(sv.device_ptr()), sv.num_qubits(), arr,
           len(paulis), out.ctypes.data, None)
    return out


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    rng = np.random.default_rng(5)
    # first call: 16 terms on a 14-qubit state; second call: fewer terms on another state,
    # so a stale value left in the shared array from the first call would show up
    cases = [(14, 16, 1), (17, 9, 2)]
    for n, n_terms, seed in cases:
        sv = lq.Statevector.from_numpy(W.gaussian_state(n, seed=seed))
        paulis = ["".join("IXYZ"[i] for i in rng.integers(0, 4, n)) for _ in range(n_terms)]
        want = regular(sv, paulis)
        got = noalloc(sv, paulis)
        assert np.max(np.abs(got - want)) < TOL


def test_noalloc_rejects_too_many_terms():
    sv = lq.Statevector(6)
    with pytest.raises(ValueError, match="at most 16 Pauli terms"):
        noalloc(sv, ["ZIIIII"] * 17)

"""ctypes binding of the engine's C ABI (include/lqcs_b200.h).

The shared library is built in-tree (``_lib/liblqcs_b200.so``, see build_native.py) and
loaded on first use.  There is no fallback: if the library is missing every engine call
raises, so a GPU run can never silently take another path.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "liblqcs_b200.so"

# status codes (enum lqcs_status)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_RANGE = 2
ERR_LOGIC = 3
ERR_CUDA = 4
ERR_OUT_OF_MEMORY = 5
ERR_TIMEOUT = 6
ERR_INTERNAL = 7


class EngineError(RuntimeError):
    """A device-side or internal failure reported by the engine."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class Instruction(C.Structure):
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


class KrausChannelC(C.Structure):
    _fields_ = [("n_ops", C.c_uint64), ("ops", C.POINTER(C.c_double))]


class SimOptions(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("has_seed", C.c_int32),
        ("fuse_gates", C.c_int32),
        ("num_threads", C.c_int32),
        ("max_fusion_width", C.c_int32),
        ("fusion_mode", C.c_int32),
        ("max_resident", C.c_int32),
        ("n_channels", C.c_uint64),
        ("channels", C.POINTER(KrausChannelC)),
        ("shot_offset", C.c_uint64),
    ]


class ParametricCircuitC(C.Structure):
    _fields_ = [
        ("n_qubits", C.c_uint32),
        ("n_insts", C.c_uint64),
        ("insts", C.POINTER(Instruction)),
        ("n_params", C.c_uint64),
        ("param_inst", C.POINTER(C.c_uint64)),
    ]


class HamiltonianC(C.Structure):
    _fields_ = [
        ("n_terms", C.c_uint64),
        ("coeffs", C.POINTER(C.c_double)),
        ("paulis", C.POINTER(C.c_char_p)),
    ]


class TuneEntry(C.Structure):
    _fields_ = [
        ("planner", C.c_int32),
        ("tile_bits", C.c_uint32),
        ("tile_low", C.c_uint32),
        ("inner", C.c_uint32),
        ("width", C.c_uint32),
        ("chosen", C.c_uint32),
        ("n_ops", C.c_uint64),
        ("device_ms", C.c_double),
    ]


class OpProfile(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("n_targets", C.c_uint32),
        ("n_gates", C.c_uint32),
        ("min_target", C.c_uint32),
        ("max_target", C.c_uint32),
        ("n_controls", C.c_uint32),
        ("device_ms", C.c_double),
        ("alg_bytes", C.c_double),
        ("alg_flops", C.c_double),
    ]


OP_KIND_NAMES = {0: "k_apply_1q", 1: "k_phase", 2: "k_dense", 3: "k_diag", 4: "k_perm",
                 5: "k_pauli", 6: "k_tile", 7: "k_regtile"}

StatePtr = C.c_void_p
ProgramPtr = C.c_void_p
_P = C.POINTER

# name -> (restype, argtypes); every name here is declared in include/lqcs_b200.h
SIGNATURES = {
    "lqcs_last_error": (C.c_char_p, []),
    "lqcs_version": (C.c_char_p, []),
    "lqcs_kernel_launch_count": (C.c_uint64, []),
    "lqcs_debug_emulate_register_passes": (C.c_int, [C.c_uint32, _P(Instruction), C.c_uint64,
                                                     C.c_uint64, C.c_int32, C.c_void_p,
                                                     C.c_uint64, _P(C.c_uint64), _P(C.c_uint64),
                                                     C.c_char_p, C.c_uint64]),
    "lqcs_state_create": (C.c_int, [C.c_uint32, C.c_void_p, _P(StatePtr)]),
    "lqcs_state_create_batch": (C.c_int, [C.c_uint32, C.c_uint32, C.c_void_p, _P(StatePtr)]),
    "lqcs_state_destroy": (C.c_int, [StatePtr]),
    "lqcs_state_num_qubits": (C.c_int, [StatePtr, _P(C.c_uint32)]),
    "lqcs_state_device_ptr": (C.c_int, [StatePtr, _P(C.c_void_p)]),
    "lqcs_state_set_zero": (C.c_int, [StatePtr]),
    "lqcs_state_load": (C.c_int, [StatePtr, C.c_void_p, C.c_uint64]),
    "lqcs_state_store": (C.c_int, [StatePtr, C.c_void_p, C.c_uint64]),
    "lqcs_state_apply": (C.c_int, [StatePtr, _P(Instruction), C.c_uint64, C.c_int32, C.c_int32,
                                   C.c_int32]),
    "lqcs_run_statevector": (C.c_int, [C.c_uint32, _P(Instruction), C.c_uint64, _P(SimOptions),
                                       C.c_void_p, _P(StatePtr)]),
    "lqcs_run": (C.c_int, [C.c_uint32, C.c_uint32, _P(Instruction), C.c_uint64, C.c_uint64,
                           _P(SimOptions), C.c_void_p]),
    "lqcs_state_read_range": (C.c_int, [StatePtr, C.c_uint64, C.c_uint64, C.c_void_p]),
    "lqcs_gate_matrix": (C.c_int, [_P(Instruction), C.c_int32, C.c_void_p, C.c_uint64,
                                   _P(C.c_uint64)]),
    "lqcs_state_probabilities": (C.c_int, [StatePtr, C.c_void_p]),
    "lqcs_state_norm": (C.c_int, [StatePtr, _P(C.c_double)]),
    "lqcs_state_sample": (C.c_int, [StatePtr, C.c_void_p, C.c_uint64, C.c_void_p,
                                    _P(C.c_double)]),
    "lqcs_state_expectation_pauli": (C.c_int, [StatePtr, C.c_char_p, _P(C.c_double)]),
    "lqcs_state_expectation_terms": (C.c_int, [StatePtr, _P(C.c_char_p), C.c_void_p, C.c_uint64,
                                               C.c_void_p, _P(C.c_double)]),
    "lqcs_expectation_terms_noalloc": (C.c_int, [C.c_void_p, C.c_uint32, _P(C.c_char_p),
                                                 C.c_uint64, C.c_void_p, C.c_void_p]),
    "lqcs_state_collapse": (C.c_int, [StatePtr, C.c_uint32, C.c_double, _P(C.c_int32)]),
    "lqcs_state_reset_qubit": (C.c_int, [StatePtr, C.c_uint32, C.c_double]),
    "lqcs_state_kraus_probability": (C.c_int, [StatePtr, C.c_uint32, C.c_void_p,
                                               _P(C.c_double)]),
    "lqcs_parameter_shift_gradient": (C.c_int, [_P(ParametricCircuitC), _P(HamiltonianC),
                                                C.c_void_p, C.c_void_p]),
    "lqcs_adjoint_gradient": (C.c_int, [_P(ParametricCircuitC), _P(HamiltonianC), C.c_void_p,
                                        C.c_uint64, C.c_uint32, C.c_void_p, C.c_void_p]),
    "lqcs_adjoint_gradient_multi": (C.c_int, [C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p]),
    "lqcs_release_caches": (C.c_int, []),
    "lqcs_batched_energy": (C.c_int, [_P(ParametricCircuitC), _P(HamiltonianC), C.c_void_p,
                                      C.c_uint64, C.c_uint32, C.c_void_p]),
    "lqcs_fusion_plan": (C.c_int, [C.c_uint32, _P(Instruction), C.c_uint64, C.c_int32, C.c_int32,
                                   C.c_uint64, C.c_void_p, C.c_void_p, _P(C.c_uint64)]),
    "lqcs_rng_uniforms": (C.c_int, [C.c_uint64, C.c_uint64, C.c_void_p]),
    "lqcs_rng_u64": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p]),
    "lqcs_autotune": (C.c_int, [C.c_uint32, _P(Instruction), C.c_uint64, C.c_uint64,
                                _P(TuneEntry), _P(C.c_uint64)]),
    "lqcs_dm_create": (C.c_int, [C.c_uint32, _P(Instruction), C.c_uint64, _P(SimOptions),
                                 _P(StatePtr)]),
    "lqcs_dm_probabilities": (C.c_int, [StatePtr, C.c_void_p]),
    "lqcs_dm_run": (C.c_int, [C.c_uint32, C.c_uint32, _P(Instruction), C.c_uint64, C.c_uint64,
                              _P(SimOptions), C.c_void_p]),
    "lqcs_costmodel_features": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_uint32, C.c_uint32, C.c_double, C.c_void_p]),
    "lqcs_costmodel_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_float,
                                       C.c_uint64, _P(C.c_float)]),
    "lqcs_costmodel_predict": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    "lqcs_costmodel_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, _P(C.c_float), C.c_void_p,
                                      C.c_uint64, _P(C.c_uint64)]),
    "lqcs_costmodel_get_weights": (C.c_int, [C.c_void_p, C.c_uint64, _P(C.c_uint64)]),
    "lqcs_costmodel_set_weights": (C.c_int, [C.c_void_p, C.c_uint64]),
    "lqcs_costmodel_clear": (C.c_int, []),
    "lqcs_costmodel_plan_ms": (C.c_int, [C.c_uint32, _P(Instruction), C.c_uint64, C.c_int32,
                                         C.c_int32, _P(C.c_double)]),
    "lqcs_program_create": (C.c_int, [C.c_uint32, _P(Instruction), C.c_uint64, C.c_int32, C.c_int32,
                                      C.c_int32, _P(ProgramPtr)]),
    "lqcs_program_destroy": (C.c_int, [ProgramPtr]),
    "lqcs_program_info": (C.c_int, [ProgramPtr, _P(C.c_uint64), _P(C.c_uint64)]),
    "lqcs_program_apply": (C.c_int, [StatePtr, ProgramPtr]),
    "lqcs_program_apply_profiled": (C.c_int, [StatePtr, ProgramPtr, C.c_uint64, _P(OpProfile),
                                              _P(C.c_uint64)]),
}

_lib = None
_lock = threading.Lock()


def library_path() -> Path:
    return Path(os.environ.get("LQCS_B200_LIB", str(_LIB_PATH)))


def lib():
    """The loaded engine library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            path = library_path()
            if not path.exists():
                raise RuntimeError(
                    f"engine library {path} is missing: build it with "
                    "`python -m litequantumcomputingsimulator_b200.build_native`")
            handle = C.CDLL(str(path))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def check(status: int) -> None:
    """Raise the Python exception matching a non-zero status code."""
    if status == OK:
        return
    msg = lib().lqcs_last_error().decode("utf-8", "replace")
    if status == ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == ERR_OUT_OF_RANGE:
        raise IndexError(msg)
    if status == ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    if status == ERR_LOGIC:
        raise RuntimeError(msg)
    raise EngineError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def launch_count() -> int:
    return int(lib().lqcs_kernel_launch_count())

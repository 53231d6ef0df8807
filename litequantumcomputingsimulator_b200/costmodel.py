"""The learned fusion cost model: data collection, training and persistence.

The model (a 3-layer, 64-wide FP32 MLP inside the engine library, trained by the engine's
own kernels) predicts log(device milliseconds per 2^24 amplitudes) of one device
operation from (op kind, width, lowest / highest qubit touched, source gate count,
register size, FP64 flops per amplitude).  Training data are the engine's own per-operation timings: circuits are
compiled under several candidate plans (greedy dense blocks of width 1..6, tile passes of
several shapes) and applied once with CUDA-event timing per operation
(``lqcs_program_apply_profiled``).  ``StatevectorSimulator(fusion_mode=2)`` then scores every
candidate plan of a circuit with the model and runs the cheapest; without trained weights
it falls back to the greedy plan.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from contextlib import contextmanager
from pathlib import Path

import numpy as np

from . import _native as N
from .simulator import CompiledCircuit, Statevector

FEATURES = 7
TILE_KIND = 6
GREEDY, LEARNED, TILE = 1, 2, 4
TILE_SHAPES = [(11, 5, 2), (12, 5, 2), (12, 5, 3), (13, 5, 2), (13, 5, 3)]


@contextmanager
def tile_shape(m: int, low: int, inner: int):
    keys = ("LQCS_TILE_BITS", "LQCS_TILE_LOW", "LQCS_TILE_INNER")
    saved = {k: os.environ.get(k) for k in keys}
    os.environ.update({"LQCS_TILE_BITS": str(m), "LQCS_TILE_LOW": str(low),
                       "LQCS_TILE_INNER": str(inner)})
    try:
        yield
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def features(kind: int, width: int, lo: int, hi: int, gates: int, n: int,
             flops_per_amp: float = 0.0) -> np.ndarray:
    out = np.zeros(FEATURES, dtype=np.float32)
    N.call("lqcs_costmodel_features", kind, width, lo, hi, gates, n, float(flops_per_amp),
           out.ctypes.data)
    return out


def target_of(ms: float, n: int) -> float:
    return math.log(max(ms, 1e-6)) - (n - 24) * math.log(2.0)


def profile_rows(prog: CompiledCircuit, sv: Statevector, n: int):
    """(features, targets) of every operation of one profiled application."""
    xs, ys = [], []
    for r in prog.profile(sv):
        kind = r["kind"]
        lo, hi = r["min_target"], r["max_target"]
        xs.append(features(kind, r["width"], lo, hi, r["gates"], n, r["alg_flops"] / float(1 << n)))
        ys.append(target_of(r["ms"], n))
    return xs, ys


def candidate_programs(circuit):
    """Every candidate plan the learned mode chooses among, as compiled programs."""
    n = circuit.num_qubits()
    progs = []
    for w in range(1, 7):
        if w <= n:
            progs.append((f"greedy{w}", CompiledCircuit(circuit, True, w, GREEDY)))
    if n >= 6:
        for m, low, inner in TILE_SHAPES:
            with tile_shape(min(m, n), low, inner):
                progs.append((f"tile{m}.{inner}", CompiledCircuit(circuit, True, 0, TILE)))
    return progs


def collect(circuits, warm: bool = True):
    """Profile every candidate plan of every circuit: returns (X [rows, FEATURES], y [rows])."""
    xs, ys = [], []
    for qc in circuits:
        n = qc.num_qubits()
        sv = Statevector(n)
        for _, prog in candidate_programs(qc):
            if warm:
                prog.apply(sv)
            x, y = profile_rows(prog, sv, n)
            xs += x
            ys += y
        del sv
    return np.asarray(xs, dtype=np.float32), np.asarray(ys, dtype=np.float32)


def train(x: np.ndarray, y: np.ndarray, epochs: int = 3000, lr: float = 3e-3, seed: int = 0) -> float:
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    loss = C.c_float(0.0)
    N.call("lqcs_costmodel_train", x.ctypes.data, y.ctypes.data, y.size, epochs, lr, seed,
           C.byref(loss))
    return loss.value


def predict(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(x.shape[0], dtype=np.float32)
    N.call("lqcs_costmodel_predict", x.ctypes.data, x.shape[0], out.ctypes.data)
    return out


def gradient(x: np.ndarray, y: np.ndarray):
    """(loss, flattened gradient) of the current weights on a batch."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    n = C.c_uint64(0)
    grad = np.zeros(8192, dtype=np.float32)
    loss = C.c_float(0.0)
    N.call("lqcs_costmodel_grad", x.ctypes.data, y.ctypes.data, y.size, C.byref(loss),
           grad.ctypes.data, grad.size, C.byref(n))
    return loss.value, grad[: n.value]


def get_weights() -> np.ndarray:
    n = C.c_uint64(0)
    N.call("lqcs_costmodel_get_weights", None, 0, C.byref(n))
    w = np.zeros(n.value, dtype=np.float32)
    N.call("lqcs_costmodel_get_weights", w.ctypes.data, w.size, C.byref(n))
    return w


def set_weights(w: np.ndarray) -> None:
    w = np.ascontiguousarray(w, dtype=np.float32)
    N.call("lqcs_costmodel_set_weights", w.ctypes.data, w.size)


def clear() -> None:
    N.call("lqcs_costmodel_clear")


def save(path) -> None:
    Path(path).write_text(json.dumps({"features": FEATURES, "weights": get_weights().tolist()}))


def load(path) -> None:
    d = json.loads(Path(path).read_text())
    set_weights(np.asarray(d["weights"], dtype=np.float32))


def plan_ms(circuit, mode: int = LEARNED, width: int = 0) -> float:
    """Model-predicted device time (ms) of the plan `mode` builds for the circuit."""
    arr, n, _k = circuit.c_instructions()
    out = C.c_double(0.0)
    N.call("lqcs_costmodel_plan_ms", circuit.num_qubits(), arr, n, width, mode, C.byref(out))
    return out.value

"""litequantumcomputingsimulator_b200 — B200 statevector engine for LiteQuantumComputingSimulator.

The Python surface mirrors ``pylqcs`` for the statevector path
(``python/pylqcs/__init__.py``): QuantumCircuit, ParametricCircuit, Gate, GateType,
StatevectorSimulator, Statevector, Result, KrausChannel, NoiseModel and
``algorithms.expectation`` / ``algorithms.parameter_shift_gradient``.  All state lives in
device memory and every amplitude operation runs in the engine's sm_100a CUDA kernels,
reached through the C ABI in ``include/lqcs_b200.h``.

Quick start::

    import litequantumcomputingsimulator_b200 as lq
    qc = lq.QuantumCircuit(2, 2)
    qc.h(0).cx(0, 1).measure_all()
    print(lq.StatevectorSimulator(seed=42).run(qc, shots=1024).counts())
"""
from . import algorithms, io
from .circuit import Gate, GateType, Instruction, ParametricCircuit, QuantumCircuit
from .noise import KrausChannel, NoiseModel
from .simulator import (DensityMatrix, DensityMatrixSimulator, Result, Statevector,
                        StatevectorSimulator)

__version__ = "0.1.0"

__all__ = [
    "DensityMatrix",
    "DensityMatrixSimulator",
    "Gate",
    "GateType",
    "Instruction",
    "KrausChannel",
    "NoiseModel",
    "ParametricCircuit",
    "QuantumCircuit",
    "Result",
    "Statevector",
    "StatevectorSimulator",
    "algorithms",
    "io",
]

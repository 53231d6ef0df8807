"""The seeded cases of the golden fixtures: each names its circuit generator and arguments,
so the fixtures' producer (make_golden.py, run on the reference library) and their users
(tests/test_golden.py, tests/test_gpu_golden.py) build the same inputs."""
import litequantumcomputingsimulator_b200 as lq
from litequantumcomputingsimulator_b200 import workloads as W

from helpers import random_circuit

# amplitudes: run_statevector (fuse on / off), or evolve from a seeded Gaussian state
AMPLITUDES = {
    "amp_random5_unfused": {"gen": "random_circuit", "args": [5, 80, 101],
                            "kwargs": {"max_controls": 3, "max_unitary": 3}, "fuse": False},
    "amp_random5_fused": {"gen": "random_circuit", "args": [5, 80, 101],
                          "kwargs": {"max_controls": 3, "max_unitary": 3}, "fuse": True},
    "amp_random9_unfused": {"gen": "random_circuit", "args": [9, 120, 102],
                            "kwargs": {"max_controls": 4, "max_unitary": 4}, "fuse": False},
    "amp_random9_fused": {"gen": "random_circuit", "args": [9, 120, 102],
                          "kwargs": {"max_controls": 4, "max_unitary": 4}, "fuse": True},
    "amp_random13_fused": {"gen": "random_circuit", "args": [13, 150, 103],
                           "kwargs": {"max_controls": 3, "max_unitary": 3}, "fuse": True},
    "amp_brickwork12": {"gen": "brickwork", "args": [12, 10, 2025], "kwargs": {}, "fuse": True},
    "amp_qft10_gaussian": {"gen": "qft", "args": [10], "kwargs": {}, "fuse": False,
                           "init": [10, 104]},
    "amp_qft13_gaussian": {"gen": "qft", "args": [13], "kwargs": {}, "fuse": False,
                           "init": [13, 105]},
}

# counts: StatevectorSimulator::run (end-of-circuit sampling, a noise model on the per-shot
# path) and the per-shot semantics on explicit Kraus placements
COUNTS = {
    "counts_brickwork8": {"gen": "brickwork", "args": [8, 6, 5], "kwargs": {"measure": True},
                          "shots": 4096, "seed": 42},
    "counts_brickwork14": {"gen": "brickwork", "args": [14, 8, 6], "kwargs": {"measure": True},
                           "shots": 2048, "seed": 7},
    "counts_noise_model5": {"gen": "brickwork", "args": [5, 4, 9], "kwargs": {"measure": True},
                            "shots": 300, "seed": 17,
                            "noise_model": [["depolarizing", 0.2], ["amplitude_damping", 0.15],
                                            ["phase_flip", 0.1]]},
    "counts_kraus6": {"gen": "brickwork", "args": [6, 4, 3],
                      "kwargs": {"measure": True, "noise": [0.05, 0.1, 0.2]},
                      "shots": 256, "seed": 21, "trajectories": True},
    "counts_kraus10": {"gen": "brickwork", "args": [10, 6, 8],
                       "kwargs": {"measure": True, "noise": [0.05, 0.1, 0.2]},
                       "shots": 128, "seed": 33, "trajectories": True},
}

# algorithms::expectation of a seeded Hamiltonian on a seeded Gaussian state
EXPECTATIONS = {
    "expect10": {"state": [10, 106], "hamiltonian": [10, 60, 107], "terms_each": 12},
    "expect14": {"state": [14, 108], "hamiltonian": [14, 40, 109], "terms_each": 8},
}

# algorithms::parameter_shift_gradient of a seeded Pauli-rotation ansatz
GRADIENTS = {
    "grad6": {"ansatz": [6, 20, 110], "max_w": 6, "hamiltonian": [6, 30, 111]},
    "grad9": {"ansatz": [9, 16, 112], "max_w": 8, "hamiltonian": [9, 25, 113]},
}

# DensityMatrixSimulator outcome probabilities of noisy circuits
DENSITY = {
    "dm_kraus6": {"gen": "brickwork", "args": [6, 5, 114], "kwargs": {"noise": [0.05, 0.1, 0.2]}},
    "dm_noise_model5": {"gen": "brickwork", "args": [5, 4, 115], "kwargs": {},
                        "noise_model": [["depolarizing", 0.03], ["amplitude_damping", 0.1]]},
}

# lqcs::Rng uniforms (mt19937_64, one draw per uniform)
UNIFORMS = {
    "uniforms_seed42": {"seed": 42, "count": 64},
    "uniforms_seed2025": {"seed": 2025, "count": 64},
}


# algorithms::modular_exponentiation after X(work 0) and H on the counting register
MODEXP = {
    "modexp_7_15": {"a": 7, "N": 15, "n_count": 6, "n_work": 4},
    "modexp_5_33": {"a": 5, "N": 33, "n_count": 5, "n_work": 6},
}

# algorithms::shor with a fixed seed (quantum rounds, lucky gcds, classical shortcuts)
SHOR = {
    "shor_15": {"N": 15, "shots": 64, "max_attempts": 10, "seed": 7},
    "shor_35": {"N": 35, "shots": 64, "max_attempts": 10, "seed": 7},
    "shor_55": {"N": 55, "shots": 64, "max_attempts": 10, "seed": 7},
    "shor_91": {"N": 91, "shots": 128, "max_attempts": 10, "seed": 3},
    # 24 qubits: the reference takes about 2.5 minutes on 8 cores (per-shot sampling)
    "shor_221": {"N": 221, "shots": 64, "max_attempts": 10, "seed": 4},
    "shor_21_gcd": {"N": 21, "shots": 64, "max_attempts": 10, "seed": 7},
    "shor_27_power": {"N": 27, "shots": 64, "max_attempts": 10, "seed": 1},
    "shor_97_prime": {"N": 97, "shots": 64, "max_attempts": 10, "seed": 1},
}


def circuit(spec: dict) -> lq.QuantumCircuit:
    gen, args, kwargs = spec["gen"], spec["args"], dict(spec.get("kwargs", {}))
    if gen == "random_circuit":
        return random_circuit(*args, **kwargs)
    if gen == "brickwork":
        if kwargs.get("noise") is not None:
            kwargs["noise"] = tuple(kwargs["noise"])
        return W.brickwork(*args, **kwargs)
    if gen == "qft":
        return lq.algorithms.qft(*args)
    raise ValueError(f"unknown generator {gen}")


def noise_model(spec):
    if not spec:
        return None
    noise = lq.NoiseModel()
    for name, p in spec:
        noise.add_all_qubit_channel(getattr(lq.KrausChannel, name)(p))
    return noise


def channel_ops(spec) -> list:
    """The noise model's channels as Kraus operator lists (the oracle's `channels`)."""
    model = noise_model(spec)
    return [c.ops for c in model.channels()] if model is not None else []


def load():
    """(arrays, cases) of the committed fixtures."""
    import json
    from pathlib import Path

    import numpy as np
    here = Path(__file__).resolve().parent
    with np.load(here / "reference_vectors.npz") as z:
        arrays = {k: z[k] for k in z.files}
    return arrays, json.loads((here / "reference_cases.json").read_text())

"""Writes the golden fixtures of this folder from the reference library itself.

The reference (a CMake C++ project) is compiled from its own sources into
oracle/_ref/liblqcs_ref.so by `make -C oracle ref`; that library only exists where the
reference sources do.  This script runs it on small seeded cases and stores its outputs, so
that the oracle (tests/test_golden.py) and the engine (tests/test_gpu_golden.py) are pinned
to the reference's own results on machines without it:

* reference_vectors.npz — amplitudes (`StatevectorSimulator::run_statevector`, fused and
  not; `evolve` from a Gaussian state for the QFT), exact noisy outcome probabilities
  (`DensityMatrixSimulator`), parameter-shift gradients (`algorithms::parameter_shift_gradient`),
  `Rng` uniforms;
* reference_cases.json — the case descriptions (generator and arguments), the counts maps of
  `StatevectorSimulator::run` (noiseless sampling, a noise model, explicit Kraus placements),
  the expectation values (`algorithms::expectation`) and seeded `algorithms::shor` results;
* the period-finding register after `algorithms::modular_exponentiation` (amplitudes).

Every circuit comes from the seeded generators of `litequantumcomputingsimulator_b200.workloads`
and `tests/helpers.py`; changing either means running this script again:

    make -C oracle ref && python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (ROOT, HERE.parent):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import litequantumcomputingsimulator_b200 as lq  # noqa: E402
from litequantumcomputingsimulator_b200 import workloads as W  # noqa: E402
from oracle.oracle import Ref  # noqa: E402

import cases  # noqa: E402


def main() -> None:
    ref = Ref()
    arrays: dict[str, np.ndarray] = {}
    meta: dict[str, dict] = {}
    for name, spec in cases.AMPLITUDES.items():
        qc = cases.circuit(spec)
        if spec.get("init") is not None:
            arrays[name] = ref.evolve_from(qc, W.gaussian_state(*spec["init"]))
        else:
            arrays[name] = ref.run_statevector(qc, fuse=spec["fuse"])
        meta[name] = spec
    for name, spec in cases.COUNTS.items():
        qc = cases.circuit(spec)
        if spec.get("trajectories"):
            regs = ref.trajectories(qc, spec["shots"], spec["seed"])
            vals, cnt = np.unique(regs, return_counts=True)
            counts = {int(v): int(c) for v, c in zip(vals, cnt)}
        else:
            noise = cases.noise_model(spec.get("noise_model"))
            counts = ref.run(qc, spec["shots"], spec["seed"], noise=noise)
        meta[name] = dict(spec, counts={str(k): v for k, v in sorted(counts.items())})
    for name, spec in cases.EXPECTATIONS.items():
        st = W.gaussian_state(*spec["state"])
        h = W.random_hamiltonian(*spec["hamiltonian"])
        terms = [ref.expectation_value(st, p) for _, p in h[: spec["terms_each"]]]
        meta[name] = dict(spec, energy=ref.expectation(st, h), term_values=terms)
    for name, spec in cases.GRADIENTS.items():
        pc, theta = W.random_pauli_ansatz(*spec["ansatz"], max_w=spec["max_w"])
        h = W.random_hamiltonian(*spec["hamiltonian"])
        arrays[name] = ref.parameter_shift_gradient(h, pc, theta)
        arrays[name + "_theta"] = np.asarray(theta, dtype=np.float64)
        meta[name] = spec
    for name, spec in cases.DENSITY.items():
        qc = cases.circuit(spec)
        arrays[name] = ref.dm_probabilities(qc, noise=cases.noise_model(spec.get("noise_model")))
        meta[name] = spec
    for name, spec in cases.UNIFORMS.items():
        arrays[name] = ref.uniforms(spec["seed"], spec["count"])
        meta[name] = spec
    for name, spec in cases.MODEXP.items():
        arrays[name] = ref.modexp_statevector(spec["a"], spec["N"], spec["n_count"],
                                              spec["n_work"])
        meta[name] = spec
    for name, spec in cases.SHOR.items():
        out = ref.shor(spec["N"], spec["shots"], spec["max_attempts"], spec["seed"])
        out["counts"] = {str(k): v for k, v in sorted(out["counts"].items())}
        meta[name] = dict(spec, result=out)
    np.savez_compressed(HERE / "reference_vectors.npz", **arrays)
    (HERE / "reference_cases.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(arrays)} arrays and {len(meta)} cases")


if __name__ == "__main__":
    main()

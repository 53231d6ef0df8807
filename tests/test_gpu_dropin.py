"""Drop-in check: the reference's own QuantumCircuit objects, built with its C++ API, run
through include/lqcs_b200_backend.hpp (an lqcs::Backend over the C ABI) and through the
reference's StatevectorSimulator; amplitudes within 1e-12, identical counts for the same
seed, identical exception types.  The program is oracle/_ref/dropin_check."""
import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

EXE = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "dropin_check"


def test_reference_circuits_through_cuda_backend():
    if not EXE.exists():
        pytest.skip("oracle/_ref/dropin_check not built (needs the reference sources)")
    res = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr + res.stdout
    out = json.loads(res.stdout.strip().splitlines()[-1])
    assert out["dropin_failures"] == 0
    assert out["max_amp_diff"] < 1e-12

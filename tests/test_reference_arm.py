"""bench.py's reference arm times the reference's own CPU kernels on the engine arm's
workload without loading any engine code: its records and angles come from the oracle
(oracle/workload.py) and must equal the engine's seeded brickwork exactly.  CPU only."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("n,depth,seed", [(12, 5, 2025), (30, 2, 2025), (9, 3, 7)])
def test_oracle_brickwork_equals_engine_workload(n, depth, seed):
    from oracle import workload as OW
    from litequantumcomputingsimulator_b200 import workloads as W
    a = OW.brickwork(n, depth, seed)
    b = W.brickwork(n, depth, seed)
    assert len(a) == b.num_instructions() == depth * OW.layer_size(n)
    for (gt, nc, qs, ps), ins in zip(a.records, b.instructions()):
        assert gt == int(ins.gate.type) and nc == ins.gate.n_controls
        assert tuple(qs) == tuple(ins.qubits) and tuple(ps) == tuple(ins.gate.params)
    assert a.alg_bytes() == W.alg_bytes(b)


def test_reference_arm_runs_without_engine_code(ref):
    code = (
        "import sys, json, runpy\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--qubits', '12', '--depth', '3',\n"
        "            '--steps', '4', '--warmup', '1']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'engine_so': 'liblqcs_b200' in maps,\n"
        "                  'engine_pkg': any(m.startswith('litequantumcomputingsimulator_b200')\n"
        "                                    for m in sys.modules)}))\n")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0, res.stderr
    lines = [json.loads(x) for x in res.stdout.strip().splitlines() if x.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert "one whole brickwork layer per timed step" in line["config"]["sample"]
    assert probe == {"engine_so": False, "engine_pkg": False}

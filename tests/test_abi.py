"""The C-ABI library: it loads without a GPU, exports every function include/lqcs_b200.h
declares, its record layouts match the header as a C compiler sees it, and host-only entry
points work.  No kernel is launched here."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from litequantumcomputingsimulator_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "lqcs_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lqcs_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = N.lib()
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.library_path())],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (lqcs_[a-z0-9_]+)", out))
    assert set(names) <= exported


def test_python_binding_covers_header():
    assert set(declared_functions()) == set(N.SIGNATURES)


def test_version():
    assert b"sm_100a" in N.lib().lqcs_version()


def _c_layout(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text("""
#include <stddef.h>
#include <stdio.h>
#include "lqcs_b200.h"
#define P(T, F) printf(#T "." #F " %zu\\n", offsetof(T, F))
int main(void) {
  printf("lqcs_instruction %zu\\n", sizeof(lqcs_instruction));
  P(lqcs_instruction, params); P(lqcs_instruction, clbit); P(lqcs_instruction, qubits);
  P(lqcs_instruction, pauli);
  printf("lqcs_sim_options %zu\\n", sizeof(lqcs_sim_options));
  P(lqcs_sim_options, n_channels); P(lqcs_sim_options, channels); P(lqcs_sim_options, shot_offset);
  printf("lqcs_kraus_channel %zu\\n", sizeof(lqcs_kraus_channel));
  printf("lqcs_parametric_circuit %zu\\n", sizeof(lqcs_parametric_circuit));
  P(lqcs_parametric_circuit, n_insts); P(lqcs_parametric_circuit, param_inst);
  printf("lqcs_hamiltonian %zu\\n", sizeof(lqcs_hamiltonian));
  printf("lqcs_op_profile %zu\\n", sizeof(lqcs_op_profile));
  P(lqcs_op_profile, device_ms); P(lqcs_op_profile, alg_bytes); P(lqcs_op_profile, alg_flops);
  printf("lqcs_tune_entry %zu\\n", sizeof(lqcs_tune_entry));
  P(lqcs_tune_entry, n_ops); P(lqcs_tune_entry, device_ms);
  return 0;
}
""")
    exe = tmp_path / "probe"
    subprocess.run(["/usr/bin/gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True)
    return dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())


def test_struct_layouts_match_header(tmp_path):
    c = {k: int(v) for k, v in _c_layout(tmp_path).items()}
    assert c["lqcs_instruction"] == C.sizeof(N.Instruction)
    assert c["lqcs_instruction.params"] == N.Instruction.params.offset
    assert c["lqcs_instruction.clbit"] == N.Instruction.clbit.offset
    assert c["lqcs_instruction.qubits"] == N.Instruction.qubits.offset
    assert c["lqcs_instruction.pauli"] == N.Instruction.pauli.offset
    assert c["lqcs_sim_options"] == C.sizeof(N.SimOptions)
    assert c["lqcs_sim_options.n_channels"] == N.SimOptions.n_channels.offset
    assert c["lqcs_sim_options.channels"] == N.SimOptions.channels.offset
    assert c["lqcs_sim_options.shot_offset"] == N.SimOptions.shot_offset.offset
    assert c["lqcs_kraus_channel"] == C.sizeof(N.KrausChannelC)
    assert c["lqcs_parametric_circuit"] == C.sizeof(N.ParametricCircuitC)
    assert c["lqcs_parametric_circuit.n_insts"] == N.ParametricCircuitC.n_insts.offset
    assert c["lqcs_parametric_circuit.param_inst"] == N.ParametricCircuitC.param_inst.offset
    assert c["lqcs_hamiltonian"] == C.sizeof(N.HamiltonianC)
    assert c["lqcs_op_profile"] == C.sizeof(N.OpProfile)
    assert c["lqcs_op_profile.device_ms"] == N.OpProfile.device_ms.offset
    assert c["lqcs_op_profile.alg_bytes"] == N.OpProfile.alg_bytes.offset
    assert c["lqcs_op_profile.alg_flops"] == N.OpProfile.alg_flops.offset
    assert c["lqcs_tune_entry"] == C.sizeof(N.TuneEntry)
    assert c["lqcs_tune_entry.n_ops"] == N.TuneEntry.n_ops.offset
    assert c["lqcs_tune_entry.device_ms"] == N.TuneEntry.device_ms.offset


def test_null_arguments_are_rejected_with_messages():
    lib = N.lib()
    rc = lib.lqcs_state_num_qubits(None, None)
    assert rc == N.ERR_INVALID_ARGUMENT
    assert b"null" in lib.lqcs_last_error()
    with pytest.raises(ValueError, match="null"):
        N.call("lqcs_state_norm", None, None)


def test_rng_matches_reference_draws():
    # lqcs::Rng(seed).uniform() is uniform_real_distribution<double>(0,1) over mt19937_64:
    # one 64-bit draw / 2^64; the first draws of seed 5489 are pinned by the 64-bit MT
    # reference output 14514284786278117030 (first value of mt19937_64 default seed).
    out = np.empty(3)
    N.call("lqcs_rng_uniforms", 5489, 3, out.ctypes.data)
    assert out[0] == 14514284786278117030 / 2.0 ** 64

#!/usr/bin/env python
"""Benchmark: 30-qubit complex128 gate application on one B200.

Workload (one "step"): the 30-qubit brickwork circuit of depth 40 (per layer a U3 on every
qubit with seeded angles, then CX on a seeded random perfect matching; 1800 gates) applied
with the engine's fusion pass to a device-resident 2^30-amplitude state (16 GiB, far larger
than the 126 MB L2, so no L2 flush is needed between steps).

Metric: gate-apply GB/s = algorithmic bytes of the source gates (32 * 2^n * f per gate,
f = fraction of amplitudes the gate can change) / device time.  Also reported: the
per-target single-gate sweep (one U3 on each target 0..29), QFT(30) on a random state,
batched adjoint gradients/s against the plain one-set-at-a-time GPU path, and the
reference's OpenMP CPU path timed on this host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "30q gate-apply GB/s vs HBM peak; batched adjoint grads/s vs plain GPU path"
UNIT = "GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--seed", type=int, default=2025)
    ap.add_argument("--workload", choices=["brickwork", "random_mix"], default="brickwork",
                    help="timed circuit: the headline brickwork, or the cost-model gate mix "
                         "(50 %% U3, 30 %% CX/CZ, 10 %% RZZ, 10 %% Pauli rotations of weight "
                         "2..8) for profiling; the CPU baseline covers the brickwork only")
    ap.add_argument("--fusion-width", type=int, default=0)
    ap.add_argument("--fusion-mode", type=int, default=0)
    ap.add_argument("--no-extras", action="store_true", help="skip sweep/QFT/adjoint/CPU legs")
    ap.add_argument("--extras", default=None,
                    help="comma-separated extra legs to run (sweep, unfused, qft, trajectories, "
                         "width6, autotune, ragged, dm, costmodel, config0, kernels, adjoint, shor); "
                         "default all")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-sharded", action="store_true",
                    help="skip the sharded batched-axis leg (parameter sets, trajectory shots)")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp64_peak(torch, device):
    """FP64 throughput of a library DGEMM on this GPU (TFLOP/s, best of 10): the FP64
    roofline denominator, measured in the run like the HBM copy peak."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(3):
        torch.matmul(a, b)
    best = None
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def ncu_traffic():
    """DRAM bytes per state amplitude of each kernel, from ncu captures (profiles/)."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return {}
    d = json.loads(p.read_text())
    return {k: v for k, v in d.items() if isinstance(v, dict) and "bytes_per_amplitude" in v}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ distributed plumbing
def relaunch_under_torchrun(gpus: int) -> int:
    """`bench.py --gpus N` (N > 1) started without a launcher: start N ranks on this node
    with torch.distributed.run (rendezvous on 127.0.0.1) and return their exit status."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py")] + sys.argv[1:]
    return subprocess.call(cmd)


def dist_setup(gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but WORLD_SIZE is {world}; launch with "
                         f"torchrun --nproc-per-node {gpus} or without a launcher")
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        return rank, world, local, dist
    return 0, 1, 0, None


def max_over_ranks(value: float, dist, device) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ------------------------------------------------------------------ reference arm
def reference_layer_sample(ref, n: int, depth: int, seed: int, steps: int, warmup: int):
    """Time the reference's OpenMP kernels (oracle/_ref) on whole brickwork layers: step s
    applies layer s mod depth (n U gates then n // 2 CX, 45 gates at 30 qubits) to one
    pre-touched 2^n-amplitude host state; each warm-up step applies one gate (the state's
    allocation and first touch happen before them).  Returns (seconds per timed step,
    algorithmic bytes per step, the time of the whole depth-`depth` circuit extrapolated
    from the mean layer time)."""
    from oracle import workload as OW
    qc = OW.brickwork(n, depth, seed)
    per = OW.layer_size(n)
    layers = [qc.slice(l * per, (l + 1) * per) for l in range(depth)]
    for w in range(warmup):
        ref.time_apply(qc.slice(w % len(qc), w % len(qc) + 1), 1)
    times, nbytes = [], []
    for s in range(steps):
        lay = layers[s % depth]
        times.append(ref.time_apply(lay, 1))
        nbytes.append(lay.alg_bytes())
    mean_layer = sum(times) / len(times)
    return times, nbytes, mean_layer * depth, qc


def reference_arm(args):
    """The reference's own OpenMP CPU implementation (oracle/_ref, compiled from the
    reference's sources) on this host's cores, on the engine arm's workload: the seeded
    30-qubit brickwork of depth 40, one whole layer (45 gates, 1/40 of the circuit) per
    timed step on a 16 GiB host state.  Builds its records and angles with the oracle alone
    (the reference's own lqcs::Rng through the same library), so no engine code is loaded."""
    from oracle.oracle import Ref
    if not Ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/liblqcs_ref.so was not built"}))
        return 0
    ref = Ref()
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    n = args.qubits
    try:
        times, nbytes, full_s, qc = reference_layer_sample(ref, n, args.depth, args.seed,
                                                           args.steps, args.warmup)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference could not run: {e}"}))
        return 0
    total = sum(times)
    value = sum(nbytes) / total / 1e9
    sample = (f"one whole brickwork layer per timed step ({n} U + {n // 2} CX of the {len(qc)}-gate "
              f"circuit, layers 0..{min(args.steps, args.depth) - 1}), reference OpenMP kernels on "
              f"a pre-touched host state; warm-up steps apply one gate each")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded brickwork)",
        "config": {"workload": f"brickwork n={n} depth={args.depth} seed={args.seed} ({len(qc)} gates)",
                   "sample": sample,
                   "extrapolated_full_circuit_s": full_s,
                   "extrapolation": f"mean layer time x {args.depth} layers",
                   "l2": "state > L2"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ CPU baseline leg
def cpu_side_baselines(ref) -> dict:
    """The reference's own CPU methods for the batched legs, on bounded samples (same run,
    all host cores): the parameter-shift gradient of one config-2 parameter set, and one
    config-3 trajectory over the first 2 of its 20 layers (scaled by 10, stated), and
    algorithms::shor(119) with seed 9 (21 qubits, one period-finding round)."""
    from litequantumcomputingsimulator_b200 import workloads as W
    out = {}
    try:
        t0 = time.perf_counter()
        r = ref.shor(119, 64, 10, 9)
        out["shor_21q_s"] = time.perf_counter() - t0
        out["shor_21q_factors"] = [r["factor1"], r["factor2"]]
    except Exception as ex:  # noqa: BLE001
        out["shor_error"] = str(ex)
    try:
        pc, _ = W.random_pauli_ansatz(16, 200, seed=11)
        ham = W.random_hamiltonian(16, 500, seed=12)
        sets = W.random_parameter_sets(pc.num_parameters(), 1, seed=13)
        t0 = time.perf_counter()
        ref.parameter_shift_gradient(ham, pc, sets[0])
        dt = time.perf_counter() - t0
        out["config2_parameter_shift_s_per_set"] = dt
        out["config2_parameter_shift_grads_per_s"] = 1.0 / dt
    except Exception as ex:  # noqa: BLE001
        out["config2_error"] = str(ex)
    try:
        dq = W.brickwork(10, 20, seed=88, noise=(1e-3, 1e-2, 1e-3))
        t0 = time.perf_counter()
        ref.dm_probabilities(dq)
        out["dm_10q_d20_reference_s"] = time.perf_counter() - t0
    except Exception as ex:  # noqa: BLE001
        out["dm_reference_error"] = str(ex)
    try:
        tq = W.brickwork(26, 2, seed=303, measure=True, noise=(1e-3, 1e-2, 1e-3))
        t0 = time.perf_counter()
        ref.trajectories(tq, 1, 404)
        dt = time.perf_counter() - t0
        out["config3_trajectory_s_2_layers"] = dt
        out["config3_trajectories_per_s_est"] = 1.0 / (dt * 10)
        out["config3_sample"] = ("one 26-qubit trajectory over 2 of 20 layers (reference-semantics "
                                 "driver on the reference kernels), x10 for the full depth")
    except Exception as ex:  # noqa: BLE001
        out["config3_error"] = str(ex)
    return out


def cpu_baseline(n: int, qc, depth: int, seed: int, budget_s: float = 12.0) -> dict:
    from oracle.oracle import Ref, Port
    import litequantumcomputingsimulator_b200 as lq
    from litequantumcomputingsimulator_b200 import workloads as W
    if Ref.available():
        ref = Ref()
        cores = os.cpu_count() or 1
        ref.set_threads(cores)
        times, nbytes, full_s, _qc = reference_layer_sample(ref, n, depth, seed, 1, 1)
        t = times[0]
        out = {"value": nbytes[0] / t / 1e9, "unit": UNIT, "cores": cores,
               "kind": "reference",
               "sample": f"brickwork layer 0 of the {n}-qubit circuit ({n} U + {n // 2} CX), "
                         f"reference OpenMP kernels on a pre-touched host state, {t:.2f} s; "
                         f"whole circuit extrapolated {full_s:.0f} s"}
        out.update(cpu_side_baselines(ref))
        return out
    insts = qc.instructions()
    # the scalar port on a 26-qubit sample, one core
    m = min(n, 26)
    port = Port()
    st = np.zeros(1 << m, dtype=np.complex128)
    st[0] = 1
    small = W.brickwork(m, 1, 7)
    t0 = time.perf_counter()
    k = 0
    for inst in small.instructions():
        port.apply_instruction(st, inst)
        k += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    sub = lq.QuantumCircuit(m)
    for inst in small.instructions()[:k]:
        sub.append(inst)
    return {"value": W.alg_bytes(sub) / dt / 1e9, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"first {k} gates of a {m}-qubit brickwork layer, scalar C restatement"}


# ------------------------------------------------------------------ engine arm
def main():
    args = parse()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        return reference_arm(args)

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_under_torchrun(args.gpus)
    rank, world, local, dist = dist_setup(args.gpus)
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import litequantumcomputingsimulator_b200 as lq
    from litequantumcomputingsimulator_b200 import _native as N
    from litequantumcomputingsimulator_b200 import workloads as W

    n, depth = args.qubits, args.depth
    if args.workload == "random_mix":
        qc = W.random_mix_circuit(n, depth, args.seed)
    else:
        qc = W.brickwork(n, depth, args.seed)
    gate_bytes = W.alg_bytes(qc)
    n_gates = qc.num_instructions()
    hbm_peak, peak_kind = peaks()

    prog = lq.simulator.CompiledCircuit(qc, True, args.fusion_width, args.fusion_mode)
    sv = lq.Statevector(n)   # |0...0>, device resident

    def step():
        prog.apply(sv)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(dist)
    launches0 = N.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(args.steps):
        step()
    stop.record()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    launches = N.launch_count() - launches0
    ms = start.elapsed_time(stop)
    ms = max_over_ranks(ms, dist, device)
    barrier(dist)
    ms_per_step = ms / args.steps
    value = gate_bytes * args.steps * world / (ms / 1e3) / 1e9

    # ---- roofline of the dominant kernel: one profiled application (CUDA events per op)
    prof = prog.profile(sv)
    by_kernel = {}
    for r in prof:
        k = by_kernel.setdefault(r["kernel"], {"ms": 0.0, "bytes": 0.0, "flops": 0.0, "launches": 0})
        k["ms"] += r["ms"]
        k["bytes"] += r["alg_bytes"]
        k["flops"] += r["alg_flops"]
        k["launches"] += 1
    dom_name, dom = max(by_kernel.items(), key=lambda kv: kv[1]["ms"])
    prof_total = sum(v["ms"] for v in by_kernel.values())
    fp64 = fp64_peak(torch, device)
    gbs = dom["bytes"] / (dom["ms"] / 1e3) / 1e9
    tfs = dom["flops"] / (dom["ms"] / 1e3) / 1e12
    hbm_frac, fp64_frac = gbs / hbm_peak, tfs / fp64
    base_kernel = dom_name.split("<")[0]
    traffic = None
    t = ncu_traffic().get(base_kernel)
    if t:
        traffic = t["bytes_per_amplitude"] * float(1 << n)   # per launch, scaled to 2^n
    # the bound is the resource the kernel's algorithmic work needs most of
    if fp64_frac > hbm_frac:
        roofline = {"bound": "fp64", "achieved": tfs, "peak": fp64, "unit": "TFLOP/s",
                    "frac": fp64_frac, "peak_kind": "measured in this run (DGEMM 4096^3, best of 10)"}
    else:
        roofline = {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                    "frac": hbm_frac, "peak_kind": peak_kind}
    roofline.update({
        "kernel": dom_name, "traffic": traffic, "launches": dom["launches"],
        "share": dom["ms"] / prof_total,
        "alg_bytes_per_launch": dom["bytes"] / dom["launches"],
        "alg_flops_per_launch": dom["flops"] / dom["launches"],
        "hbm": {"achieved_gbs": gbs, "peak_gbs": hbm_peak, "frac": hbm_frac, "peak_kind": peak_kind},
        "fp64": {"achieved_tflops": tfs, "peak_tflops": fp64, "frac": fp64_frac,
                 "peak_kind": "measured in this run (DGEMM 4096^3, best of 10)"},
        "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                        "share": round(v["ms"] / prof_total, 4),
                        "gbs": round(v["bytes"] / (v["ms"] / 1e3) / 1e9, 1),
                        "tflops": round(v["flops"] / (v["ms"] / 1e3) / 1e12, 2)}
                    for k, v in by_kernel.items()}})

    # extra legs (sweeps, other workloads) in the one-GPU run only: a multi-GPU run holds
    # every GPU while rank 0 works
    extras = {}
    if not args.no_extras and world == 1:
        extras = run_extras(lq, W, N, n, sv, hbm_peak, args)

    # ---- e2e through the public API on every rank: run_statevector + D2H of the final state
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(lq, qc, gate_bytes, args, dist, device, world)

    # ---- the batched axes sharded over the ranks (every N, weak scaling)
    sharded = None
    if not args.no_sharded:
        sharded = run_sharded(lq, W, dist, device, world)

    cpu = None
    if rank == 0 and not args.no_cpu and world == 1 and args.workload == "brickwork":
        try:
            cpu = cpu_baseline(n, qc, depth, args.seed)
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": f"synthetic (seeded {args.workload} circuit, |0> initial state)",
            "config": {"workload": f"{args.workload} n={n} depth={depth} seed={args.seed} "
                                   f"({n_gates} gates), fused ({prog.n_ops} device ops)",
                       "qubits": n, "depth": depth, "gates": n_gates,
                       "fusion_width": args.fusion_width or "default", "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (16 GiB state)"},
            "gpu_launches": launches,
            "gates_per_s": n_gates * args.steps * world / (ms / 1e3),
            "clocks": clock_info,
            "roofline": roofline,
            "e2e": e2e,
            "sharded": sharded,
            "cpu_baseline": cpu,
            "extras": extras,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_sharded(lq, W, dist, device, world) -> dict:
    """The two batched axes split over the ranks, each rank on its own GPU with no exchange
    while it computes and one NCCL all-gather at the end (sharding.py): 256 parameter sets
    per rank of the 16-qubit adjoint-gradient workload (200 rp gates, 500 terms), and 64
    trajectory shots per rank of the 26-qubit noisy brickwork (depth 20, config-3 rates),
    the ranks taking consecutive shot ranges of one seeded run.  Times are host-timed around
    the synchronous calls plus the gather, max over ranks; rates count all ranks' work."""
    import torch
    from litequantumcomputingsimulator_b200 import sharding as SH
    out = {"ranks": world}
    group = None
    if dist is None:   # one rank: the same workloads without the gather
        return out | _sharded_single(lq, W)
    pc, _ = W.random_pauli_ansatz(16, 200, seed=11)
    ham = W.random_hamiltonian(16, 500, seed=12)
    sets = W.random_parameter_sets(pc.num_parameters(), 256 * world, seed=13)
    SH.sharded_adjoint_gradient(ham, pc, sets[: 2 * world], group=group)   # plan + graph
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    e, g = SH.sharded_adjoint_gradient(ham, pc, sets, group=group)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, dist, device)
    out["adjoint_sets"] = int(sets.shape[0])
    out["adjoint_sets_per_s"] = sets.shape[0] / dt
    out["adjoint_gradient_checksum"] = float(np.sum(g))
    tq = W.brickwork(26, 20, seed=303, measure=True, noise=(1e-3, 1e-2, 1e-3))
    sim = lq.StatevectorSimulator(seed=404, max_resident=64)
    sim.run_registers(W.brickwork(12, 2, seed=1, measure=True, noise=(1e-3, 1e-2, 1e-3)), 8)
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    regs = SH.sharded_run_registers(sim, tq, 64 * world, group=group)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, dist, device)
    out["trajectory_shots"] = int(regs.size)
    out["trajectories_per_s"] = regs.size / dt
    out["trajectory_register_checksum"] = int(np.bitwise_xor.reduce(regs)) if regs.size else 0
    return out


def _sharded_single(lq, W) -> dict:
    """The sharded leg's two workloads on one rank (256 sets, 64 shots), for the per-N rate."""
    import torch
    pc, _ = W.random_pauli_ansatz(16, 200, seed=11)
    ham = W.random_hamiltonian(16, 500, seed=12)
    sets = W.random_parameter_sets(pc.num_parameters(), 256, seed=13)
    lq.algorithms.adjoint_gradient(ham, pc, sets[:2])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _e, g = lq.algorithms.adjoint_gradient(ham, pc, sets)
    out = {"adjoint_sets": 256, "adjoint_sets_per_s": 256 / (time.perf_counter() - t0),
           "adjoint_gradient_checksum": float(np.sum(g))}
    tq = W.brickwork(26, 20, seed=303, measure=True, noise=(1e-3, 1e-2, 1e-3))
    sim = lq.StatevectorSimulator(seed=404, max_resident=64)
    sim.run_registers(W.brickwork(12, 2, seed=1, measure=True, noise=(1e-3, 1e-2, 1e-3)), 8)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    regs = sim.run_registers(tq, 64)
    out.update({"trajectory_shots": 64, "trajectories_per_s": 64 / (time.perf_counter() - t0),
                "trajectory_register_checksum": int(np.bitwise_xor.reduce(regs))})
    return out


def run_e2e(lq, qc, gate_bytes, args, dist=None, device=None, world=1):
    import torch
    n = qc.num_qubits()
    try:
        host = torch.empty(1 << n, dtype=torch.complex128, pin_memory=True).numpy()
        pinned = True
    except Exception:  # noqa: BLE001
        host = np.empty(1 << n, dtype=np.complex128)
        pinned = False
    sim = lq.StatevectorSimulator(fuse_gates=True, max_fusion_width=args.fusion_width,
                                  fusion_mode=args.fusion_mode)
    arr, cnt, _k = qc.c_instructions()
    h2d = cnt * 80 + sum(len(i.gate.mat) * 16 for i in qc.instructions())
    reps = max(1, min(args.steps, 2))
    sv = sim.run_statevector(qc)
    sv.to_numpy(out=host)
    del sv
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(reps):
        sv = sim.run_statevector(qc)
        sv.to_numpy(out=host)
        del sv
    dt = max_over_ranks((time.perf_counter() - t0) / reps, dist, device)
    return {"value": world * gate_bytes / dt / 1e9, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(16 << n), "s_per_step": dt, "pinned": pinned,
            "path": "StatevectorSimulator.run_statevector + Statevector.to_numpy (D2H)"}


def device_maxdiff(a, b, chunk: int = 1 << 26) -> float:
    """max |a_i - b_i| of two device states, in chunks (no full-size temporaries)."""
    ta, tb = a.to_torch(), b.to_torch()
    worst = 0.0
    for lo in range(0, ta.numel(), chunk):
        worst = max(worst, (ta[lo:lo + chunk] - tb[lo:lo + chunk]).abs().max().item())
    return worst


def run_extras(lq, W, N, n, sv, hbm_peak, args):
    import torch
    out = {}
    legs = None if args.extras in (None, "all") else set(args.extras.split(","))

    def want(name):
        return legs is None or name in legs

    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # per-target sweep: one U3 on target t, timed over R launches
    if want("sweep"):
        sweep = {}
        reps = 5
        for t in range(n):
            c = lq.QuantumCircuit(n)
            c.u(0.3, 0.5, 0.7, t)
            p = lq.simulator.CompiledCircuit(c, fuse_gates=False)
            p.apply(sv)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            for _ in range(reps):
                p.apply(sv)
            e.record()
            torch.cuda.synchronize()
            ms = s.elapsed_time(e) / reps
            sweep[t] = 32.0 * (1 << n) / (ms / 1e3) / 1e9
        vals = list(sweep.values())
        out["per_target_u3_gbs"] = {str(k): round(v, 1) for k, v in sweep.items()}
        out["per_target_u3_min_frac"] = min(vals) / hbm_peak
        out["per_target_u3_median_frac"] = statistics.median(vals) / hbm_peak

    # unfused gate-by-gate path on the same brickwork (for the fusion speed-up)
    if want("unfused"):
        qc = W.brickwork(n, args.depth, args.seed)
        plain = lq.simulator.CompiledCircuit(qc, fuse_gates=False)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        plain.apply(sv)
        e.record()
        torch.cuda.synchronize()
        ms_plain = s.elapsed_time(e)
        out["brickwork_unfused_gbs"] = W.alg_bytes(qc) / (ms_plain / 1e3) / 1e9
        out["brickwork_unfused_ms"] = ms_plain

    # QFT(n) on a random state: the state is filled on the device side by a random circuit
    # would change the workload; instead the Gaussian state is uploaded once (not timed)
    if want("qft"):
        try:
            qft = lq.algorithms.qft(n)
            pq = lq.simulator.CompiledCircuit(qft, fuse_gates=True)
            pq.apply(sv)
            torch.cuda.synchronize()
            s.record()
            pq.apply(sv)
            e.record()
            torch.cuda.synchronize()
            ms_q = s.elapsed_time(e)
            out["qft_ms"] = ms_q
            out["qft_gates"] = qft.num_instructions()
            out["qft_gbs"] = W.alg_bytes(qft) / (ms_q / 1e3) / 1e9
            out["qft_device_ops"] = pq.n_ops
        except Exception as ex:  # noqa: BLE001
            out["qft_error"] = str(ex)

    # noisy trajectories: 26-qubit brickwork depth 20, depolarizing 1e-3 after each U3,
    # 1e-2 on both qubits after each CX, amplitude damping 1e-3 per qubit per layer; up to 64
    # resident per batch.  Fused driver: 128 trajectories (2 batches, a bounded sample of the
    # 1024-trajectory run); gate-by-gate driver: 16 trajectories, for the comparison.
    if want("trajectories"):
        try:
            tq = W.brickwork(26, 20, seed=303, measure=True, noise=(1e-3, 1e-2, 1e-3))
            warm = W.brickwork(12, 2, seed=1, measure=True, noise=(1e-3, 1e-2, 1e-3))
            sim = lq.StatevectorSimulator(seed=404, max_resident=64)
            sim.run_registers(warm, 8)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fused_regs = sim.run_registers(tq, 128)
            dt = time.perf_counter() - t0
            out["trajectories_26q_per_s"] = 128 / dt
            out["trajectories_26q_sample"] = ("128 trajectories, 64 resident per batch (1 GiB each), "
                                              "fused driver, host-timed")
            os.environ["LQCS_TRAJ_FUSED"] = "0"
            try:
                plain = lq.StatevectorSimulator(seed=404, max_resident=16)
                plain.run_registers(warm, 8)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                plain_regs = plain.run_registers(tq, 16)
                dtp = time.perf_counter() - t0
            finally:
                os.environ.pop("LQCS_TRAJ_FUSED", None)
            out["trajectories_26q_plain_per_s"] = 16 / dtp
            out["trajectories_26q_fused_speedup"] = (128 / dt) / (16 / dtp)
            out["trajectories_26q_same_registers"] = bool((fused_regs[:16] == plain_regs).all())
        except Exception as ex:  # noqa: BLE001
            out["trajectories_error"] = str(ex)

    # wide fused blocks: 28-qubit brickwork depth 20 fused greedily to 6-qubit blocks, on the
    # FP64 tensor path (mma.sync.m8n8k4.f64) and on the FFMA kernel
    if want("width6"):
        try:
            wq = W.brickwork(28, 20, seed=55)
            wsv = lq.Statevector(28)
            wprog = lq.simulator.CompiledCircuit(wq, True, 6, 1)
            res = {}
            for name, flag in (("dmma", "1"), ("ffma", "0")):
                os.environ["LQCS_DENSE_MMA"] = flag
                try:
                    wprog.apply(wsv)
                    torch.cuda.synchronize()
                    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    s.record()
                    wprog.apply(wsv)
                    e.record()
                    torch.cuda.synchronize()
                    res[name] = s.elapsed_time(e)
                finally:
                    os.environ.pop("LQCS_DENSE_MMA", None)
            prof = wprog.profile(wsv)
            k6 = [r for r in prof if r["kernel"] == "k_dense<6>"]
            out["width6_28q_ms"] = {k: round(v, 2) for k, v in res.items()}
            out["width6_28q_dmma_speedup"] = res["ffma"] / res["dmma"]
            if k6:
                out["width6_dmma_k6_tflops"] = (sum(r["alg_flops"] for r in k6) /
                                                (sum(r["ms"] for r in k6) / 1e3) / 1e12)
            del wsv
        except Exception as ex:  # noqa: BLE001
            out["width6_error"] = str(ex)

    # autotuner: every candidate plan of a 28-qubit brickwork (depth 40) timed on the device;
    # the chosen plan against the default one
    if want("autotune"):
        try:
            aq = W.brickwork(28, 40, seed=66)
            t0 = time.perf_counter()
            tune = lq.simulator.autotune(aq)
            out["autotune_28q_s"] = time.perf_counter() - t0
            out["autotune_28q"] = [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in r.items()}
                                   for r in tune]
            chosen = [r for r in tune if r["chosen"]]
            default = [r for r in tune if r["planner"] == "register tile passes" and
                       r["tile_bits"] == 12 and r["inner"] == 2]
            if chosen and default:
                out["autotune_28q_gain_vs_default"] = default[0]["ms"] / chosen[0]["ms"]
        except Exception as ex:  # noqa: BLE001
            out["autotune_error"] = str(ex)

    # uneven qubit counts: 8 problems of 10..17 qubits (100 rp gates, 100 terms, 32 parameter
    # sets each) as one captured graph with concurrent branches, against the same problems
    # one call after another
    if want("ragged"):
        try:
            probs = []
            for i, nq in enumerate(range(10, 18)):
                pc_i, _ = W.random_pauli_ansatz(nq, 100, seed=200 + i)
                probs.append((W.random_hamiltonian(nq, 100, seed=300 + i), pc_i))
            def sets_for(seed):
                return [W.random_parameter_sets(pc_i.num_parameters(), 32, seed=seed + j)
                        for j, (h_i, pc_i) in enumerate(probs)]
            lq.algorithms.adjoint_gradient_multi([(h, pc_i, s) for (h, pc_i), s in zip(probs, sets_for(1))])
            for (h, pc_i), s in zip(probs, sets_for(1)):
                lq.algorithms.adjoint_gradient(h, pc_i, s)
            torch.cuda.synchronize()
            s2 = sets_for(2)
            t0 = time.perf_counter()
            lq.algorithms.adjoint_gradient_multi([(h, pc_i, s) for (h, pc_i), s in zip(probs, s2)])
            t_m = time.perf_counter() - t0
            t0 = time.perf_counter()
            for (h, pc_i), s in zip(probs, s2):
                lq.algorithms.adjoint_gradient(h, pc_i, s)
            t_s = time.perf_counter() - t0
            out["ragged_8x32_sets_per_s"] = 8 * 32 / t_m
            out["ragged_sequential_sets_per_s"] = 8 * 32 / t_s
            out["ragged_speedup"] = t_s / t_m
        except Exception as ex:  # noqa: BLE001
            out["ragged_error"] = str(ex)

    # density-matrix backend: config-3 noise on a 13-qubit brickwork, depth 20 (rho as a
    # 26-qubit device state, 1 GiB), and the 10-qubit cross-check size
    if want("dm"):
        try:
            for nq in (10, 13):
                dq = W.brickwork(nq, 20, seed=88, noise=(1e-3, 1e-2, 1e-3))
                dsim = lq.DensityMatrixSimulator()
                dsim.run_density_matrix(W.brickwork(nq, 1, seed=1))
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                p = dsim.run_density_matrix(dq).probabilities()
                out[f"dm_{nq}q_d20_s"] = time.perf_counter() - t0
                out[f"dm_{nq}q_trace"] = float(p.sum())
        except Exception as ex:  # noqa: BLE001
            out["dm_error"] = str(ex)

    # learned fusion cost model: trained on the engine's own per-operation timings of
    # random-mix circuits shaped like the cost-model workload (50 % U3, 30 % CX/CZ, 10 % RZZ,
    # 10 % Pauli rotations of weight 2..8; depth 10..60) at 22..26 qubits (every candidate
    # plan of each, profiled op by op; 32-qubit circuits are too slow to collect in a bench
    # run, and the model predicts time per 2^24 amplitudes), then five held-out 32-qubit
    # circuits (64 GiB states) run under the greedy plan, the default plan and the model's own
    # pick (LQCS_LEARNED_JUDGE=1: no candidate timed), amplitudes compared between the plans
    if want("costmodel"):
        try:
            from litequantumcomputingsimulator_b200 import costmodel as CM
            # 25..27 qubits (0.5..2 GiB states): larger than L2, as the 32-qubit plans are
            corpus = [(25 + (i % 3), 10 + (7 * i) % 21, 1000 + i) for i in range(12)]
            train_set = [W.random_mix_circuit(nq, d, s_) for nq, d, s_ in corpus]
            t0 = time.perf_counter()
            x, y = CM.collect(train_set)
            t1 = time.perf_counter()
            loss = CM.train(x, y, epochs=3000, lr=3e-3, seed=0)
            t_train = time.perf_counter() - t1
            out["costmodel_corpus"] = {"circuits": len(corpus), "qubits": "25..27",
                                       "depths": "10, 17, 24", "rows": int(y.size),
                                       "collect_s": t1 - t0}
            out["costmodel_train_rows_x_epochs_per_s"] = y.size * 3000 / t_train
            xi = np.repeat(x, max(1, 1_000_000 // max(1, len(x))), axis=0)
            CM.predict(xi[:1024])
            t1 = time.perf_counter()
            CM.predict(xi)
            out["costmodel_infer_rows_per_s"] = len(xi) / (time.perf_counter() - t1)
            out["costmodel_train_mse"] = loss
            big = lq.Statevector(32)
            first = lq.Statevector(32)   # the greedy plan's result, for the amplitude check
            held_rows, worst = [], 0.0
            os.environ["LQCS_LEARNED_JUDGE"] = "1"
            try:
                for k, depth in enumerate((8, 12, 16, 20, 24)):
                    held = W.random_mix_circuit(32, depth, seed=777 + k)
                    row = {"depth": depth}
                    for name, mode in (("greedy", CM.GREEDY), ("learned", CM.LEARNED), ("default", 0)):
                        prog = lq.simulator.CompiledCircuit(held, True, 0, mode)
                        N.call("lqcs_state_set_zero", big.handle)
                        torch.cuda.synchronize()
                        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        s.record()
                        prog.apply(big)
                        e.record()
                        torch.cuda.synchronize()
                        row[name + "_ms"] = round(s.elapsed_time(e), 2)
                        row[name + "_ops"] = prog.n_ops
                        if name == "greedy":
                            first.to_torch().copy_(big.to_torch())
                        else:
                            d = device_maxdiff(big, first)
                            row[name + "_max_amp_diff"] = d
                            worst = max(worst, d)
                    held_rows.append(row)
            finally:
                os.environ.pop("LQCS_LEARNED_JUDGE", None)
            out["costmodel_32q_heldout"] = held_rows
            out["costmodel_32q_learned_vs_greedy"] = (sum(r["greedy_ms"] for r in held_rows) /
                                                      sum(r["learned_ms"] for r in held_rows))
            out["costmodel_32q_learned_vs_default"] = (sum(r["default_ms"] for r in held_rows) /
                                                       sum(r["learned_ms"] for r in held_rows))
            del big, first
            torch.cuda.empty_cache()
            if worst > 1e-12:
                raise AssertionError(f"32-qubit plans disagree: max |d psi| {worst}")
        except Exception as ex:  # noqa: BLE001
            out["costmodel_error"] = str(ex)

    # the 20-qubit workload (brickwork depth 20, measure_all, 4096 shots under a fixed seed)
    # through StatevectorSimulator.run, and the smallest distance of any shot's uniform from
    # a bin edge of the prefix sum (relative to the total): what keeps the counts identical
    # to those of the reference's sequential sum
    if want("config0"):
        try:
            q0 = W.brickwork(20, 20, seed=2024, measure=True)
            sim0 = lq.StatevectorSimulator(seed=42)
            for _ in range(2):
                sim0.run(q0, 4096)
            torch.cuda.synchronize()
            calls = []
            for _ in range(7):   # one call is a few ms: the median of 7 resists host jitter
                t0 = time.perf_counter()
                sim0.run(q0, 4096)
                calls.append(time.perf_counter() - t0)
            dt = statistics.median(calls)
            out["config0_run_ms_min"] = min(calls) * 1e3
            n_gates = sum(1 for ins in q0.instructions() if ins.gate.is_unitary())
            sv0 = lq.StatevectorSimulator(seed=42).run_statevector(W.brickwork(20, 20, seed=2024))
            _, margin0 = sv0.sample(W.UniformStream(42).take(4096))
            out["config0_run_ms"] = dt * 1e3
            out["config0_gates_per_s"] = n_gates / dt
            out["config0_min_margin"] = margin0
        except Exception as ex:  # noqa: BLE001
            out["config0_error"] = str(ex)

    # Shor's period finding (a caller of the controlled-permutation kernel): one controlled
    # modular multiplication y -> 2^(2^(n-11)) y mod 899 on the bench state (control qubit
    # n-11, work qubits n-10..n-1), CUDA-event timed over 3 launches, GB/s from 32 B per
    # amplitude of the control-1 half; then seeded algorithms.shor end to end at 21 qubits
    # (N = 119, the reference's CPU sample) and, on the 30-qubit bench, at 30 qubits
    # (N = 899 = 29 * 31: 20 counting + 10 work)
    if want("shor") and n >= 11:
        try:
            mx = lq.algorithms.modular_exponentiation(2, 899, n - 10, 10)
            one = lq.QuantumCircuit(n)
            one.append(mx.instructions()[n - 11])
            pk = lq.simulator.CompiledCircuit(one, fuse_gates=False)
            pk.apply(sv)
            torch.cuda.synchronize()
            s.record()
            for _ in range(3):
                pk.apply(sv)
            e.record()
            torch.cuda.synchronize()
            ms = s.elapsed_time(e) / 3
            out["shor_modmul_ms"] = ms
            out["shor_modmul_gbs"] = W.alg_bytes(one) / (ms / 1e3) / 1e9
            lq.algorithms.shor(119, 64, 10, 9)   # warm-up: planning, allocations
            for tag, N_, seed in (("21q", 119, 9), ("30q", 899, 1))[: 2 if n == 30 else 1]:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = lq.algorithms.shor(N_, 64, 10, seed)
                dt = time.perf_counter() - t0
                out[f"shor_{tag}"] = {"N": N_, "seed": seed, "s": dt, "success": r.success,
                                      "factors": [r.factor1, r.factor2], "a": r.a,
                                      "period": r.period, "attempts": r.attempts}
        except Exception as ex:  # noqa: BLE001
            out["shor_error"] = str(ex)

    # primitive kernels one gate (or reduction) at a time on the bench state, unfused: the
    # gate kernels (1q at the lowest and highest target, controlled, phase, 2q dense, 2q
    # diagonal, swap, Toffoli, Pauli rotations with and without X bits) timed with CUDA
    # events over 3 launches, GB/s from the algorithmic bytes (32 B per amplitude the gate can
    # change); the reductions (norm, Pauli expectation, 4096-shot sampling: prefix sum and
    # search, collapse) host-timed around the call, GB/s from one 16 B read per amplitude
    if want("kernels"):
        try:
            q = np.linalg.qr(np.random.default_rng(5).normal(size=(4, 4)) +
                             1j * np.random.default_rng(6).normal(size=(4, 4)))[0]
            cases = [
                ("u3_t0", lambda c: c.u(0.3, 0.5, 0.7, 0)),
                ("u3_t_top", lambda c: c.u(0.3, 0.5, 0.7, n - 1)),
                ("cx", lambda c: c.cx(3, n - 2)),
                ("cp", lambda c: c.cp(0.3, 2, n - 3)),
                ("unitary_2q", lambda c: c.unitary(q, [1, n - 4])),
                ("rzz", lambda c: c.rzz(0.4, 5, n - 5)),
                ("swap", lambda c: c.swap(4, n - 6)),
                ("ccx", lambda c: c.ccx(0, n - 1, 6)),
                ("rp_XYZ", lambda c: c.rp(0.4, "XYZ", [0, 7, n - 1])),
                ("rp_ZZ", lambda c: c.rp(0.4, "ZZ", [2, n - 2])),
            ]
            kern = {}
            for name, add in cases:
                c = lq.QuantumCircuit(n)
                add(c)
                pk = lq.simulator.CompiledCircuit(c, fuse_gates=False)
                pk.apply(sv)
                torch.cuda.synchronize()
                s.record()
                for _ in range(3):
                    pk.apply(sv)
                e.record()
                torch.cuda.synchronize()
                ms = s.elapsed_time(e) / 3
                kern[name] = {"ms": round(ms, 3), "gbs": round(W.alg_bytes(c) / (ms / 1e3) / 1e9, 1)}
            read_bytes = 16.0 * (1 << n)
            pauli = "XZ" + "I" * (n - 4) + "YZ"
            uni = np.random.default_rng(7).random(4096)
            reductions = [("norm", lambda: sv.norm()),
                          ("expectation_XZ..YZ", lambda: sv.expectation_value(pauli)),
                          ("sample_4096", lambda: sv.sample(uni)),
                          ("collapse", lambda: sv.collapse(n - 1, 0.25))]
            for name, fn in reductions:
                fn()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for _ in range(3):
                    fn()
                ms = (time.perf_counter() - t0) / 3 * 1e3
                kern[name] = {"ms": round(ms, 3), "gbs": round(read_bytes / (ms / 1e3) / 1e9, 1)}
            out["kernels"] = kern
            out["kernels_hbm_peak_gbs"] = hbm_peak
        except Exception as ex:  # noqa: BLE001
            out["kernels_error"] = str(ex)

    # batched adjoint gradients (16 qubits, 200 rp gates, 500 terms, 256 sets per call, all
    # resident — the default resident count): the first
    # call builds the plan and captures its CUDA graph, the timed call replays it with new
    # parameters; against direct launches, the plain one-set-at-a-time adjoint and the
    # reference's parameter-shift method run on the GPU
    if want("adjoint"):
        try:
            pc, _ = W.random_pauli_ansatz(16, 200, seed=11)
            ham = W.random_hamiltonian(16, 500, seed=12)
            sets = W.random_parameter_sets(pc.num_parameters(), 256, seed=13)
            sets2 = W.random_parameter_sets(pc.num_parameters(), 256, seed=14)
            lq.algorithms.adjoint_gradient(ham, pc, sets)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            lq.algorithms.adjoint_gradient(ham, pc, sets2)
            t_b = time.perf_counter() - t0
            os.environ["LQCS_GRAPHS"] = "0"
            try:
                lq.algorithms.adjoint_gradient(ham, pc, sets[:1], max_resident=1)
                t0 = time.perf_counter()
                lq.algorithms.adjoint_gradient(ham, pc, sets2)
                t_d = time.perf_counter() - t0
                t0 = time.perf_counter()
                for b in range(16):
                    lq.algorithms.adjoint_gradient(ham, pc, sets[b], max_resident=1)
                t_p = (time.perf_counter() - t0) / 16
            finally:
                os.environ.pop("LQCS_GRAPHS", None)
            t0 = time.perf_counter()
            lq.algorithms.parameter_shift_gradient(ham, pc, sets[0])
            t_s = time.perf_counter() - t0
            out["adjoint_batched_grads_per_s"] = 256 / t_b
            out["adjoint_batched_direct_grads_per_s"] = 256 / t_d
            out["adjoint_graph_speedup"] = t_d / t_b
            out["adjoint_plain_grads_per_s"] = 1 / t_p
            out["adjoint_speedup_vs_plain"] = (256 / t_b) * t_p
            out["parameter_shift_gpu_grads_per_s"] = 1 / t_s
            out["adjoint_speedup_vs_parameter_shift"] = (256 / t_b) * t_s
        except Exception as ex:  # noqa: BLE001
            out["adjoint_error"] = str(ex)
    return out


if __name__ == "__main__":
    sys.exit(main())

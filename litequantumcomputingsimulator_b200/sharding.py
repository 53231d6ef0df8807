"""Sharding of the batched axes over ranks (one process per GPU, torch.distributed).

A single statevector does not shard in this engine: its workloads run as replicas.  The
batched axes do — parameter sets of a gradient batch, shots of a trajectory run — and need
no exchange while they compute: each rank takes a contiguous slice, computes it on its own
GPU, and one all-gather at the end assembles the result in batch order.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def shard_bounds(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous slice [lo, hi) of `total` items for `rank`; sizes differ by at most one."""
    base, extra = divmod(total, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def sharded_map(fn: Callable[[np.ndarray], np.ndarray], items: np.ndarray, group=None,
                device=None) -> np.ndarray:
    """Apply fn to this rank's slice of items (first axis) and all-gather the results in
    order.  fn must return an array whose first axis matches its input's."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard_bounds(items.shape[0], world, rank)
    local = np.asarray(fn(items[lo:hi]), dtype=np.float64)
    width = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    counts = [shard_bounds(items.shape[0], world, r) for r in range(world)]
    longest = max(h - l for l, h in counts)
    dev = device if device is not None else torch.device("cpu")
    buf = torch.zeros((longest, width), dtype=torch.float64, device=dev)
    if hi > lo:
        buf[: hi - lo] = torch.as_tensor(local.reshape(hi - lo, width), device=dev)
    gathered = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(gathered, buf, group=group)
    parts = [gathered[r][: h - l].cpu().numpy() for r, (l, h) in enumerate(counts)]
    out = np.concatenate(parts, axis=0)
    return out.reshape((items.shape[0],) + local.shape[1:])


def sharded_adjoint_gradient(hamiltonian, ansatz, params: np.ndarray, group=None,
                             max_resident: int = 0):
    """Batched adjoint gradients with the parameter sets split over ranks.  Returns
    (energies (B,), gradients (B, P)) on every rank."""
    import torch
    from .algorithms import adjoint_gradient
    from .algorithms import _parameter_sets
    p, _ = _parameter_sets(params, ansatz.num_parameters())

    def fn(chunk):
        if chunk.shape[0] == 0:
            return np.zeros((0, 1 + ansatz.num_parameters()))
        e, g = adjoint_gradient(hamiltonian, ansatz, chunk, max_resident=max_resident)
        return np.concatenate([np.asarray(e).reshape(-1, 1), np.asarray(g)], axis=1)

    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None
    both = sharded_map(fn, p, group=group, device=dev)
    return both[:, 0], both[:, 1:]


def gather_registers(local: np.ndarray, total: int, group=None, device=None) -> np.ndarray:
    """All-gather each rank's slice of per-shot registers (uint64) into shot order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    counts = [shard_bounds(total, world, r) for r in range(world)]
    longest = max(h - l for l, h in counts)
    dev = device if device is not None else torch.device("cpu")
    buf = torch.zeros(longest, dtype=torch.int64, device=dev)
    if local.size:
        buf[: local.size] = torch.as_tensor(local.astype(np.uint64).view(np.int64), device=dev)
    gathered = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(gathered, buf, group=group)
    parts = [gathered[r][: h - l].cpu().numpy() for r, (l, h) in enumerate(counts)]
    return np.concatenate(parts).view(np.uint64)


def sharded_run_registers(sim, circuit, shots: int, group=None) -> np.ndarray:
    """Per-shot registers of `shots` shots with the shots split over ranks: rank r runs its
    contiguous range with the seeded stream advanced past the earlier ranks' shots
    (run_registers(shot_offset=lo)), so the gathered registers equal one process's run.
    Trajectories (noise, mid-circuit measurement) need no exchange while they run; a
    sampling run recomputes the state on every rank."""
    import torch
    import torch.distributed as dist
    lo, hi = shard_bounds(shots, dist.get_world_size(group), dist.get_rank(group))
    local = sim.run_registers(circuit, hi - lo, shot_offset=lo) if hi > lo else np.zeros(0, np.uint64)
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None
    return gather_registers(np.asarray(local, dtype=np.uint64), shots, group=group, device=dev)

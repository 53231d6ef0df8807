"""Multi-rank logic on CPU: two gloo ranks shard a batch of parameter sets, compute their
slices (here with the oracle's CPU energies, standing in for a GPU per rank) and all-gather;
the result must equal the single-process computation in batch order."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from litequantumcomputingsimulator_b200.sharding import shard_bounds


def test_shard_bounds_cover_everything():
    for total in (0, 1, 5, 256, 257):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(total, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _energies(chunk):
    import litequantumcomputingsimulator_b200 as lq
    from oracle.oracle import Port
    port = Port()
    pc = lq.ParametricCircuit(3)
    pc.h(0)
    pc.ry(0)
    pc.cx(0, 1)
    pc.rp("XZ", [1, 2])
    ham = [(0.5, "ZZI"), (-1.2, "IXY"), (0.3, "ZIZ")]
    return np.array([[port.expectation(port.run_statevector(pc.bind(list(p))), ham)] for p in chunk])


def _worker(rank, world, port, items, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from datetime import timedelta
    from litequantumcomputingsimulator_b200.sharding import sharded_map
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res = sharded_map(_energies, items)
        if rank == 0:
            np.save(out_path, res)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_sets", [7, 8])
def test_two_gloo_ranks_gather_in_order(tmp_path, n_sets):
    rng = np.random.default_rng(n_sets)
    items = rng.uniform(-np.pi, np.pi, (n_sets, 2))
    out = str(tmp_path / "res.npy")
    mp.spawn(_worker, args=(2, _free_port(), items, out), nprocs=2, join=True)
    got = np.load(out)
    want = _energies(items)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) < 1e-14


class _ShotRangeSim:
    """Stands in for a simulator on CPU: shot s of the seeded run has register
    s * 2654435761 mod 2^64 (any function of the global shot index), so a rank that ignores
    its shot_offset or a gather out of order is caught."""

    def run_registers(self, circuit, shots, shot_offset=0):
        s = np.arange(shot_offset, shot_offset + shots, dtype=np.uint64)
        return s * np.uint64(2654435761) + np.uint64(1 << 63)


def _shots_worker(rank, world, port, shots, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from datetime import timedelta
    from litequantumcomputingsimulator_b200.sharding import sharded_run_registers
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        regs = sharded_run_registers(_ShotRangeSim(), None, shots)
        if rank == 0:
            np.save(out_path, regs)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("shots", [1, 9, 64])
def test_two_gloo_ranks_shard_trajectory_shots(tmp_path, shots):
    out = str(tmp_path / "regs.npy")
    mp.spawn(_shots_worker, args=(2, _free_port(), shots, out), nprocs=2, join=True)
    got = np.load(out)
    assert got.dtype == np.uint64
    assert np.array_equal(got, _ShotRangeSim().run_registers(None, shots))

"""Multi-GPU sharding logic on the CPU: balanced contiguous ranges, and a
world-size-2 gloo run whose gathered result equals the single-process result
(a deterministic per-cell map stands in for the GPU integration, so the test
needs no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from hpc_ode_b200 import shard, workloads as W


def test_ranges_cover_and_balance():
    rng = np.random.default_rng(0)
    for n in (0, 1, 5, 100, 1001):
        for world in (1, 2, 3, 8):
            cost = rng.uniform(0.1, 10.0, n)
            r = shard.balanced_ranges(cost, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == n
            for (a, b), (c, d) in zip(r, r[1:]):
                assert b == c and a <= b
            if n >= 100:
                sums = [cost[a:b].sum() for a, b in r]
                assert max(sums) - min(sums) <= 2 * cost.max() + 1e-9


def test_cost_proxy_prefers_ignition_window():
    c = shard.temperature_cost(np.array([300.0, 800.0, 1400.0, 2400.0]))
    assert c[2] > c[3] > 0 and c[2] > c[0] and c[0] == c[1] == 1.0


def test_invalid_costs():
    with pytest.raises(ValueError):
        shard.balanced_ranges([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        shard.balanced_ranges([1.0], 0)


def _fake_integrate(T, Y, P, dt):
    """Deterministic per-cell stand-in for the GPU integration."""
    T += 1000.0 * dt * np.sin(T)
    Y *= 1.0 + dt
    return (T > 1500.0).astype(np.int32)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = W.make("gri_bimodal", 300, seed=9)
    sl, Tp, Yp, st = shard.integrate_shard(rank, world, b.T, b.Y, b.P, b.dt, _fake_integrate)
    res = shard.gather_to(0, sl, Tp, Yp, st, b.ncells)
    if rank == 0:
        np.savez(out, T=res[0], Y=res[1], st=res[2])
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gloo_world2_equals_single_process(tmp_path):
    out = str(tmp_path / "res.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    r = np.load(out)
    b = W.make("gri_bimodal", 300, seed=9)
    T, Y = b.T.copy(), b.Y.copy()
    st = _fake_integrate(T, Y, b.P, b.dt)
    assert np.array_equal(r["T"], T) and np.array_equal(r["Y"], Y) and np.array_equal(r["st"], st)


def _strong_worker(rank, world, port, out):
    """bench.py --scaling strong's split, on gloo ranks: every rank builds the
    same seeded workload, takes its cost-balanced range (shard.rank_range) as a
    subset batch, integrates it (fake per-cell map) and the parts are gathered."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    full = W.make("gri_1m", 4096, seed=5)
    a, b = shard.rank_range(full.T, world, rank)
    part = full.subset(np.arange(a, b))
    T, Y = part.T.copy(), np.ascontiguousarray(part.Y.copy())
    st = _fake_integrate(T, Y, part.P, part.dt)
    res = shard.gather_to(0, slice(a, b), T, Y, st, full.ncells)
    ranges = [None] * world if rank == 0 else None
    dist.gather_object((a, b), ranges, dst=0)
    if rank == 0:
        np.savez(out, T=res[0], Y=res[1], st=res[2], ranges=np.array(ranges))
    dist.barrier()
    dist.destroy_process_group()


def test_strong_scaling_split_gloo_world2(tmp_path):
    out = str(tmp_path / "strong.npz")
    mp.start_processes(_strong_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    r = np.load(out)
    full = W.make("gri_1m", 4096, seed=5)
    want = shard.balanced_ranges(shard.temperature_cost(full.T), 2)
    assert [tuple(x) for x in r["ranges"]] == want
    assert want[0][1] == want[1][0] and 0 < want[0][1] < full.ncells
    cost = shard.temperature_cost(full.T)
    s0, s1 = cost[:want[0][1]].sum(), cost[want[0][1]:].sum()
    assert abs(s0 - s1) <= 2 * cost.max()
    T, Y = full.T.copy(), full.Y.copy()
    st = _fake_integrate(T, Y, full.P, full.dt)
    assert np.array_equal(r["T"], T) and np.array_equal(r["Y"], Y) and np.array_equal(r["st"], st)

"""Sweep host logic and its multi-rank path on CPU (gloo, world size 2): the parameter law,
the deterministic sharding, and the result gather.  The per-disk runner is the CPU oracle
on small grids here (the product runner is diskgpu.sweep.run_point on the GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from diskgpu import sweep as S


def test_draw_is_counter_based_and_in_range():
    a = S.draw(64, seed=7)
    b = S.draw(80, seed=7)
    assert [p.as_dict() for p in a] == [p.as_dict() for p in b[:64]]  # prefix-stable
    for p in b:
        assert p.N in S.GRIDS
        assert 1.0 <= p.Qmin < 2.0 and 0.2 <= p.mass_ratio < 1.0
        assert 0.05 <= p.soft_over_r < 0.2 and 1.5 <= p.gamma < 2.0 and 0.0 <= p.phase0 < np.pi
    assert len({p.N for p in b}) == 4
    assert S.draw(8, seed=8)[0].Qmin != a[0].Qmin


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_partitions_and_balances(world):
    pts = S.draw(256)
    parts = [S.shard(pts, world, r) for r in range(world)]
    idx = sorted(p.index for part in parts for p in part)
    assert idx == list(range(256))
    loads = [sum(S.cost(p) for p in part) for part in parts]
    assert max(loads) <= min(loads) + S.cost(max(pts, key=S.cost)) + 1e-9


def _cpu_runner(pt):
    import oracle as O

    n = {128: 8, 256: 12, 384: 16, 512: 16}[pt.N]
    d = O.Disk(Nu=n, Nphi=n, eps=pt.soft_over_r ** 2, amp=0.05, gamma_gas=pt.gamma, phase0=pt.phase0)
    for _ in range(5):
        d.step()
    c2, ph = d.cm(2)
    return {"index": pt.index, "c2": c2, "ph2": ph}


def _worker(rank, world, port, out):
    import sys

    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    for sub in ("../heavy-disks_b200", "../oracle"):
        sys.path.insert(0, os.path.join(here, sub))
    from diskgpu import sweep as S2

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pts = S2.draw(12, seed=3)
    mine = S2.shard(pts, world, rank)
    res = S2.gather([_cpu_runner(p) for p in mine])
    if rank == 0:
        out.put(res)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_rank_sweep_matches_serial():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    serial = [_cpu_runner(p) for p in S.draw(12, seed=3)]
    assert [r["index"] for r in res] == list(range(12))
    for a, b in zip(res, serial):
        assert a == b

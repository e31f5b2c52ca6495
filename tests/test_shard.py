"""Sharding of ensemble members across ranks (CPU; gloo, world size 2)."""
import os
import socket

import pytest

from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P
from meumapps_ss_b200.shard import gather_by_member, shard_members


def test_shard_covers_and_balances():
    ws = CF.ensemble_config(96, precision=P.PREC_F32)
    cells = [w.params.nx ** 3 for w in ws]
    for world in (1, 2, 4, 8):
        sh = shard_members(cells, world)
        flat = sorted(m for s in sh for m in s)
        assert flat == list(range(96))
        loads = [sum(cells[m] for m in s) for s in sh]
        # greedy largest-first: no rank exceeds the mean by more than the largest member
        assert max(loads) - sum(loads) / world <= max(cells)
        assert sh == shard_members(cells, world)  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, cells, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_members(cells, world)[rank]
        local = {m: (rank, cells[m] * 2) for m in mine}
        got = gather_by_member(local, len(cells))
        q.put((rank, mine, got))
    finally:
        dist.destroy_process_group()


def test_gather_by_member_gloo_two_ranks():
    mp = pytest.importorskip("torch.multiprocessing")
    cells = [n ** 3 for n in (32, 128, 48, 96, 64, 32, 128, 48)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, cells, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, mine, got = q.get(timeout=120)
        res[r] = (mine, got)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][0] + res[1][0]) == list(range(len(cells)))
    assert res[1][1] is None
    got = res[0][1]
    assert [g[1] for g in got] == [c * 2 for c in cells]
    assert all(g[0] == (0 if m in res[0][0] else 1) for m, g in enumerate(got))

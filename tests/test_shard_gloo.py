"""Sharding a scene's work units over ranks (lipika_b200/shard.py), on CPU:
the plan, and a world_size-2 gloo run in which each rank renders its share
with the oracle and rank 0 gathers the manifests, which must equal a
single-process render unit for unit."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from lipika_b200 import shard as S
from oracle import oracle as O
from tests import scenes


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assign_keeps_receivers_whole_and_balances():
    units = [S.Unit(w, rx, b, n, k) for w, (rx, b, n, k) in enumerate(
        [(0, 0, 1000, 24), (0, 1, 50, 24), (1, 0, 4000, 24), (2, 0, 800, 24), (2, 1, 800, 24), (3, 0, 300, 2)])]
    plan = S.assign(units, 2)
    assert sorted(w for p in plan for w in p) == list(range(len(units)))
    for rx in {u.rx for u in units}:
        ranks = {k for k, p in enumerate(plan) for w in p if units[w].rx == rx}
        assert len(ranks) == 1, rx
    loads = [sum(units[w].cost for w in p) for p in plan]
    assert max(loads) <= 1.5 * min(loads)
    assert S.assign(units, 2) == plan  # deterministic on every rank
    assert S.assign(units, 1) == [list(range(len(units)))]
    with pytest.raises(ValueError):
        S.assign(units, 0)


@pytest.mark.parametrize("n,world,align", [(1000, 2, 64), (4096, 3, 1024), (10, 4, 8), (0, 2, 16)])
def test_time_shards_cover_the_band_once(n, world, align):
    sh = S.time_shards(n, world, align)
    assert len(sh) == world
    pos = 0
    for i0, m in sh:
        assert i0 == pos and m >= 0
        assert i0 % align == 0 or i0 == n
        pos += m
    assert pos == n


def _scene():
    return scenes.config_c2(duration_s=0.01, n_rx=3, noise=True)


def _render(osc, w, r, b):
    return osc.generate_band(r, b, 2026, w, 1 << 12, 1, O.NOISE_COUNTER)["iq"]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        osc = O.Scene(_scene())
        mine = S.render_rank(osc, rank, world, lambda w, r, b: _render(osc, w, r, b))
        man = S.gather_manifests(mine)
        if rank == 0:
            q.put(man)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_render_every_unit_once():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    man = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    osc = O.Scene(_scene())
    ref = {w: (len(iq), S.checksum(iq)) for w, (r, b) in enumerate(osc.work()) for iq in [_render(osc, w, r, b)]}
    assert man == ref

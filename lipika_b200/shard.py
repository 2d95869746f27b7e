"""Work-unit sharding of a scene across ranks (one process per GPU).

The reference renders (receiver, band) work units independently
(src/pipeline.rs:506-535, one rayon task each). Here the units of a scene
are split over the ranks of a torch.distributed group:

* every band of a receiver goes to the same rank (they share the
  receiver's clock walk, which the batched fan-out scans once per
  receiver), and receivers are assigned longest-processing-time first by
  their tx·rx sample count, so ranks get near-equal work;
* no data-path collective is needed: every per-sample random quantity
  (clock walk, AWGN) is counter-based on (seed, global index), so any rank
  regenerates any unit bit for bit. The only communication is the final
  gather of what each rank rendered (a manifest per unit), for the writer
  on rank 0.

A single long band (one receiver, one band) can be cut in time instead
(`time_shards`): each rank renders a contiguous, tile-aligned range of the
band; the walk carries a range needs are recomputed on that rank from the
same counter-based increments, so no carry crosses ranks either.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np


@dataclass(frozen=True)
class Unit:
    work_idx: int
    rx: int
    band: int
    n_samples: int
    n_active: int

    @property
    def cost(self) -> int:  # tx·rx samples, plus the band's own per-sample epilogue
        return self.n_samples * (self.n_active + 1)


def assign(units: Sequence[Unit], world: int) -> list[list[int]]:
    """Work indices per rank: receivers kept whole, longest first onto the
    least-loaded rank (ties to the lowest rank, so every rank computes the
    same plan)."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    by_rx: dict[int, list[Unit]] = {}
    for u in units:
        by_rx.setdefault(u.rx, []).append(u)
    order = sorted(by_rx, key=lambda r: (-sum(u.cost for u in by_rx[r]), r))
    load = [0] * world
    plan: list[list[int]] = [[] for _ in range(world)]
    for r in order:
        k = min(range(world), key=lambda i: (load[i], i))
        load[k] += sum(u.cost for u in by_rx[r])
        plan[k].extend(sorted(u.work_idx for u in by_rx[r]))
    return [sorted(p) for p in plan]


def time_shards(n_samples: int, world: int, align: int = 1024) -> list[tuple[int, int]]:
    """Contiguous (i0, n) ranges of one band, one per rank, starting on
    multiples of `align` (the fan-out's tiles), covering [0, n_samples)."""
    if world < 1 or align < 1:
        raise ValueError("world size and alignment must be >= 1")
    tiles = -(-n_samples // align)
    out, t = [], 0
    for k in range(world):
        nt = tiles // world + (1 if k < tiles % world else 0)
        i0 = min(t * align, n_samples)
        i1 = min((t + nt) * align, n_samples)
        out.append((i0, i1 - i0))
        t += nt
    return out


def scene_units(prep) -> list[Unit]:
    """The work units of a prepared scene (lipika_b200.pipeline.Prepared or
    the oracle's Scene: both expose work(), n_samples() and active())."""
    return [Unit(w, r, b, prep.n_samples(r, b), len(prep.active(r, b))) for w, (r, b) in enumerate(prep.work())]


def checksum(iq: np.ndarray) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(iq).view(np.uint8)).hexdigest()


def gather_manifests(rendered: dict[int, np.ndarray], group=None) -> Optional[dict[int, tuple[int, str]]]:
    """All ranks' {work_idx: (n_samples, sha256)} on rank 0 (None elsewhere)."""
    import torch.distributed as dist
    mine = {w: (int(len(iq)), checksum(iq)) for w, iq in rendered.items()}
    world = dist.get_world_size(group)
    got: list = [None] * world
    dist.all_gather_object(got, mine, group=group)
    if dist.get_rank(group) != 0:
        return None
    out: dict[int, tuple[int, str]] = {}
    for part in got:
        for w, v in part.items():
            if w in out:
                raise RuntimeError(f"work unit {w} rendered on two ranks")
            out[w] = v
    return out


def render_rank(prep, rank: int, world: int, render_unit: Callable[[int, int, int], np.ndarray]) -> dict[int, np.ndarray]:
    """Render this rank's share: render_unit(work_idx, rx, band) -> IQ."""
    units = scene_units(prep)
    mine = set(assign(units, world)[rank])
    return {u.work_idx: render_unit(u.work_idx, u.rx, u.band) for u in units if u.work_idx in mine}


def render_rank_gpu(prep, rank: int, world: int, seed: int, round_s: float, noise: bool = True,
                    split: bool = True) -> dict[int, np.ndarray]:
    """This rank's units through one lpk_batch on this process's context
    (stationary receivers with a deterministic or device-walk clock)."""
    from . import native as N
    units = scene_units(prep)
    mine = assign(units, world)[rank]
    descs = []
    for w in mine:
        u = units[w]
        d = prep.band_desc(u.rx, u.band, seed, w)
        if d.clock_mode == N.LPK_CLOCK_HOST:
            d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
        d.solver = N.LPK_SOLVER_SPLIT if split else N.LPK_SOLVER_REFERENCE
        if not noise:
            d.noise_power_w = 0.0
        descs.append((d, prep.active(u.rx, u.band), u.n_samples))
    if not descs:
        return {}
    b = N.Batch(prep.ctx, descs, round_s)
    out = b.render()
    b.close()
    return dict(zip(mine, out))

"""Batched tissues over several GPUs: whole tissues per rank, no collective on the data path.

A batch of independent tissues shards naturally: each rank (one process per GPU) takes a subset of
the tissues, runs them as one batched context on its own GPU, and the host gathers the final
positions at the end. Tissues are assigned by greedy longest-processing-time bin packing on an
estimate of each tissue's work per step, prisms x sqrt(nodes): the element work grows with the
prism count and the BiCGStab iteration count with the mesh's linear size.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np


def tissue_weight(n_elems: int, n_nodes: int) -> float:
    """Expected work of one implicit step of a tissue (arbitrary units)."""
    return float(n_elems) * float(np.sqrt(max(n_nodes, 1)))


def shard_tissues(weights: Sequence[float], world: int) -> List[List[int]]:
    """Assign tissue indices to `world` ranks: heaviest first, each to the least-loaded rank
    (ties to the lower rank). Every rank's list is returned in ascending tissue order; the
    assignment depends only on the weights, so every rank computes the same one."""
    if world <= 0:
        raise ValueError("world must be positive")
    w = np.asarray(weights, dtype=np.float64)
    if np.any(~np.isfinite(w)) or np.any(w < 0):
        raise ValueError("weights must be finite and non-negative")
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += w[i]
    return [sorted(s) for s in out]


def shard_loads(weights: Sequence[float], shards: Sequence[Sequence[int]]) -> List[float]:
    w = np.asarray(weights, dtype=np.float64)
    return [float(w[list(s)].sum()) if len(s) else 0.0 for s in shards]


class ShardedBatch:
    """This rank's share of a batch of tissues.

    `make_solver(tissues)` builds the batched context for the rank's tissues (``BatchSolver`` on
    the rank's GPU in production; any object with ``join``, ``split`` and
    ``runOneStep(x, dt) -> (x, rc, stats)`` works). `gather` collects every rank's final positions
    on the host in the original tissue order through ``torch.distributed.all_gather_object``
    (host objects only: the GPU data path has no collective).
    """

    def __init__(self, tissues, rank: int, world: int, make_solver: Callable, weights: Optional[Sequence[float]] = None):
        self.tissues = list(tissues)
        self.rank, self.world = int(rank), int(world)
        if weights is None:
            weights = [tissue_weight(t.n_elems, t.n_nodes) for t in self.tissues]
        self.shards = shard_tissues(weights, self.world)
        self.mine = self.shards[self.rank]
        self.solver = make_solver([self.tissues[i] for i in self.mine]) if self.mine else None

    @property
    def n_elems(self) -> int:
        return int(sum(self.tissues[i].n_elems for i in self.mine))

    def initial_positions(self):
        if self.solver is None:
            return None
        return self.solver.join([self.tissues[i].x for i in self.mine])

    def run(self, n_steps: int, dt: float):
        """Run n_steps on this rank's tissues; returns ({tissue index: positions}, per-step stats)."""
        if self.solver is None:
            return {}, []
        x = self.initial_positions()
        stats = []
        for _ in range(n_steps):
            x, rc, st = self.solver.runOneStep(x, dt)
            st = dict(st)
            st["rc"] = rc
            stats.append(st)
        return dict(zip(self.mine, self.solver.split(x))), stats

    def gather(self, local: dict, group=None):
        """All ranks' {tissue index: positions} merged into a list in tissue order (every rank
        receives it). Without an initialised process group this rank's results are returned."""
        import torch.distributed as dist

        if not (dist.is_available() and dist.is_initialized()):
            parts = [local]
        else:
            parts = [None] * dist.get_world_size(group)
            dist.all_gather_object(parts, {int(k): np.asarray(v) for k, v in local.items()}, group=group)
        merged = {}
        for p in parts:
            for k, v in p.items():
                if k in merged:
                    raise RuntimeError(f"tissue {k} was run on two ranks")
                merged[k] = v
        return [merged.get(i) for i in range(len(self.tissues))]

    def close(self):
        if self.solver is not None and hasattr(self.solver, "close"):
            self.solver.close()
        self.solver = None

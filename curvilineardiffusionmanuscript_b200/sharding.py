"""Multi-GPU sharding of independent APT problems (one process per GPU).

A batch of independent problems (the reference runs one `step!` per problem)
partitions without any exchange of field data: each rank steps the problems
assigned to it on its own GPU, and only the per-problem statistics are
gathered on the host.  Problems are assigned longest-processing-time first by
their cost (cells, optionally × expected pseudo-iterations), which bounds the
slowest rank at 4/3 of the optimum.

Collectives here are host-side bookkeeping (statistics, timing maxima) over
whatever process group is initialised: NCCL on GPUs, gloo on CPU (the tests).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import torch
import torch.distributed as dist


def world() -> tuple:
    """(rank, world_size) of the default process group, (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def reduce_max(x: float) -> float:
    """Maximum of x over ranks (the job's time is the slowest rank's)."""
    r, ws = world()
    if ws == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float) -> float:
    """Sum of x over ranks (whole-job work)."""
    r, ws = world()
    if ws == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def lpt_assign(costs: Sequence[float], nranks: int) -> List[List[int]]:
    """Longest-processing-time-first assignment of problem indices to ranks;
    ties go to the lowest rank, so every rank computes the same assignment."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * nranks
    out: List[List[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


class ShardError(RuntimeError):
    """A rank's step failed; raised on every rank with the failed ranks' errors."""


class ShardedBatch:
    """A batch of problems split over the ranks of the default process group.

    Every rank is given the full lists (meshes, boundary conditions, and at each
    step the arrays of all problems); it builds a local batch of its own
    problems only and updates only their temperature arrays.  `step` returns
    the statistics of all problems in the global order on every rank.
    """

    def __init__(self, meshes, bcs, costs: Optional[Sequence[float]] = None,
                 make_batch: Optional[Callable] = None, **batch_kwargs):
        if costs is None:
            costs = [m.ni * m.nj * max(1, getattr(m, "nk", 1) or 1) for m in meshes]
        self._setup(costs, lambda idx: ([meshes[i] for i in idx], [bcs[i] for i in idx]), make_batch,
                    batch_kwargs)

    @classmethod
    def from_factory(cls, costs: Sequence[float], build: Callable, make_batch: Optional[Callable] = None,
                     **batch_kwargs) -> "ShardedBatch":
        """A sharded batch whose ranks build only their own problems:
        build(indices) -> (meshes, bcs) of those global problem indices."""
        self = cls.__new__(cls)
        self._setup(costs, build, make_batch, batch_kwargs)
        return self

    def _setup(self, costs, build, make_batch, batch_kwargs):
        self.rank, self.world = world()
        self.n = len(costs)
        self.assignment = lpt_assign(costs, self.world)
        self.local = self.assignment[self.rank]
        if make_batch is None:
            from .solver import PseudoTransientBatch
            make_batch = PseudoTransientBatch
        self.batch = None
        if self.local:
            meshes, bcs = build(self.local)
            self.batch = make_batch(meshes, bcs, **batch_kwargs)

    def _pick(self, xs):
        return [xs[i] for i in self.local]

    def step(self, Ts, rhos, cps, kappas, dts, **kwargs):
        """Steps this rank's problems, then gathers every problem's statistics.
        A rank whose own step fails still takes part in the gather, with its
        error in place of statistics, so that every rank takes the same
        collective steps and raises the same ShardError instead of waiting for
        the failed rank until the process group's timeout."""
        stats, ndts, err = [], [], None
        if self.batch is not None:
            try:
                stats, ndts = self.batch.step(self._pick(Ts), self._pick(rhos), self._pick(cps),
                                              self._pick(kappas), self._pick(dts), **kwargs)
            except Exception as e:  # reported on every rank after the gather
                err = f"rank {self.rank}: {type(e).__name__}: {e}"
        mine = (err, list(zip(self.local, stats, ndts)))
        if self.world > 1:
            parts: list = [None] * self.world
            dist.all_gather_object(parts, mine)
        else:
            parts = [mine]
        errors = [e for e, _ in parts if e]
        if errors:
            raise ShardError("; ".join(errors))
        all_stats: list = [None] * self.n
        all_ndt: list = [None] * self.n
        for _, part in parts:
            for i, st, nd in part:
                all_stats[i] = st
                all_ndt[i] = nd
        return all_stats, all_ndt

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None

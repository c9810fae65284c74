"""Multi-rank host logic of the sharded batch, as world-size-2 gloo process
groups on CPU (no GPU): assignment, statistics gather, timing reductions, and
failures made on the host (a rank whose step raises, a rank that leaves)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from curvilineardiffusionmanuscript_b200.sharding import ShardError, ShardedBatch, lpt_assign, reduce_max, reduce_sum


class FakeMesh:
    def __init__(self, n):
        self.ni = self.nj = n
        self.nk = 1


class FakeBatch:
    """Stands in for PseudoTransientBatch: records its problems and returns
    per-problem statistics derived from them."""

    def __init__(self, meshes, bcs, **kw):
        self.sizes = [m.ni for m in meshes]
        self.bcs = bcs

    def step(self, Ts, rhos, cps, kappas, dts, **kw):
        for T in Ts:
            T += 1.0
        return [{"niter": s, "bc": b} for s, b in zip(self.sizes, self.bcs)], [d * 2 for d in dts]

    def close(self):
        pass


def test_lpt_assignment_covers_and_balances():
    costs = [9, 7, 6, 5, 4, 4, 3, 1]
    parts = lpt_assign(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= 4 / 3 * (sum(costs) / 3) + max(costs)
    assert lpt_assign(costs, 1) == [list(range(len(costs)))]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [64, 512, 128, 96, 300, 200, 80]
        meshes = [FakeMesh(n) for n in sizes]
        bcs = [f"bc{i}" for i in range(len(sizes))]
        sb = ShardedBatch(meshes, bcs, make_batch=FakeBatch)
        Ts = [torch.zeros(3) for _ in sizes]
        stats, ndt = sb.step(Ts, [None] * 7, [1.0] * 7, [None] * 7, [0.5 * (i + 1) for i in range(7)])
        updated = [i for i, T in enumerate(Ts) if float(T[0]) == 1.0]
        tmax = reduce_max(10.0 + rank)
        tsum = reduce_sum(rank + 1)
        q.put((rank, sb.local, updated, [s["niter"] for s in stats], [s["bc"] for s in stats], ndt, tmax, tsum))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [64, 512, 128, 96, 300, 200, 80]
    l0, l1 = res[0][1], res[1][1]
    assert sorted(l0 + l1) == list(range(7)) and not set(l0) & set(l1)
    for rank, local, updated, niters, bcs, ndt, tmax, tsum in res:
        # each rank updates only its own problems' arrays
        assert updated == local
        # statistics of every problem, in global order, on every rank
        assert niters == sizes and bcs == [f"bc{i}" for i in range(7)]
        assert ndt == [1.0 * (i + 1) for i in range(7)]
        assert tmax == 11.0 and tsum == 3.0
    # the heaviest problem (512²) sits alone with lighter ones on its rank
    cost = [n * n for n in sizes]
    loads = [sum(cost[i] for i in r[1]) for r in res]
    assert max(loads) <= 1.34 * max(max(cost), sum(cost) / 2)


class FailingBatch(FakeBatch):
    """A FakeBatch whose step raises on the rank that holds the 512² problem."""

    def step(self, Ts, rhos, cps, kappas, dts, **kw):
        if 512 in self.sizes:
            raise RuntimeError("injected failure")
        return super().step(Ts, rhos, cps, kappas, dts, **kw)


def _put_and_exit(q, item):
    # flush the queue's feeder thread before leaving without interpreter teardown
    q.put(item)
    q.close()
    q.join_thread()
    os._exit(0)


def _failure_worker(rank, world, port, q, mode):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import time
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    sizes = [64, 512, 128, 96, 300, 200, 80]
    meshes = [FakeMesh(n) for n in sizes]
    sb = ShardedBatch(meshes, [None] * 7, make_batch=FailingBatch if mode == "raise" else FakeBatch)
    args = ([torch.zeros(3) for _ in sizes], [None] * 7, [1.0] * 7, [None] * 7, [1.0] * 7)
    if mode == "leave" and rank == 1:
        _put_and_exit(q, (rank, "left", 0.0))  # leaves between steps, with no collective in flight
    t0 = time.time()
    try:
        sb.step(*args)
        out = (rank, "ok", time.time() - t0)
    except ShardError as e:
        out = (rank, "ShardError: " + str(e), time.time() - t0)
    except Exception as e:  # the process group reports the missing peer
        out = (rank, type(e).__name__, time.time() - t0)
    _put_and_exit(q, out)


def _run_failure(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failure_worker, args=(r, 2, port, q, mode)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_a_failing_rank_is_reported_on_every_rank():
    """The rank holding the 512² problem raises in its step; both ranks finish
    the gather and raise the same ShardError naming it."""
    res = _run_failure("raise")
    failed = 0 if 1 in lpt_assign([n * n for n in [64, 512, 128, 96, 300, 200, 80]], 2)[0] else 1
    for rank, what, dt in res:
        assert what.startswith("ShardError") and f"rank {failed}" in what and "injected failure" in what, what
        assert dt < 15.0


def test_a_rank_that_leaves_ends_the_others_step_with_an_error():
    """Rank 1 exits between steps; rank 0's statistics gather ends with an error
    (the closed connection, at the latest the process group's 20 s timeout)
    instead of waiting for good."""
    res = _run_failure("leave")
    assert res[1][1] == "left"
    rank, what, dt = res[0]
    assert what != "ok" and dt < 60.0, (what, dt)


def _factory_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [64, 512, 128, 96, 300, 200, 80]
        built = []

        def build(idx):
            built.extend(idx)
            return [FakeMesh(sizes[i]) for i in idx], [f"bc{i}" for i in idx]

        sb = ShardedBatch.from_factory([n * n for n in sizes], build, make_batch=FakeBatch)
        # the bench's calling convention: global-order lists holding this rank's entries only
        Ts = [torch.zeros(3) if i in sb.local else None for i in range(7)]
        stats, _ = sb.step(Ts, [None] * 7, [1.0] * 7, [None] * 7, [1.0] * 7)
        q.put((rank, sb.local, sorted(built), [s["niter"] for s in stats]))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_from_factory_builds_only_local_problems():
    """ShardedBatch.from_factory: every rank builds only the problems LPT gives
    it, and still receives every problem's statistics."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_factory_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [64, 512, 128, 96, 300, 200, 80]
    assert sorted(res[0][1] + res[1][1]) == list(range(7))
    for rank, local, built, niters in res:
        assert built == local and niters == sizes


def test_batch_weights_follow_the_expected_iterations():
    """The bench's LPT weights: expected iterations grow with the side and, at
    the batch's larger sides, with the conductivity exponent; on 8 seeded
    batches over 8 ranks the weighted assignment carries less spread of
    expected work than the assignment by cells alone."""
    from curvilineardiffusionmanuscript_b200 import problems as P
    from curvilineardiffusionmanuscript_b200.sharding import lpt_assign
    e = P.batch_expected_iterations
    assert e({"n": 512, "kn": 3.0}) > e({"n": 256, "kn": 3.0}) > e({"n": 64, "kn": 3.0})
    assert e({"n": 400, "kn": 3.0}) > e({"n": 400, "kn": 1.0}) > e({"n": 400, "kn": 0.0})
    params = [q for r in range(8) for q in P.batch_2d_params(256, seed=P.BATCH_SEED + r)]
    cells = [q["n"] ** 2 for q in params]
    work = [c * e(q) for c, q in zip(cells, params)]

    def spread(assign):
        loads = [sum(work[i] for i in a) for a in assign]
        return max(loads) / (sum(loads) / len(loads))

    assert spread(lpt_assign(work, 8)) < spread(lpt_assign(cells, 8))
    assert spread(lpt_assign(work, 8)) < 1.01

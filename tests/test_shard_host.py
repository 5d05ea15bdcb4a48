"""Sharding one problem over ranks: the host side, on CPU.

The plan (fss_shard_partition: contiguous unit ranges of near-equal counted
cost) is checked against a brute-force optimum and must come out the same on
every rank; the exchange (each rank's own rows, -0.0 elsewhere, summed by an
all-reduce) must give every rank every row bit for bit; and the driver in
fss_b200.shard (per stage: own targets, all-reduce, combine) must give two
gloo ranks the one-rank trajectory bit for bit.  The GPU evaluation of a rank
is stood in for by a CPU context built on the oracle (rhs_eval.h:15-56 for
its own rows); tests/test_gpu_shard.py runs the library's own shard
contexts.  Two gloo ranks, rendezvous on 127.0.0.1.
"""
import itertools
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "fast-sphere-sum_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def loads(cost, b):
    return [float(np.sum(cost[b[i]:b[i + 1]])) for i in range(len(b) - 1)]


def best_max_load(cost, R):
    """min over contiguous R-way splits of the largest range cost (brute force)."""
    U = len(cost)
    best = np.inf
    for cuts in itertools.combinations(range(1, U), R - 1):
        b = (0,) + cuts + (U,)
        best = min(best, max(loads(cost, b)))
    return best


def test_partition_is_optimal_and_covers(fss):
    rng = np.random.default_rng(3)
    for trial in range(40):
        U = int(rng.integers(4, 11))
        R = int(rng.integers(2, min(U, 5) + 1))
        cost = rng.random(U) ** 3 * (10 if trial % 2 else 1)
        b = fss.shard_partition(cost, R)
        assert b[0] == 0 and b[-1] == U and len(b) == R + 1
        assert np.all(np.diff(b) >= 1)                     # contiguous, every rank has a unit
        assert max(loads(cost, b)) <= best_max_load(cost, R) * (1 + 1e-9)
    # degenerate inputs: zero costs split evenly; as many ranks as units
    assert list(fss.shard_partition(np.zeros(8), 4)) == [0, 2, 4, 6, 8]
    assert list(fss.shard_partition(np.ones(5), 5)) == [0, 1, 2, 3, 4, 5]


class OracleShard:
    """A CPU stand-in for a sharded context with the library's stage
    semantics: the stage's velocity for this rank's rows only (the oracle's
    direct sum), -0.0 in the other rows of the exchange buffer; the combine
    advances every particle (RK4 of new_dynamics.cpp:170-229, project_points
    of helpers.h:362-372)."""

    def __init__(self, oracle, state, area, lo, hi):
        self.O, self.s0, self.area, self.lo, self.hi = oracle, state.copy(), area, lo, hi
        self.n = state.shape[0]
        self.xs = self.s0.copy()
        self.acc = None

    def shard_stage(self, stage, ex):
        rows = np.arange(self.lo, self.hi)
        u = self.O.rhs_direct_rows(self.xs, self.area, rows, threads=2)
        buf = np.full((self.n, 4), -0.0)
        buf[rows, :3] = u
        buf[rows, 3] = 0.0
        ex.copy_(__import__("torch").from_numpy(buf))

    def shard_combine(self, stage, dt, ex, omega):
        X = ex.numpy()
        k = np.concatenate([X[:, :3], (-2 * omega * X[:, 2])[:, None]], axis=1)
        if stage == 1:
            self.acc = k.copy()
        else:
            self.acc = self.acc + (1.0 if stage == 4 else 2.0) * k
        h = {1: dt / 2, 2: dt / 2, 3: dt}.get(stage, dt / 6)
        t = self.s0[:, :4] + h * (k if stage < 4 else self.acc)
        p = t[:, :3] / np.linalg.norm(t[:, :3], axis=1, keepdims=True)
        z = t[:, 3] + (-2 * omega) * (p[:, 2] - t[:, 2])
        self.xs = self.s0.copy()
        self.xs[:, :3], self.xs[:, 3] = p, z
        if stage == 4:
            self.s0 = self.xs.copy()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        import fss_b200 as F
        import oracle as O
        from fss_b200 import shard
        out = {}
        # 1. the plan, computed independently on every rank
        cost = np.random.default_rng(11).random(80) ** 2
        b = F.shard_partition(cost, ws)
        plans = [None] * ws
        dist.all_gather_object(plans, b.tolist())
        out["plans_equal"] = all(p == plans[0] for p in plans)
        # 2. the exchange: own rows + -0.0 elsewhere, summed over the ranks
        full = np.random.default_rng(5).standard_normal((1000, 4))
        full[::7] = 0.0
        full[3::7] = -0.0
        lo, hi = int(1000 * rank / ws), int(1000 * (rank + 1) / ws)
        t = torch.from_numpy(shard.owned_rows_exact(full, lo, hi))
        shard.torch_allreduce()(t)
        out["exchange_exact"] = bool(np.array_equal(t.numpy().view(np.uint64), full.view(np.uint64)))
        # 3. the driver over the ranks against one rank
        s, a = O.rh_vortices_state(3, 4, 1)
        n = s.shape[0]
        blocks = F.shard_partition(np.ones((n + 63) // 64), ws)
        lo, hi = int(blocks[rank]) * 64, min(n, int(blocks[rank + 1]) * 64)
        ctx = OracleShard(O, s, a, lo, hi)
        ex = torch.empty((n, 4), dtype=torch.float64)
        shard.rk4_steps(ctx, ex, 0.01, nsteps=2, allreduce=shard.torch_allreduce(), omega=O.OMEGA)
        if rank == 0:
            one = OracleShard(O, s, a, 0, n)
            shard.rk4_steps(one, torch.empty((n, 4), dtype=torch.float64), 0.01, nsteps=2, omega=O.OMEGA)
            out["driver_equals_one_rank"] = bool(np.array_equal(ctx.s0.view(np.uint64), one.s0.view(np.uint64)))
            out["moved"] = float(np.abs(ctx.s0[:, :3] - s[:, :3]).max())
        q.put((rank, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_plan_exchange_and_driver():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, out in res.items():
        assert out["plans_equal"] and out["exchange_exact"], (rank, out)
    assert res[0]["driver_equals_one_rank"], res[0]
    assert res[0]["moved"] > 0

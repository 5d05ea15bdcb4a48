"""One problem sharded over ranks, on one GPU: several shard contexts of the
same process stand in for the ranks (each its own context, as each GPU of a
sharded run holds its own), and the exchange buffers are summed on the
device, as the all-reduce of a multi-GPU run sums them.  No kernel of one
context waits on another's.  The sharded trajectory must equal the unsharded
context's bit for bit (same source split, same degrees), every work item must
run on exactly one rank, and the ranks' targets must tile the particles.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    ("treecode mixed, target clusters", dict(method=1, precision=1, degree=8, theta=0.7, cluster_targets=1,
                                             src_parts=2), 5, 2),
    ("treecode mixed, target clusters, 3 ranks", dict(method=1, precision=1, degree=8, theta=0.7,
                                                      cluster_targets=1, src_parts=1), 5, 3),
    ("treecode FP64", dict(method=1, precision=0, degree=8, theta=0.7, src_parts=2), 5, 2),
    ("direct FP64", dict(method=0, precision=0, src_parts=2), 4, 2),
    ("direct mixed, 4 ranks", dict(method=0, precision=1, src_parts=1), 4, 4),
]


def run_sharded(fss, kw, s, a, nranks, steps, dt=0.01):
    import torch
    st = torch.cuda.Stream()               # a real stream (the legacy default would mean "the context's own")
    ctxs = []
    for r in range(nranks):
        c = fss.Context(**kw)
        c.set_stream(st.cuda_stream)   # stages, exchange and combine in one stream order
        c.set_particles(s, a)
        c.shard(r, nranks)
        ctxs.append(c)
    n = s.shape[0]
    bufs = [torch.empty((n, 4), dtype=torch.float64, device="cuda") for _ in range(nranks)]
    total = torch.empty((n, 4), dtype=torch.float64, device="cuda")
    try:
        with torch.cuda.stream(st):
            for _ in range(steps):
                for stage in (1, 2, 3, 4):
                    for c, b in zip(ctxs, bufs):
                        c.shard_stage(stage, b)
                    total.copy_(bufs[0])
                    for b in bufs[1:]:
                        total += b                 # what the all-reduce computes
                    for c in ctxs:
                        c.shard_combine(stage, dt, total)
        st.synchronize()
        states = [c.get_state() for c in ctxs]
        infos = [c.shard_info() for c in ctxs]
        work = [c.work_per_rhs()[0] for c in ctxs]
    finally:
        for c in ctxs:
            c.close()
    return states, infos, work


@pytest.mark.parametrize("name,kw,level,nranks", CASES, ids=[c[0] for c in CASES])
def test_sharded_steps_equal_unsharded(fss, name, kw, level, nranks):
    s, a = fss.make_state(level, "rh_vortices", n_vortex=8, seed=4)
    steps = 3
    with fss.Context(**kw) as one:
        one.set_particles(s, a)
        work_one = one.work_per_rhs()[0]
        one.rk4_step(0.01, nsteps=steps)
        want = one.get_state()
    states, infos, work = run_sharded(fss, kw, s, a, nranks, steps)
    for got in states:
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), name
    assert np.abs(want[:, :3] - s[:, :3]).max() > 0
    # every rank's own targets, together, are all targets exactly once
    assert infos[0]["target_lo"] == 0
    for i in range(nranks - 1):
        assert infos[i]["target_hi"] == infos[i + 1]["target_lo"]
        assert infos[i]["unit_hi"] == infos[i + 1]["unit_lo"]
    assert sum(i["cost_own"] for i in infos) == pytest.approx(infos[0]["cost_total"])
    assert all(i["cost_own"] > 0 for i in infos)
    # every interaction is evaluated by exactly one rank
    assert sum(work) == pytest.approx(work_one, rel=1e-12)


def test_one_rank_shard_equals_unsharded(fss):
    """nranks = 1: the sharded driver alone (no exchange) is the plain step."""
    import torch
    from fss_b200 import shard
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=2)
    kw = dict(method=1, precision=1, degree=8, theta=0.7, cluster_targets=1, src_parts=2)
    with fss.Context(**kw) as one:
        one.set_particles(s, a)
        one.rk4_step(0.01, nsteps=2)
        want = one.get_state()
    with fss.Context(**kw) as c:
        c.set_particles(s, a)                     # the context's own stream
        c.shard(0, 1)
        ex = shard.exchange_buffer(c, "cuda")
        torch.cuda.synchronize()                  # the buffer exists before the context's stream uses it
        shard.rk4_steps(c, ex, 0.01, nsteps=2)
        got = c.get_state()
        c.shard(0, 0)                         # unshard: the full lists again
        assert c.shard_info()["nranks"] == 0
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))

"""The pair kernel's bounded waits, made to run out on purpose.

Every wait of the pair kernel on its tile ring gives up after the context's
wait_limit_us and the call returns FSS_ERR_TIMEOUT.  The test hook
fss_test_hold_tile makes one block of the next evaluation withhold its first
source tile (no copy issued, arrival never signalled -- a flag that nothing
sets), so that block's waits run out; the block waits for the copies it did
issue, then exits.  The call must report FSS_ERR_TIMEOUT, the error word must
be cleared, and the next call on the same context must give the normal
result.  No GPU fault is involved: the kernel returns on its own.  The same
for the batched V^-1 kernels' one wait, on the bulk copy of their matrix:
fss_test_hold_stage makes block 0 of the proxy-charge or cluster-coefficient
launch expect that copy without issuing it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TIMEOUT = 4
LIMIT_US = 20000  # 20 ms: far above any normal wait, short for the test


@pytest.fixture(scope="module")
def field(fss):
    return fss.make_state(5, "rh_vortices", n_vortex=8, seed=1)


@pytest.mark.parametrize("method,prec", [(1, 1), (1, 0), (0, 1), (0, 0)])
def test_wait_runs_out_then_context_recovers(fss, field, method, prec):
    s, a = field
    with fss.Context(method=method, precision=prec, degree=8, wait_limit_us=LIMIT_US) as ctx:
        ctx.set_particles(s, a)
        expect = ctx.rhs(s, a)
        for block in (0, 7):
            ctx.test_hold_tile(block)
            with pytest.raises(fss.FssError) as e:
                ctx.rhs(s, a)
            assert e.value.code == TIMEOUT, str(e.value)
            got = ctx.rhs(s, a)  # hook cleared, error word cleared
            assert np.array_equal(got.view(np.uint64), expect.view(np.uint64))


def test_rk4_step_reports_timeout_and_next_step_matches(fss, field):
    s, a = field
    with fss.Context(method=1, precision=1, wait_limit_us=LIMIT_US) as ref_ctx:
        ref_ctx.set_particles(s, a)
        want = ref_ctx.rk4_step_host(s.copy(), 0.01)
    with fss.Context(method=1, precision=1, wait_limit_us=LIMIT_US) as ctx:
        ctx.set_particles(s, a)
        ctx.test_hold_tile(3)
        with pytest.raises(fss.FssError) as e:
            ctx.rk4_step_host(s.copy(), 0.01)
        assert e.value.code == TIMEOUT
        got = ctx.rk4_step_host(s.copy(), 0.01)  # from the same host state again
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_default_limit_is_two_seconds(fss, field):
    """wait_limit_us = 0 keeps the 2 s default; normal runs never time out."""
    s, a = field
    with fss.Context(method=1, precision=1) as ctx:
        ctx.set_particles(s, a)
        ctx.rk4_step(0.01, nsteps=3)
        assert np.all(np.isfinite(ctx.get_state()))


@pytest.mark.parametrize("which", [0, 1], ids=["proxy charges", "cluster coefficients"])
def test_batched_staging_wait_runs_out_then_context_recovers(fss, field, which):
    s, a = field
    with fss.Context(method=1, precision=1, degree=8, cluster_targets=1, wait_limit_us=LIMIT_US) as ctx:
        ctx.set_particles(s, a)
        assert ctx.tree_info()["target_clusters"] > 0
        expect = ctx.rhs(s, a)
        ctx.test_hold_stage(which)
        with pytest.raises(fss.FssError) as e:
            ctx.rhs(s, a)
        assert e.value.code == TIMEOUT, str(e.value)
        got = ctx.rhs(s, a)  # hook cleared, error word cleared
        assert np.array_equal(got.view(np.uint64), expect.view(np.uint64))

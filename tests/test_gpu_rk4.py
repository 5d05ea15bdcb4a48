"""Fused RK4 stage combine + renormalisation on the GPU (new_dynamics.cpp
RK4 order, helpers.h:362 project_points) against the oracle's RK4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rk4_direct_fp64_matches_oracle(fss, oracle):
    s, a = fss.make_state(3, "rh4_ref")
    ref = oracle.rk4_step(oracle.rk4_step(s, a, 0.01), a, 0.01)
    with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_FP64) as ctx:
        ctx.set_particles(s, a)
        ctx.rk4_step(0.01, nsteps=2)
        out = ctx.get_state()
    assert np.max(np.abs(out[:, :3] - ref[:, :3])) < 1e-13
    assert np.max(np.abs(out[:, 3] - ref[:, 3])) < 1e-10 * np.max(np.abs(ref[:, 3]))
    assert np.array_equal(out[:, 4], s[:, 4])                        # tracer untouched
    assert np.allclose(np.linalg.norm(out[:, :3], axis=1), 1.0, atol=1e-15)


def test_rk4_graph_equals_eager(fss):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=4, seed=3)
    outs = []
    for g in (0, 1):
        with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, use_graph=g) as ctx:
            ctx.set_particles(s, a)
            ctx.rk4_step(0.01, nsteps=3)
            outs.append(ctx.get_state())
    assert np.array_equal(outs[0], outs[1])


def test_rk4_host_equals_device(fss):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=4, seed=3)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        ctx.rk4_step(0.01, nsteps=2)
        dev = ctx.get_state()
        # the same start again after two steps: the particles were re-sorted
        # in between, so sums run in another order (equal to rounding)
        again = ctx.rk4_step_host(np.ascontiguousarray(s.copy()), 0.01, nsteps=2)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        host = ctx.rk4_step_host(np.ascontiguousarray(s.copy()), 0.01, nsteps=2)
    assert np.array_equal(dev, host)
    disp = dev[:, :3] - s[:, :3]
    assert np.linalg.norm(again[:, :3] - dev[:, :3]) / np.linalg.norm(disp) < 1e-6
    assert np.array_equal(again[:, 4], dev[:, 4])


def test_rhs_between_steps_does_not_disturb(fss):
    """A stand-alone right-hand side between steps leaves the trajectory alone."""
    s, a = fss.make_state(5, "rh_vortices", n_vortex=4, seed=3)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64) as c1:
        c1.set_particles(s, a)
        c1.rk4_step(0.01, nsteps=2)
        ref = c1.get_state()
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64) as c2:
        c2.set_particles(s, a)
        c2.rk4_step(0.01, nsteps=1)
        c2.rhs(s * 1.0, a)
        c2.rk4_step(0.01, nsteps=1)
        out = c2.get_state()
    assert np.array_equal(out, ref)


def test_rk4_treecode_tracks_direct(fss):
    """Ten steps of the mixed treecode stay on the FP64 direct trajectory."""
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=1)
    out = {}
    for method, prec in ((fss.METHOD_DIRECT, fss.PREC_FP64), (fss.METHOD_TREECODE, fss.PREC_MIXED)):
        with fss.Context(method=method, precision=prec, degree=8, theta=0.7) as ctx:
            ctx.set_particles(s, a)
            ctx.rk4_step(0.01, nsteps=10)
            out[method] = ctx.get_state()
    disp_d = out[0][:, :3] - s[:, :3]
    disp_t = out[1][:, :3] - s[:, :3]
    # relative L2 error of the displacement, of the order of the RHS error
    err = np.linalg.norm(disp_t - disp_d) / np.linalg.norm(disp_d)
    assert err < 2e-6, err
    dz = np.linalg.norm(out[0][:, 3] - out[1][:, 3]) / np.linalg.norm(out[0][:, 3])
    assert dz < 1e-6


def test_rhs_current_matches_rhs(fss):
    s, a = fss.make_state(4, "rh_vortices", n_vortex=4, seed=2)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        m1 = ctx.rhs_current()
        m2 = ctx.rhs(s, a)
    assert np.array_equal(m1, m2)


def test_non_finite_positions_are_reported(fss):
    """A NaN position fails every point-in-face test; the tree assignment
    and the per-step re-sort report it (FSS_ERR_INVALID) instead of piling
    such particles into one leaf, and a diverged state costs no more than a
    normal step."""
    import time
    s, a = fss.make_state(5, "rh_vortices", n_vortex=4, seed=1)
    bad = s.copy()
    bad[7, 0] = np.nan
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        with pytest.raises(fss.FssError):
            ctx.set_particles(bad, a)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        ctx.rk4_step(0.01, nsteps=1)
        diverged = np.ascontiguousarray(s.copy())
        diverged[:, :3] = np.nan
        t0 = time.perf_counter()
        with pytest.raises(fss.FssError):
            ctx.rk4_step_host(diverged, 0.01)
        assert time.perf_counter() - t0 < 5.0

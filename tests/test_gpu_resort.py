"""Re-sorting particles into the leaves they are in now at every RK4 step
(FSS_REBUILD_RESORT, the default for complete assignment) against the
reference's fixed tree (FSS_REBUILD_STATIC; new_dynamics.cpp:87-88 assigns
once before the time loop) and the FP64 direct sum."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _steps(fss, s, a, nsteps, **kw):
    with fss.Context(**kw) as ctx:
        ctx.set_particles(s, a)
        ctx.rk4_step(0.01, nsteps=nsteps)
        loc = ctx.get_tree()[0] if kw.get("method", fss.METHOD_TREECODE) == fss.METHOD_TREECODE else None
        return ctx.get_state(), loc


def test_resort_membership_follows_particles(fss, oracle):
    """After k steps the leaves are those of the state at the start of step k."""
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=4)
    kw = dict(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, tree_levels=4, rebuild=fss.REBUILD_RESORT)
    _, loc0 = _steps(fss, s, a, 0, **kw)
    s5, _ = _steps(fss, s, a, 5, **kw)
    _, loc6 = _steps(fss, s, a, 6, **kw)
    ref = oracle.points_assign(4, s5)
    ok = ref[3] >= 0
    # the oracle takes the first containing face, the re-sort keeps the
    # previous leaf while it still contains the particle: they differ only
    # for particles on a shared edge
    agree = np.mean(loc6[3][ok] == ref[3][ok])
    assert agree > 0.995, agree
    assert np.any(loc6[3] != loc0[3])             # particles changed leaves
    for l in range(3):
        assert np.array_equal(loc6[l], loc6[3] >> (2 * (3 - l)))


def test_static_policy_keeps_build_membership(fss):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=4)
    kw = dict(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, tree_levels=4, rebuild=fss.REBUILD_STATIC)
    _, loc0 = _steps(fss, s, a, 0, **kw)
    _, loc3 = _steps(fss, s, a, 3, **kw)
    assert np.array_equal(loc0, loc3)


@pytest.mark.parametrize("list_mode", [0, 1])
def test_resort_tracks_direct_over_many_steps(fss, list_mode):
    """Twenty steps of a vortex field (particles cross many leaves)."""
    s, a = fss.make_state(6, "rh_vortices", n_vortex=16, seed=11)
    ref, _ = _steps(fss, s, a, 20, method=fss.METHOD_DIRECT, precision=fss.PREC_FP64)
    got, _ = _steps(fss, s, a, 20, method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, degree=8, theta=0.7,
                    list_mode=list_mode, rebuild=fss.REBUILD_RESORT)
    assert np.all(np.isfinite(got))
    disp = ref[:, :3] - s[:, :3]
    err = np.linalg.norm(got[:, :3] - ref[:, :3]) / np.linalg.norm(disp)
    assert err < 2e-6, err
    dz = np.linalg.norm(got[:, 3] - ref[:, 3]) / np.linalg.norm(ref[:, 3])
    assert dz < 1e-6, dz
    assert np.array_equal(got[:, 4], s[:, 4])    # tracers ride along with their particles


def test_resort_graph_equals_eager(fss):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=12)
    outs = [_steps(fss, s, a, 4, method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, use_graph=g,
                   rebuild=fss.REBUILD_RESORT)[0] for g in (0, 1)]
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("precision,use_graph,dt,level,tree_levels",
                         [("mixed", 1, 0.01, 6, 5), ("mixed", 0, 0.01, 6, 5), ("fp64", 1, 0.01, 6, 5),
                          ("mixed", 1, 0.05, 6, 3)])
def test_partition_resort_equals_radix_sort(fss, precision, use_graph, dt, level, tree_levels):
    """The per-step re-sort by partition of the old order (the default) and
    the radix key sort both give the stable order of the new leaf keys: the
    states, the leaf membership and the leaf counts agree to the bit.  The
    second step's re-sort moves the particles that crossed leaves in the
    first; with 128 particles per leaf at dt = 0.05 about a quarter of them
    change leaves and some leaf receives more than a warp's 32 movers (69
    in the oracle's step)."""
    s, a = fss.make_state(level, "rh_vortices", n_vortex=16, seed=21)
    prec = fss.PREC_MIXED if precision == "mixed" else fss.PREC_FP64
    outs = []
    for mode in (0, 1):
        with fss.Context(method=fss.METHOD_TREECODE, precision=prec, tree_levels=tree_levels, use_graph=use_graph,
                         rebuild=fss.REBUILD_RESORT) as ctx:
            ctx.test_resort_mode(mode)
            ctx.set_particles(s, a)
            loc0 = ctx.get_tree()[0][-1]
            ctx.rk4_step(dt, nsteps=2)
            loc, counts, _ = ctx.get_tree()
            outs.append((ctx.get_state(), loc, counts))
    moved = loc[-1] != loc0
    assert moved.any()
    if tree_levels == 3:
        assert np.bincount(loc[-1][moved]).max() > 32
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][2], outs[1][2])


def test_resort_mode_rejects_unknown(fss):
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        with pytest.raises(fss.FssError):
            ctx.test_resort_mode(2)


@pytest.mark.parametrize("level,tree_levels,precision", [(4, 1, "mixed"), (4, 2, "fp64"), (3, 5, "mixed")])
def test_partition_resort_edge_trees(fss, level, tree_levels, precision):
    """The partition re-sort against the radix sort on the trees at its
    edges: leaves on level 0 (the root faces: every mover descends from the
    root, no ancestor to start below), leaves on level 1, and more leaves
    (5,120) than particles (642), so that most leaves are empty and stay or
    become empty between steps."""
    s, a = fss.make_state(level, "rh_vortices", n_vortex=8, seed=5)
    prec = fss.PREC_MIXED if precision == "mixed" else fss.PREC_FP64
    outs = []
    for mode in (0, 1):
        with fss.Context(method=fss.METHOD_TREECODE, precision=prec, tree_levels=tree_levels,
                         rebuild=fss.REBUILD_RESORT) as ctx:
            ctx.test_resort_mode(mode)
            ctx.set_particles(s, a)
            loc0 = ctx.get_tree()[0][-1]
            ctx.rk4_step(0.05, nsteps=3)
            loc, counts, _ = ctx.get_tree()
            outs.append((ctx.get_state(), loc, counts))
    assert np.any(loc[-1] != loc0)
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][2], outs[1][2])

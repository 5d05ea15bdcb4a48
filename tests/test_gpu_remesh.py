"""The remesh step on the GPU (remesh.h:109-178 regrid_points2, helpers.h:251
tri_interp) against the oracle, which is bit-exact with the reference's
own code for the same vertex -> triangles adjacency."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _moved(oracle, level, scale, seed, far=0):
    s, _, tris = oracle.icos_state(level)
    h = np.sqrt(4 * np.pi / s.shape[0])
    rng = np.random.default_rng(seed)
    m = s.copy()
    d = scale * h * rng.standard_normal((s.shape[0], 3))
    if far:
        d[rng.choice(s.shape[0], far, replace=False)] *= 3.0 / scale
    m[:, :3] += d
    m[:, :3] /= np.linalg.norm(m[:, :3], axis=1, keepdims=True)
    m[:, 3] += 0.1 * rng.standard_normal(s.shape[0])
    return m, s, tris


@pytest.mark.parametrize("level,scale,far", [(4, 0.05, 0), (4, 0.3, 12), (6, 0.2, 40), (6, 0.2, 400)])
def test_remesh_bit_exact_vs_oracle(fss, oracle, level, scale, far):
    m, s, tris = _moved(oracle, level, scale, seed=level + far, far=far)
    ref, fb_ref, bad_ref = oracle.remesh(m, s, tris)
    got, fb, bad = fss.remesh(m, s, tris)
    assert bad == bad_ref == 0 and fb == fb_ref
    if far:
        assert fb > 0
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


def test_remesh_current_after_rk4_steps(fss, oracle):
    """The device-resident variant: regrid the state reached after RK4 steps
    onto the starting grid, bit-exact with the oracle on that state, then
    keep stepping."""
    level = 5
    s, a = fss.make_state(level, "rh_vortices", n_vortex=8, seed=5)
    _, tris = fss.icos_grid(level)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        ctx.rk4_step(0.01, nsteps=5)
        moved = ctx.get_state()
        target = moved.copy()
        target[:, :3] = s[:, :3]
        ref, fb_ref, bad_ref = oracle.remesh(moved, target, tris)
        fb, bad = ctx.remesh_current(tris)
        got = ctx.get_state()
        assert bad == bad_ref == 0 and fb == fb_ref
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
        ctx.rk4_step(0.01, nsteps=2)
        assert np.all(np.isfinite(ctx.get_state()))


def test_remesh_rejects_bad_triangles(fss, oracle):
    s, _, tris = oracle.icos_state(3)
    bad = tris.copy()
    bad[0, 0] = s.shape[0]
    with pytest.raises(fss.FssError):
        fss.remesh(s, s, bad)



def test_remesh_many_fallbacks_cell_grid(fss, oracle):
    """Hundreds of points outside their adjacent triangles, on a mesh
    tangled enough that some triangles go to the always-tested list: the
    cell-grid search picks the same (first) triangle as the oracle's scan."""
    m, s, tris = _moved(oracle, 5, 1.5, seed=1)
    ref, fb_ref, bad_ref = oracle.remesh(m, s, tris)
    got, fb, bad = fss.remesh(m, s, tris)
    assert fb == fb_ref and fb > 64 and bad == bad_ref
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


def test_remesh_current_cached_adjacency(fss, oracle):
    """Repeated regrids with the same triangles reuse the device adjacency;
    a bad triangle list in between is refused and the next call rebuilds; a
    call without triangles uses those of the previous call."""
    level = 5
    s, a = fss.make_state(level, "rh_vortices", n_vortex=8, seed=9)
    _, tris = fss.icos_grid(level)
    bad = tris.copy()
    bad[7, 1] = -1
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        with pytest.raises(fss.FssError):
            ctx.remesh_current()  # nothing to reuse yet
        for k in range(3):
            ctx.rk4_step(0.02, nsteps=2)
            moved = ctx.get_state()
            target = moved.copy()
            target[:, :3] = s[:, :3]
            ref, fb_ref, _ = oracle.remesh(moved, target, tris)
            if k == 1:
                with pytest.raises(fss.FssError):
                    ctx.remesh_current(bad)
            # the last call passes no triangles: those of the previous call
            fb, nf = ctx.remesh_current(None if k == 2 else tris)
            assert fb == fb_ref and nf == 0
            assert np.array_equal(ctx.get_state().view(np.uint64), ref.view(np.uint64))


def test_remesh_lists_follow_list_order(fss, oracle):
    """fss_remesh_lists tries each vertex's triangles in the order of its
    vert_tris list (here shuffled), as regrid_points2 does with the lists it
    reads; bit-exact with the oracle ordered by the same lists."""
    from test_state_files import list_keys
    m, s, tris = _moved(oracle, 5, 0.4, seed=8, far=25)
    n = s.shape[0]
    lists = [[] for _ in range(n)]
    for j, t in enumerate(tris):
        for v in t:
            lists[v].append(j)
    rng = np.random.default_rng(1)
    lists = [list(rng.permutation(l)) for l in lists]
    off = np.concatenate([[0], np.cumsum([len(l) for l in lists])]).astype(np.int32)
    adj = np.concatenate(lists).astype(np.int32)
    ref, fb_ref, bad_ref = oracle.remesh(m, s, tris, keys=list_keys(tris, off, adj))
    got, fb, bad = fss.remesh_lists(m, s, tris, off, adj)
    assert (fb, bad) == (fb_ref, bad_ref) and fb > 0
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    with pytest.raises(fss.FssError):
        fss.remesh_lists(m, s, tris, off[::-1].copy(), adj)  # offsets must not decrease

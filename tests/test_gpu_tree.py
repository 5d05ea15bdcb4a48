"""GPU tree build (assignment + key sort) and interaction lists against the
oracle's restatement of icos_utils.h:145-190 and fast_rhs.h:16-91."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level,tree_levels", [(3, 2), (4, 3), (5, 3), (5, 4), (6, 4)])
def test_reference_membership_and_pairs_bit_exact(fss, oracle, level, tree_levels):
    s, a = fss.make_state(level, "rh4_ref")
    loc_o = oracle.points_assign(tree_levels, s)
    cnt_o = oracle.level_counts(loc_o, tree_levels)
    pairs_o = oracle.tree_traverse(tree_levels, 0.7, 10, cnt_o)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, tree_levels=tree_levels,
                     theta=0.7, many_count=10, degree=2, assign_mode=fss.ASSIGN_REFERENCE) as ctx:
        ctx.set_particles(s, a)
        loc, cnt, pairs = ctx.get_tree()
        info = ctx.tree_info()
    assert np.array_equal(loc, loc_o)
    assert np.array_equal(cnt, cnt_o)
    assert np.array_equal(pairs, pairs_o)
    assert info["unassigned"] == int((loc_o[-1] < 0).sum())


@pytest.mark.parametrize("level,tree_levels", [(4, 3), (6, 4)])
def test_complete_mode_extends_reference(fss, oracle, level, tree_levels):
    """Complete mode: same faces wherever the reference assigns a particle on
    every level; every particle gets exactly one leaf."""
    s, a = fss.make_state(level, "rh4_ref")
    loc_o = oracle.points_assign(tree_levels, s)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, tree_levels=tree_levels) as ctx:
        ctx.set_particles(s, a)
        loc, cnt, pairs = ctx.get_tree()
    assert (loc >= 0).all()
    keep = (loc_o >= 0).all(axis=0)
    assert np.array_equal(loc[:, keep], loc_o[:, keep])
    # counts are consistent parent/children and sum to N on every level
    off = oracle.face_offsets(tree_levels)
    for l in range(tree_levels):
        lc = cnt[off[l]:off[l] + 20 * 4 ** l]
        assert lc.sum() == s.shape[0]
        if l > 0:
            assert np.array_equal(lc.reshape(-1, 4).sum(1), cnt[off[l - 1]:off[l - 1] + 20 * 4 ** (l - 1)])
    # the pair list follows the reference traversal on these counts
    assert np.array_equal(pairs, oracle.tree_traverse(tree_levels, 0.7, 45, cnt))


def test_moved_particles_membership(fss, oracle):
    """Assignment of perturbed (off-grid) particles, as after RK4 steps."""
    s, a = fss.make_state(5, "rh_vortices", n_vortex=4, seed=5)
    rng = np.random.default_rng(7)
    s[:, :3] += 1e-3 * rng.standard_normal((s.shape[0], 3))
    s[:, :3] /= np.linalg.norm(s[:, :3], axis=1, keepdims=True)
    loc_o = oracle.points_assign(4, s)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, tree_levels=4,
                     assign_mode=fss.ASSIGN_REFERENCE) as ctx:
        ctx.set_particles(s, a)
        loc, _, _ = ctx.get_tree()
    assert np.array_equal(loc, loc_o)

"""Treecode (BLTC) on the GPU against the FP64 direct-sum oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def field5(fss, oracle):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=1)
    return s, a, oracle.rhs_direct(s, a)


@pytest.mark.parametrize("prec", [0, 1])
def test_treecode_n8_theta07(fss, field5, prec):
    s, a, ref = field5
    with fss.Context(method=fss.METHOD_TREECODE, precision=prec, degree=8, theta=0.7) as ctx:
        ctx.set_particles(s, a)
        out = ctx.rhs(s, a)
        info = ctx.tree_info()
    assert info["pc_interactions"] > 0 and info["pp_interactions"] > 0
    err = rel_l2(out[:, :3], ref[:, :3])
    assert err < 1e-6, err


def test_treecode_converges_with_degree(fss, field5):
    s, a, ref = field5
    errs = []
    for n in (2, 4, 6, 8, 10):
        with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, degree=n, theta=0.7) as ctx:
            ctx.set_particles(s, a)
            errs.append(rel_l2(ctx.rhs(s, a)[:, :3], ref[:, :3]))
    assert all(errs[i + 1] < errs[i] for i in range(len(errs) - 1)), errs
    assert errs[-1] < 1e-7, errs


def test_treecode_high_degrees(fss, field5):
    """Degrees 9 and 11 form the moments beyond the 8 x 8 corner in one
    permuted tile, degree 12 (the maximum) in two.  Both must beat degree 9
    by far (a wrong moment costs digits, not a factor); 11 and 12 need not be
    ordered (at theta = 0.7 on this field, 1.5e-9 and 3.0e-9)."""
    s, a, ref = field5
    errs = {}
    for n in (9, 11, 12):
        with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, degree=n, theta=0.7) as ctx:
            ctx.set_particles(s, a)
            errs[n] = rel_l2(ctx.rhs(s, a)[:, :3], ref[:, :3])
    assert errs[9] < 1e-7, errs
    assert max(errs[11], errs[12]) < errs[9] / 4, errs


def test_treecode_theta_tightens(fss, field5):
    s, a, ref = field5
    e = {}
    for th in (0.5, 0.7):
        with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, degree=6, theta=th) as ctx:
            ctx.set_particles(s, a)
            e[th] = rel_l2(ctx.rhs(s, a)[:, :3], ref[:, :3])
    assert e[0.5] < e[0.7], e


def test_treecode_leaf_lists_match_dual(fss, field5):
    """Per-leaf traversal with uniform (n, theta) is as accurate as the dual one."""
    s, a, ref = field5
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, list_mode=fss.LIST_LEAF) as ctx:
        ctx.set_particles(s, a)
        out = ctx.rhs(s, a)
    assert rel_l2(out[:, :3], ref[:, :3]) < 1e-6


def test_treecode_stream_function(fss, oracle, field5):
    s, a, _ = field5
    rows = np.arange(0, s.shape[0], 7)
    ref = oracle.stream_rows(s, a, rows)
    for prec in (fss.PREC_FP64, fss.PREC_MIXED):
        with fss.Context(method=fss.METHOD_TREECODE, precision=prec, degree=8) as ctx:
            ctx.set_particles(s, a)
            _, psi = ctx.rhs(s, a, psi=True)
        assert rel_l2(psi[rows], ref) < 1e-6, prec


def test_treecode_level7_sampled(fss, oracle):
    """C2-size field (163,842 particles) on 2,048 seeded sample targets."""
    s, a = fss.make_state(7, "rh_vortices", n_vortex=8, seed=1)
    rows = np.sort(np.random.default_rng(7).choice(s.shape[0], 2048, replace=False))
    ref = oracle.rhs_direct_rows(s, a, rows)
    for prec in (fss.PREC_FP64, fss.PREC_MIXED):
        with fss.Context(method=fss.METHOD_TREECODE, precision=prec, degree=8, theta=0.7) as ctx:
            ctx.set_particles(s, a)
            out = ctx.rhs(s, a)
        assert rel_l2(out[rows, :3], ref) < 1e-6, prec


def test_autotune_depth_and_split(fss, oracle):
    """autotune = 2: the tree depth (automatic depth and one level either
    side, timed on a whole right-hand side) and the source split are chosen
    by timing; the result stays within the treecode's tolerance, and a later
    fss_set_particles with the same particle count keeps the tuned depth."""
    s, a = fss.make_state(6, "rh_vortices", n_vortex=8, seed=3)
    rows = np.arange(0, s.shape[0], 17)
    ref = oracle.rhs_direct_rows(s, a, rows)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as auto:
        auto.set_particles(s, a)
        base = auto.tree_info()["tree_levels"]
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, autotune=2) as ctx:
        ctx.set_particles(s, a)
        info = ctx.tree_info()
        out = ctx.rhs(s, a)
        ctx.set_particles(s, a)
        again = ctx.tree_info()
    assert abs(info["tree_levels"] - base) <= 1
    assert info["src_parts"] in (1, 2, 4)
    assert again["tree_levels"] == info["tree_levels"]
    assert rel_l2(out[rows, :3], ref) < 1e-6

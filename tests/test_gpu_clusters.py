"""Target clusters (the reference's cp and cc interaction types, fast_rhs.h
cp/cc): a well-separated target face with more than many_count particles
takes its far sources at its interpolation points, and the field there is
interpolated down to its particles.  Checked against the FP64 direct-sum
oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def field6(fss, oracle):
    s, a = fss.make_state(6, "rh_vortices", n_vortex=8, seed=3)
    return s, a, oracle.rhs_direct(s, a)


def _rhs(fss, s, a, **kw):
    with fss.Context(method=fss.METHOD_TREECODE, cluster_targets=1, **kw) as ctx:
        ctx.set_particles(s, a)
        return ctx.rhs(s, a), ctx.tree_info()


@pytest.mark.parametrize("prec", [0, 1])
def test_clusters_accuracy(fss, field6, prec):
    s, a, ref = field6
    out, info = _rhs(fss, s, a, precision=prec, degree=10, theta=0.7, tree_levels=4)
    assert info["target_clusters"] > 0 and info["cc_interactions"] > 0
    err = rel_l2(out[:, :3], ref[:, :3])
    assert err < 2e-6, err
    assert np.allclose(out[:, 3], -2 * fss.OMEGA * out[:, 2], rtol=0, atol=1e-12 * np.abs(out[:, 2]).max())


def test_clusters_converge_with_degree(fss, field6):
    s, a, ref = field6
    errs = []
    for n in (2, 4, 6, 8, 10):
        out, _ = _rhs(fss, s, a, precision=fss.PREC_FP64, degree=n, theta=0.7, tree_levels=4)
        errs.append(rel_l2(out[:, :3], ref[:, :3]))
    assert all(errs[i + 1] < errs[i] for i in range(len(errs) - 1)), errs


def test_clusters_cut_work(fss, field6):
    """Cluster-cluster pairs cost K_t K_s instead of N_t K_s."""
    s, a, _ = field6
    _, on = _rhs(fss, s, a, precision=fss.PREC_MIXED, degree=8, theta=0.7, tree_levels=4)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, degree=8, theta=0.7,
                     tree_levels=4) as ctx:
        ctx.set_particles(s, a)
        off = ctx.tree_info()
    w_on = on["pp_interactions"] + on["pc_interactions"] + on["cp_interactions"] + on["cc_interactions"]
    w_off = off["pp_interactions"] + off["pc_interactions"]
    assert off["target_clusters"] == 0 and w_on < 0.6 * w_off, (w_on, w_off)


def test_clusters_rk4_tracks_direct(fss):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=1)
    out = {}
    for method, prec, ct in ((fss.METHOD_DIRECT, fss.PREC_FP64, 0), (fss.METHOD_TREECODE, fss.PREC_MIXED, 1)):
        with fss.Context(method=method, precision=prec, degree=10, theta=0.7, cluster_targets=ct,
                         tree_levels=4) as ctx:
            ctx.set_particles(s, a)
            ctx.rk4_step(0.01, nsteps=10)
            out[method] = ctx.get_state()
    disp = out[0][:, :3] - s[:, :3]
    err = np.linalg.norm(out[1][:, :3] - out[0][:, :3]) / np.linalg.norm(disp)
    assert err < 5e-6, err


def test_clusters_stream_function(fss, oracle, field6):
    s, a, _ = field6
    rows = np.arange(0, s.shape[0], 97)
    ref = oracle.stream_rows(s, a, rows)
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_FP64, degree=10, theta=0.7, tree_levels=4,
                     cluster_targets=1) as ctx:
        ctx.set_particles(s, a)
        _, psi = ctx.rhs(s, a, psi=True)
    assert rel_l2(psi[rows], ref) < 1e-6

"""Host-side product logic (no GPU): synthetic inputs, tree geometry, the
reference-format traversal and the interpolation node set, all through the
C ABI of libfss.so, checked against the oracle."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def test_library_exports_every_declared_symbol(fss):
    header = open(os.path.join(ROOT, "include", "fss.h")).read()
    declared = sorted(set(re.findall(r"^(?:int|int32_t|int64_t|void|const char\s*\*)\s+(fss_[a-z0-9_]+)\s*\(", header, re.M)))
    assert len(declared) > 20
    L = fss.lib()
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared) == set(fss.SYMBOLS), set(declared) ^ set(fss.SYMBOLS)
    assert "sm_100a" in fss.version()


@pytest.mark.parametrize("level", [0, 2, 4, 6])
def test_icos_grid_matches_oracle(fss, oracle, level):
    xyz, faces = fss.icos_grid(level)
    verts, tv, _ = oracle.icos_init(level, info=False)
    assert np.array_equal(bits(xyz), bits(verts))
    assert np.array_equal(faces, tv[oracle.face_offsets(level)[level]:])


def test_inputs_match_oracle(fss, oracle):
    s, a = fss.make_state(4, "rh4_ref")
    so, ao, _ = oracle.icos_state(4)
    assert np.array_equal(bits(s), bits(so))
    assert np.array_equal(bits(a), bits(ao))


def test_rh_vortices_field(fss):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=1)
    s2, _ = fss.make_state(5, "rh_vortices", n_vortex=8, seed=1)
    s3, _ = fss.make_state(5, "rh_vortices", n_vortex=8, seed=2)
    assert np.array_equal(s, s2) and not np.array_equal(s, s3)
    assert abs((s[:, 3] * a).sum()) < 1e-12          # mean removed
    lat = np.pi / 2 - np.arctan2(np.hypot(s[:, 0], s[:, 1]), s[:, 2])
    assert np.allclose(s[:, 4], 2 + lat)


@pytest.mark.parametrize("tree_levels", [1, 2, 4])
def test_tree_geometry_matches_oracle(fss, oracle, tree_levels):
    ti = fss.tree_geometry(tree_levels)
    _, _, to = oracle.icos_init(tree_levels, info=True)
    assert np.array_equal(bits(ti), bits(to[:ti.shape[0]]))


@pytest.mark.parametrize("level,tree_levels,theta,many", [(4, 3, 0.7, 10), (5, 4, 0.7, 45), (5, 3, 0.5, 10),
                                                          (6, 5, 0.7, 45)])
def test_traversal_bit_exact(fss, oracle, level, tree_levels, theta, many):
    s, _ = fss.make_state(level)
    loc = oracle.points_assign(tree_levels, s)
    counts = oracle.level_counts(loc, tree_levels)
    assert np.array_equal(fss.tree_traverse(tree_levels, theta, many, counts),
                          oracle.tree_traverse(tree_levels, theta, many, counts))


def test_traversal_empty_faces(fss, oracle):
    """Sparse particle sets: faces with no particles are skipped."""
    s, _ = fss.make_state(4)
    s = s[::7]
    loc = oracle.points_assign(3, s)
    counts = oracle.level_counts(loc, 3)
    assert (counts == 0).any()
    assert np.array_equal(fss.tree_traverse(3, 0.7, 10, counts), oracle.tree_traverse(3, 0.7, 10, counts))


@pytest.mark.parametrize("n", [1, 2, 4, 6, 8, 10])
def test_interp_nodes(fss, n):
    nodes, vinv = fss.interp_nodes(n)
    K = (n + 1) * (n + 2) // 2
    assert nodes.shape == (K, 3)
    assert np.allclose(nodes.sum(1), 1.0) and (nodes > -1e-14).all()
    assert len({tuple(np.round(p, 12)) for p in nodes}) == K

    def basis(l1, l2):
        u, v = 2 * l1 - 1, 2 * l2 - 1
        Tu = [np.ones_like(u), u]
        Tv = [np.ones_like(v), v]
        for a in range(2, n + 1):
            Tu.append(2 * u * Tu[-1] - Tu[-2])
            Tv.append(2 * v * Tv[-1] - Tv[-2])
        return np.stack([Tu[g - b] * Tv[b] for g in range(n + 1) for b in range(g + 1)], -1)

    V = basis(nodes[:, 0], nodes[:, 1])
    # the Chebyshev product basis is not orthogonal on the triangle: its
    # Vandermonde matrix has cond ~3e7 at n = 10, so the inverse is exact to
    # ~cond * eps
    assert np.abs(V @ vinv - np.eye(K)).max() < 1e-15 * K * np.linalg.cond(V)
    # Lagrange property and a modest Lebesgue constant on a fine grid
    t = np.linspace(0, 1, 61)
    l1, l2 = np.meshgrid(t, t)
    m = (l1 + l2) <= 1
    L = basis(l1[m], l2[m]) @ vinv
    assert np.allclose(L.sum(1), 1.0, atol=1e-7)
    leb = np.abs(L).sum(1).max()
    assert leb < {1: 1.01, 2: 1.7, 4: 3.5, 6: 6.0, 8: 10.0, 10: 20.0}[n], leb


def test_interpolation_reproduces_polynomials(fss):
    """q_k = sum_j w_j l_k(b_j) reproduces the moments of any degree <= n
    polynomial exactly: sum_k q_k p(node_k) = sum_j w_j p(b_j)."""
    n = 8
    nodes, vinv = fss.interp_nodes(n)
    rng = np.random.default_rng(0)
    b = rng.dirichlet([1, 1, 1], size=200)
    w = rng.standard_normal(200)

    def basis(l1, l2):
        u, v = 2 * l1 - 1, 2 * l2 - 1
        Tu = [np.ones_like(u), u]
        Tv = [np.ones_like(v), v]
        for a in range(2, n + 1):
            Tu.append(2 * u * Tu[-1] - Tu[-2])
            Tv.append(2 * v * Tv[-1] - Tv[-2])
        return np.stack([Tu[g - b_] * Tv[b_] for g in range(n + 1) for b_ in range(g + 1)], -1)

    q = (basis(b[:, 0], b[:, 1]) @ vinv).T @ w
    p = lambda l1, l2: l1 ** 3 * l2 ** 2 - 2 * l1 * l2 ** 5 + l2 - 0.5
    assert abs(q @ p(nodes[:, 0], nodes[:, 1]) - w @ p(b[:, 0], b[:, 1])) < 1e-9


def test_context_needs_gpu_or_reports(fss):
    """Without a GPU the library refuses loudly (no CPU fallback)."""
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("GPU present")
    with pytest.raises(fss.FssError) as e:
        fss.Context()
    assert e.value.code == 7
    # settings are validated on the host first
    with pytest.raises(fss.FssError) as e:
        fss.Context(wait_limit_us=-1)
    assert e.value.code == 1


def test_amr_and_remesh_need_gpu_or_report(fss):
    """The AMR handle and the remesh step refuse loudly without a GPU, after
    validating their arguments on the host."""
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("GPU present")
    xyz, tris = fss.icos_grid(2)
    with pytest.raises(fss.FssError) as e:
        fss.Amr(tris, xyz.shape[0], 4 * xyz.shape[0], 4 * tris.shape[0])
    assert e.value.code == 7
    bad = tris.copy()
    bad[0, 0] = xyz.shape[0]
    with pytest.raises(fss.FssError) as e:
        fss.Amr(bad, xyz.shape[0], 4 * xyz.shape[0], 4 * tris.shape[0])
    assert e.value.code == 1  # checked before any device call
    with pytest.raises(fss.FssError) as e:
        fss.Amr(tris, xyz.shape[0], xyz.shape[0] - 1, 4 * tris.shape[0])
    assert e.value.code == 1
    s = np.zeros((xyz.shape[0], 5))
    s[:, :3] = xyz
    with pytest.raises(fss.FssError):
        fss.remesh(s, s, tris)

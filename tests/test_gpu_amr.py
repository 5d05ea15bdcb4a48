"""AMR (amr.h:13-178 amr) on the GPU against the oracle, which is pinned bit
for bit to the reference's own amr() (tests/test_oracle_pins.py): points,
triangles, parent pairs and the vert_tris order (corner keys) exactly;
areas within 1e-13 relative (the spherical-triangle area goes through
CUDA's acos/tan/atan, which may differ from the host's libm in the last
bit); then regrid_points2 on the refined mesh."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gauss_state(fss, level):
    s, area = fss.make_state(level, "gauss_ref")
    return s, area, fss.icos_grid(level)[1]


def check(M, st, ar, amr):
    tris, keys, par = amr.mesh()
    assert (st.shape[0], tris.shape[0]) == (M["n"], M["ntri"])
    assert np.array_equal(st.view(np.uint64), M["state5"].view(np.uint64))
    assert np.array_equal(tris, M["tris"]) and np.array_equal(keys, M["keys"]) and np.array_equal(par, M["parent"])
    np.testing.assert_allclose(ar, M["area"], rtol=1e-13, atol=0)


def test_amr_golden_case(fss, oracle):
    g = np.load(os.path.join(GOLD, "amr_l2.npz"))
    mc = int(g["max_count"])
    M = oracle.amr(g["state"], g["area"], g["faces"], mc, 4 * mc)
    with fss.Amr(g["faces"], g["state"].shape[0], mc, 4 * mc) as amr:
        st, ar = amr.refine(g["state"], g["area"])
        check(M, st, ar, amr)
        assert np.array_equal(st.view(np.uint64), g["out_state"].view(np.uint64))
        out, fb, bad = amr.remesh(g["remesh_moved"], g["remesh_target"])
        assert bad == 0 and np.array_equal(out.view(np.uint64), g["remesh_out"].view(np.uint64))


@pytest.mark.parametrize("level", [3, 4])
def test_amr_gauss_vortex_two_calls(fss, oracle, level):
    """The full vortex at the reference's tolerances, then a second call on
    the refined mesh (vortex 10% stronger, positions projected) that must
    reuse the midpoints of the first."""
    s, a, tris = gauss_state(fss, level)
    mc = 10 * 4 ** (level + 3) + 2
    mt = 4 * mc
    M = oracle.amr(s, a, tris, mc, mt)
    with fss.Amr(tris, s.shape[0], mc, mt) as amr:
        st, ar = amr.refine(s, a)
        check(M, st, ar, amr)
        assert M["n"] > 3 * s.shape[0]
        s2 = M["state5"].copy()
        s2[:, :3] /= np.linalg.norm(s2[:, :3], axis=1, keepdims=True)
        s2[:, 3] *= 1.1
        M2 = oracle.amr(s2, M["area"], M["tris"], mc, mt, parent=M["parent"], keys=M["keys"], seq=M["seq"])
        st2, ar2 = amr.refine(s2, M["area"])
        assert M2["rc"] == 0 and M2["n"] > M["n"]
        check(M2, st2, ar2, amr)


def test_amr_remesh_matches_oracle(fss, oracle):
    s, a, tris = gauss_state(fss, 4)
    mc = 10 * 4 ** 7 + 2
    with fss.Amr(tris, s.shape[0], mc, 4 * mc) as amr:
        st, _ = amr.refine(s, a)
        t, keys, _ = amr.mesh()
        grid = st.copy()
        grid[:, :3] /= np.linalg.norm(grid[:, :3], axis=1, keepdims=True)
        c, sn = np.cos(0.005), np.sin(0.005)
        moved = grid.copy()
        moved[:, :3] = grid[:, :3] @ np.array([[c, -sn, 0], [sn, c, 0], [0, 0, 1]]).T
        ref, fb_ref, bad_ref = oracle.remesh(moved, grid, t, keys=keys)
        got, fb, bad = amr.remesh(moved, grid)
        assert (fb, bad) == (fb_ref, bad_ref) and fb > 1000
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


def test_amr_limits(fss):
    s, a, tris = gauss_state(fss, 3)
    # at max_count already: nothing happens (the reference's entry test)
    with fss.Amr(tris, s.shape[0], s.shape[0], 4 * tris.shape[0]) as amr:
        st, ar = amr.refine(s, a)
        assert st.shape[0] == s.shape[0] and np.array_equal(ar, a)
    # too few triangle slots: FSS_ERR_CAPACITY, then the handle refuses
    with fss.Amr(tris, s.shape[0], 10 * s.shape[0], tris.shape[0] + 30) as amr:
        with pytest.raises(fss.FssError):
            amr.refine(s, a)
        with pytest.raises(fss.FssError):
            amr.refine(s, a)


def test_amr_refine_current_matches_host_path(fss, oracle):
    """The device-resident AMR step (new_dynamics.cpp:219-228: amr, then the
    new points projected, then the new particle set) gives the context the
    same state as the host path: refine on host arrays, project the new
    points (oracle project_points), set_particles."""
    s, a, tris = gauss_state(fss, 4)
    mc = 10 * 4 ** 7 + 2
    with fss.Amr(tris, s.shape[0], mc, 4 * mc) as amr:
        st, ar = amr.refine(s, a)
    proj = st.copy()
    tail = np.ascontiguousarray(proj[s.shape[0]:])
    oracle.lib().orc_project_points(tail.shape[0], tail.reshape(-1), oracle.OMEGA)
    proj[s.shape[0]:] = tail
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(proj, ar)
        want = ctx.get_state()
    with fss.Amr(tris, s.shape[0], mc, 4 * mc) as amr, \
            fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        n = ctx.amr_refine_current(amr)
        assert n == st.shape[0] > s.shape[0]
        got = ctx.get_state()
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        ctx.rk4_step(0.01, nsteps=2)  # the context steps on with the new set
        assert np.all(np.isfinite(ctx.get_state()))
    # a context whose particles are not the mesh's points is refused
    with fss.Amr(tris, s.shape[0], mc, 4 * mc) as amr, \
            fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(proj, ar)
        with pytest.raises(fss.FssError):
            ctx.amr_refine_current(amr)

"""State files and input files in the reference's formats
(new_dynamics.cpp:123-139, 228-236; helpers.h:299-340 read_points)."""
import os

import numpy as np
import pytest

from test_oracle_pins import need_ref


def awkward_state(n=400, seed=4):
    rng = np.random.default_rng(seed)
    s = rng.standard_normal((n, 5)) * 10.0 ** rng.integers(-12, 12, (n, 5))
    s[:5] = [[0.0, -0.0, 1.0, -1.0, 123456.0], [1e-5, 1e-4, 999999.5, 1e16, -2.5e-300],
             [np.nan, -np.inf, np.inf, 0.1, 1 / 3], [7.0, 70.0, 700000.0, 7e6, 1e-310],
             [-np.nan, 2 ** 53, 0.5, 1.5, 2.5]]
    a = np.abs(rng.standard_normal(n)) * 1e-3
    return s, a


def g6(v):
    """C's %g (Python's drops the sign of a NaN; C prints -nan)."""
    return ("-nan" if np.signbit(v) else "nan") if np.isnan(v) else "%g" % v


def test_state_csv_is_printf_g(fss, tmp_path):
    """Each line: the six numbers as %g (6 significant digits), comma-separated."""
    s, a = awkward_state()
    p = tmp_path / "out.csv"
    fss.state_csv_append(p, s, a)
    fss.state_csv_append(p, s[:7], a[:7])  # a second step appends
    want = "".join(",".join(g6(v) for v in (*s[i], a[i])) + "\n" for i in range(len(a)))
    want += "".join(",".join(g6(v) for v in (*s[i], a[i])) + "\n" for i in range(7))
    assert p.read_text() == want


@need_ref
def test_state_csv_matches_reference_bytes(fss, oracle, tmp_path):
    s, a = awkward_state(2000, seed=9)
    fss.state_csv_append(tmp_path / "ours.csv", s, a)
    assert oracle.ref_write_state(tmp_path / "ref.csv", s, a) == 0
    assert (tmp_path / "ours.csv").read_bytes() == (tmp_path / "ref.csv").read_bytes()


def test_output_names_and_point_counts(fss, tmp_path):
    assert fss.output_name(10242, "rh4", True, 4, time_steps=100) == "10242_rh4_fast_4_100"
    assert fss.output_name(2562, "gv", False, use_amr=True, use_mpi=True, use_remesh=True, time_steps=3) == \
        "2562_gv_direct_amr_mpi_remesh_3"
    p = tmp_path / "point_counts.csv"
    for n in (2562, 2600, 2733):
        fss.point_count_append(p, n)
    assert p.read_text() == "2562\n2600\n2733\n"


def test_state_bin_round_trip(fss, tmp_path):
    p = tmp_path / "out.bin"
    steps = [awkward_state(n, seed=n) for n in (10, 300, 7)]
    for s, a in steps:
        fss.state_bin_append(p, s, a)
    assert p.stat().st_size == sum(16 + 48 * len(a) for _, a in steps)
    for k, (s, a) in enumerate(steps):
        s2, a2 = fss.state_bin_read(p, k)
        assert np.array_equal(s2.view(np.uint64), s.view(np.uint64))
        assert np.array_equal(a2.view(np.uint64), a.view(np.uint64))
    with pytest.raises(fss.FssError):
        fss.state_bin_read(p, 3)


def write_reference_inputs(fss, d, level, seed=5):
    """The reference's four input files for the level-`level` grid, each
    vertex's triangle list in a shuffled order."""
    s, _ = fss.make_state(level, "rh4_ref")
    _, tris = fss.icos_grid(level)
    n = s.shape[0]
    with open(os.path.join(d, f"{n}points_rh4.csv"), "w") as f:
        for r in s:
            f.write(",".join(repr(float(v)) for v in r) + "\n")
    with open(os.path.join(d, f"{n}tris.csv"), "w") as f:
        for t in tris:
            f.write(f"{t[0]},{t[1]},{t[2]}\n")
    lists = [[] for _ in range(n)]
    for j, t in enumerate(tris):
        for v in t:
            lists[v].append(j)
    rng = np.random.default_rng(seed)
    lists = [list(rng.permutation(l)) for l in lists]
    with open(os.path.join(d, f"{n}vert_tris.csv"), "w") as f:
        for l in lists:
            f.write(",".join(str(x) for x in l) + "\n")
    with open(os.path.join(d, f"{n}vert_tri_count.csv"), "w") as f:
        for l in lists:
            f.write(f"{len(l)}\n")
    return s, tris, lists


def test_readers_parse_reference_inputs(fss, tmp_path):
    s, tris, lists = write_reference_inputs(fss, tmp_path, 3)
    n = s.shape[0]
    got = fss.read_points_csv(tmp_path / f"{n}points_rh4.csv", n)
    assert np.array_equal(got[:, :4], s[:, :4]) and not got[:, 4].any()  # the tracer is not read
    assert np.array_equal(fss.read_tris_csv(tmp_path / f"{n}tris.csv", tris.shape[0]), tris)
    off, adj = fss.read_vert_tris_csv(tmp_path / f"{n}vert_tris.csv", tmp_path / f"{n}vert_tri_count.csv", n,
                                      3 * tris.shape[0])
    assert all(list(adj[off[i]:off[i + 1]]) == lists[i] for i in range(n))


@need_ref
def test_readers_match_reference_read_points(fss, oracle, tmp_path):
    s, tris, lists = write_reference_inputs(fss, tmp_path, 3)
    n, ntri = s.shape[0], tris.shape[0]
    (tmp_path / "run").mkdir()
    rs, rt, roff, radj = oracle.ref_read_points(tmp_path / "run", n, ntri, 3 * ntri)
    got = fss.read_points_csv(tmp_path / f"{n}points_rh4.csv", n)
    assert np.array_equal(got.view(np.uint64), rs.view(np.uint64))
    assert np.array_equal(fss.read_tris_csv(tmp_path / f"{n}tris.csv", ntri), rt)
    off, adj = fss.read_vert_tris_csv(tmp_path / f"{n}vert_tris.csv", tmp_path / f"{n}vert_tri_count.csv", n,
                                      3 * ntri)
    assert np.array_equal(off, roff) and np.array_equal(adj, radj)


def list_keys(tris, off, adj):
    """Corner keys that order each vertex's triangles as its list does."""
    keys = np.zeros(tris.shape, dtype=np.uint64)
    for v in range(len(off) - 1):
        for p, t in enumerate(adj[off[v]:off[v + 1]]):
            keys[t][list(tris[t]).index(v)] = p
    return keys


@need_ref
def test_oracle_list_order_matches_reference(fss, oracle, tmp_path):
    """The oracle's list-ordered regrid equals regrid_points2 given the same
    (shuffled) vert_tris lists."""
    s, tris, lists = write_reference_inputs(fss, tmp_path, 4)
    off = np.concatenate([[0], np.cumsum([len(l) for l in lists])]).astype(np.int32)
    adj = np.concatenate(lists).astype(np.int32)
    m = s.copy()
    h = np.sqrt(4 * np.pi / s.shape[0])
    m[:, :3] += 0.4 * h * np.random.default_rng(2).standard_normal((s.shape[0], 3))
    m[:, :3] /= np.linalg.norm(m[:, :3], axis=1, keepdims=True)
    ref, rc = oracle.ref_remesh_lists(m, s, tris, [adj[off[i]:off[i + 1]] for i in range(s.shape[0])])
    got, fb, bad = oracle.remesh(m, s, tris, keys=list_keys(tris, off, adj))
    assert rc == 0 and bad == 0 and fb > 0
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))

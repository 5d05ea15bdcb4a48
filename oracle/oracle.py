"""TEST INFRASTRUCTURE ONLY -- numpy/ctypes front end of the oracle.

Loads ``liboracle.so`` (the C restatement in ``fss_oracle.c``) and, when it
was built here, ``_ref/libref.so`` (the reference's own headers compiled in
place, see ``Makefile``).  Only ``tests/``, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` import this module; the product never does.
"""
import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_L = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
i64 = C.c_int64


def _load(path):
    if not os.path.exists(path):
        return None
    return C.CDLL(path)


def build():
    """Compile liboracle.so (and _ref/libref.so when the reference is here)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = _load(os.path.join(HERE, "liboracle.so"))
_ref = _load(os.path.join(HERE, "_ref", "libref.so"))


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = _load(os.path.join(HERE, "liboracle.so"))
        _setup(_lib)
    return _lib


def ref():
    """The reference library, or None when it was not built."""
    return _ref


def _setup(L):
    if L is None:
        return
    L.orc_icos_counts.argtypes = [C.c_int, C.POINTER(i64), C.POINTER(i64)]
    L.orc_icos_init.argtypes = [C.c_int, C.c_double, _D, _I, C.c_void_p]
    L.orc_icos_init.restype = i64
    L.orc_area_init.argtypes = [i64, _D, i64, _I, _D]
    L.orc_rossby_haurwitz_4.argtypes = [i64, _D]
    L.orc_rh_vortices.argtypes = [i64, _D, C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_uint64]
    L.orc_mt64_draws.argtypes = [C.c_uint64, i64, np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")]
    L.orc_rhs_direct.argtypes = [i64, _D, _D, C.c_double, _D, C.c_int]
    L.orc_rhs_direct_rows.argtypes = [i64, _D, _D, i64, C.c_void_p, _D, C.c_int]
    L.orc_stream_rows.argtypes = [i64, _D, _D, i64, C.c_void_p, _D]
    L.orc_project_points.argtypes = [i64, _D, C.c_double]
    L.orc_rk4_step.argtypes = [i64, _D, _D, C.c_double, C.c_double, C.c_int]
    L.orc_points_assign.argtypes = [C.c_int, _D, _I, i64, _D, _I]
    L.orc_tree_traverse.argtypes = [C.c_int, C.c_double, C.c_int, _I, _D, C.c_double, _I, i64]
    L.orc_tree_traverse.restype = i64
    L.orc_barycoords.argtypes = [_D, _D, _D, _D, _D]
    L.orc_remesh.argtypes = [i64, _D, _D, i64, _I, C.c_double, C.POINTER(i64)]
    L.orc_remesh.restype = i64
    _U = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
    L.orc_remesh_keyed.argtypes = [i64, _D, _D, i64, _I, C.c_void_p, C.c_double, C.POINTER(i64)]
    L.orc_remesh_keyed.restype = i64
    L.orc_amr.argtypes = [C.POINTER(i64), i64, _D, _D, C.POINTER(i64), i64, _I, _U, _I, C.POINTER(C.c_uint64),
                          C.c_double, C.c_double]
    L.orc_amr.restype = C.c_int


def _setup_ref(R):
    if R is None:
        return
    R.ref_icos_init.argtypes = [C.c_int, C.c_double, _D, _I, C.c_void_p]
    R.ref_icos_init.restype = i64
    R.ref_area_init.argtypes = [i64, _D, i64, _I, _D]
    R.ref_rossby_haurwitz_4.argtypes = [i64, _D]
    R.ref_gauss_vortex.argtypes = [i64, _D, _D]
    R.ref_rhs_func_direct.argtypes = [i64, _D, _D, C.c_double, _D]
    R.ref_rhs_direct_rows.argtypes = [i64, _D, _D, i64, C.c_void_p, _D, C.c_int]
    R.ref_project_points.argtypes = [i64, _D, C.c_double]
    R.ref_rk4_step.argtypes = [i64, _D, _D, C.c_double, C.c_double]
    R.ref_tree.argtypes = [C.c_int, C.c_double, C.c_int, i64, _D, _I, _I, _I, i64]
    R.ref_tree.restype = i64
    R.ref_tree_members.argtypes = [C.c_int, i64, _D, C.c_int, C.c_int, _I, i64]
    R.ref_tree_members.restype = i64
    R.ref_rhs_fast.argtypes = [i64, _D, _D, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, _D]
    R.ref_rhs_fast.restype = C.c_int
    R.ref_rhs_fast_timed.argtypes = [i64, _D, _D, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _D,
                                     C.c_void_p, _D]
    R.ref_rhs_fast_timed.restype = C.c_int
    R.ref_regrid.argtypes = [i64, _D, _D, i64, _I, C.c_double]
    R.ref_regrid.restype = C.c_int
    R.ref_regrid_range.argtypes = [i64, _D, _D, i64, _I, C.c_double, i64, i64]
    R.ref_regrid_range.restype = C.c_int
    R.ref_amr.argtypes = [i64, i64, i64, _D, _D, _I, C.c_void_p, i64, i64, C.POINTER(i64), C.POINTER(i64), _D, _D, _I,
                          _I, _I, _I]
    R.ref_amr.restype = C.c_int
    R.ref_regrid_csr.argtypes = [i64, _D, _D, i64, _I, _I, _I, C.c_double]
    R.ref_regrid_csr.restype = C.c_int
    R.ref_read_points.argtypes = [C.c_char_p, i64, i64, _D, _I, _I, _I, i64]
    R.ref_read_points.restype = C.c_int


_setup(_lib)
_setup_ref(_ref)

OMEGA = 2.0 * np.pi


def icos_counts(levels):
    v, f = i64(), i64()
    lib().orc_icos_counts(levels, C.byref(v), C.byref(f))
    return v.value, f.value


def face_offsets(levels):
    """Start of each level's faces in the concatenated face arrays."""
    off, o, nf = [], 0, 20
    for _ in range(levels + 1):
        off.append(o)
        o += nf
        nf *= 4
    return off


def icos_init(levels, radius=1.0, info=True, use_ref=False):
    """(verts[V,3], tri_verts[F,3], tri_info[F,4] or None), levels concatenated."""
    V, F = icos_counts(levels)
    verts = np.zeros((V, 3))
    tv = np.zeros((F, 3), dtype=np.int32)
    ti = np.zeros((F, 4)) if info else None
    L = ref() if use_ref else lib()
    fn = L.ref_icos_init if use_ref else L.orc_icos_init
    nv = fn(levels, radius, verts.reshape(-1), tv.reshape(-1),
            ti.ctypes.data_as(C.c_void_p) if info else None)
    assert nv == V
    return verts, tv, ti


def icos_state(level, use_ref=False):
    """Particles = level-`level` icosahedral vertices in icos_init order, the
    level's faces, areas (area_init) and reference RH4 vorticity/tracer."""
    verts, tv, _ = icos_init(level, info=False, use_ref=use_ref)
    n = verts.shape[0]
    tris = np.ascontiguousarray(tv[face_offsets(level)[level]:])
    s = np.zeros((n, 5))
    s[:, :3] = verts
    area = np.zeros(n)
    L = ref() if use_ref else lib()
    (L.ref_area_init if use_ref else L.orc_area_init)(n, s.reshape(-1), tris.shape[0], tris.reshape(-1), area)
    (L.ref_rossby_haurwitz_4 if use_ref else L.orc_rossby_haurwitz_4)(n, s.reshape(-1))
    return s, area, tris


RH_AMP = 7.848e-6 * 86400.0  # w = K of the benchmark's Rossby-Haurwitz wave, per day


def mt64_draws(seed, count):
    """First `count` outputs of MT19937-64 seeded with `seed`."""
    out = np.zeros(count, dtype=np.uint64)
    lib().orc_mt64_draws(seed, count, out)
    return out


def rh_vortices(state5, area, n_vortex, seed, amp=RH_AMP, width=0.1):
    """The benchmark's seeded RH R=4 wave + Gaussian vortices on the
    positions of state5 (zeta and tracer overwritten; returns a copy)."""
    s = np.array(state5, dtype=np.float64)
    a = np.ascontiguousarray(area, dtype=np.float64)
    lib().orc_rh_vortices(s.shape[0], s.reshape(-1), a.ctypes.data_as(C.c_void_p), amp, n_vortex, width, seed)
    return s


def rh_vortices_state(level, n_vortex, seed, amp=RH_AMP, width=0.1):
    """(state5, area) of the benchmark field on the level-`level`
    icosahedral grid, built by the oracle alone (icos_init, area_init and the
    field restated above), without the product library."""
    s, area, _ = icos_state(level)
    return rh_vortices(s, area, n_vortex, seed, amp, width), area


def rhs_direct(state5, area, omega=OMEGA, threads=None, use_ref=False):
    s = np.ascontiguousarray(state5, dtype=np.float64).reshape(-1)
    n = s.size // 5
    out = np.zeros(5 * n)
    a = np.ascontiguousarray(area, dtype=np.float64)
    if use_ref:
        ref().ref_rhs_func_direct(n, s, a, omega, out)
    else:
        lib().orc_rhs_direct(n, s, a, omega, out, threads or os.cpu_count())
    return out.reshape(n, 5)


def rhs_direct_rows(state5, area, rows, threads=None, use_ref=False):
    s = np.ascontiguousarray(state5, dtype=np.float64).reshape(-1)
    n = s.size // 5
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.zeros(3 * rows.size)
    a = np.ascontiguousarray(area, dtype=np.float64)
    fn = ref().ref_rhs_direct_rows if use_ref else lib().orc_rhs_direct_rows
    fn(n, s, a, rows.size, rows.ctypes.data_as(C.c_void_p), out, threads or os.cpu_count())
    return out.reshape(-1, 3)


def stream_rows(state5, area, rows):
    s = np.ascontiguousarray(state5, dtype=np.float64).reshape(-1)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.zeros(rows.size)
    lib().orc_stream_rows(s.size // 5, s, np.ascontiguousarray(area, dtype=np.float64), rows.size,
                          rows.ctypes.data_as(C.c_void_p), out)
    return out


def rk4_step(state5, area, dt, omega=OMEGA, threads=None, use_ref=False):
    s = np.array(state5, dtype=np.float64).reshape(-1)
    a = np.ascontiguousarray(area, dtype=np.float64)
    if use_ref:
        ref().ref_rk4_step(s.size // 5, s, a, omega, dt)
    else:
        lib().orc_rk4_step(s.size // 5, s, a, omega, dt, threads or os.cpu_count())
    return s.reshape(-1, 5)


def points_assign(tree_levels, state5):
    """loc[tree_levels, N]: face per level or -1 (oracle restatement)."""
    verts, tv, _ = icos_init(tree_levels, info=False)
    s = np.ascontiguousarray(state5, dtype=np.float64).reshape(-1)
    n = s.size // 5
    loc = np.zeros(tree_levels * n, dtype=np.int32)
    lib().orc_points_assign(tree_levels, verts.reshape(-1), tv.reshape(-1), n, s, loc)
    return loc.reshape(tree_levels, n)


def level_counts(loc, tree_levels):
    off = face_offsets(tree_levels)
    counts = np.zeros(off[tree_levels], dtype=np.int32)
    for l in range(tree_levels):
        v = loc[l][loc[l] >= 0]
        counts[off[l]:off[l] + 20 * 4 ** l] = np.bincount(v, minlength=20 * 4 ** l)
    return counts


def tree_traverse(tree_levels, theta, many_count, counts):
    _, _, ti = icos_init(tree_levels, info=True)
    counts = np.ascontiguousarray(counts, dtype=np.int32)
    cap = 1 << 16
    while True:
        out = np.zeros(7 * cap, dtype=np.int32)
        n = lib().orc_tree_traverse(tree_levels, theta, many_count, counts, ti.reshape(-1), 1.0, out, cap)
        if n >= 0:
            return out[:7 * n].reshape(n, 7)
        cap = -n


def ref_tree(tree_levels, theta, many_count, state5):
    """The reference's (loc, counts, pairs) for a state, via libref.so."""
    s = np.ascontiguousarray(state5, dtype=np.float64).reshape(-1)
    n = s.size // 5
    loc = np.zeros(tree_levels * n, dtype=np.int32)
    counts = np.zeros(face_offsets(tree_levels)[tree_levels], dtype=np.int32)
    cap = 1 << 16
    while True:
        pairs = np.zeros(7 * cap, dtype=np.int32)
        np_ = ref().ref_tree(tree_levels, theta, many_count, n, s, loc, counts, pairs, cap)
        if np_ >= 0:
            return loc.reshape(tree_levels, n), counts, pairs[:7 * np_].reshape(np_, 7)
        cap = -np_


def remesh(moved5, target5, tris, omega=OMEGA, use_ref=False, rows=None, keys=None):
    """remesh.h regrid_points2: (new target state, fallback count, not-found
    count); adjacency in increasing triangle order.  With use_ref, `rows` =
    (lb, ub) regrids only those targets (the reference's lb/ub)."""
    m = np.ascontiguousarray(moved5, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(target5, dtype=np.float64).copy().reshape(-1)
    tr = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    n, ntri = m.size // 5, tr.size // 3
    if use_ref:
        lb, ub = rows if rows is not None else (0, n)
        rc = ref().ref_regrid_range(n, m, t, ntri, tr, omega, lb, ub)
        return t.reshape(n, 5), None, (0 if rc == 0 else -1)
    fb = C.c_int64()
    if keys is not None:
        k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1)
        bad = lib().orc_remesh_keyed(n, m, t, ntri, tr, k.ctypes.data_as(C.c_void_p), omega, C.byref(fb))
    else:
        bad = lib().orc_remesh(n, m, t, ntri, tr, omega, C.byref(fb))
    return t.reshape(n, 5), fb.value, bad


AMR_VTOL, AMR_CTOL = 0.2, 0.0025  # amr.h:14-15


def amr(state5, area, tris, max_points, max_tris, parent=None, keys=None, seq=0, vtol=AMR_VTOL, ctol=AMR_CTOL):
    """amr.h amr (oracle restatement): dict of n, ntri, state5, area, tris,
    keys (adjacency order per corner), parent, seq, rc."""
    n, ntri = state5.shape[0], tris.shape[0]
    st = np.zeros((max_points, 5)); st[:n] = state5
    ar = np.zeros(max_points); ar[:n] = area
    tr = np.zeros((max_tris, 3), dtype=np.int32); tr[:ntri] = tris
    ky = np.zeros((max_tris, 3), dtype=np.uint64)
    ky[:ntri] = np.arange(ntri, dtype=np.uint64)[:, None] if keys is None else keys
    pa = np.zeros((max_points, 2), dtype=np.int32)
    if parent is not None:
        pa[:n] = parent
    nn, nt, sq = i64(n), i64(ntri), C.c_uint64(seq)
    rc = lib().orc_amr(C.byref(nn), max_points, st.reshape(-1), ar, C.byref(nt), max_tris, tr.reshape(-1),
                       ky.reshape(-1), pa.reshape(-1), C.byref(sq), vtol, ctol)
    n, ntri = nn.value, nt.value
    return dict(n=n, ntri=ntri, state5=st[:n], area=ar[:n], tris=tr[:ntri], keys=ky[:ntri], parent=pa[:n],
                seq=sq.value, rc=rc)


def vert_tris(n, tris, keys=None):
    """Each vertex's triangles in adjacency order (by corner key, else by index)."""
    tris = np.asarray(tris)
    corners = np.arange(tris.size)
    order = np.lexsort((corners if keys is None else np.asarray(keys, dtype=np.uint64).reshape(-1),
                        tris.reshape(-1)))
    v = tris.reshape(-1)[order]
    cut = np.searchsorted(v, np.arange(n + 1))
    t = order // 3
    return [t[cut[i]:cut[i + 1]] for i in range(n)]


def ref_amr(state5, area, tris, max_count, parent=None, cap_points=None, cap_tris=None):
    """The reference's own amr() (oracle/_ref): dict of n, ntri, state5, area,
    tris, parent, vert_tris (list of arrays)."""
    n, ntri = state5.shape[0], tris.shape[0]
    cap_points = cap_points or max_count
    cap_tris = cap_tris or 4 * max_count
    st = np.zeros((cap_points, 5)); ar = np.zeros(cap_points)
    tr = np.zeros((cap_tris, 3), dtype=np.int32); pa = np.zeros((cap_points, 2), dtype=np.int32)
    off = np.zeros(cap_points + 1, dtype=np.int32); adj = np.zeros(3 * cap_tris, dtype=np.int32)
    pin = None if parent is None else np.ascontiguousarray(parent, dtype=np.int32)
    nn, nt = i64(), i64()
    rc = ref().ref_amr(n, max_count, ntri, np.ascontiguousarray(state5, dtype=np.float64).reshape(-1),
                       np.ascontiguousarray(area, dtype=np.float64), np.ascontiguousarray(tris, dtype=np.int32).reshape(-1),
                       None if pin is None else pin.ctypes.data_as(C.c_void_p), cap_points, cap_tris,
                       C.byref(nn), C.byref(nt), st.reshape(-1), ar, tr.reshape(-1), pa.reshape(-1), off, adj)
    assert rc == 0, "output capacity"
    n, ntri = nn.value, nt.value
    return dict(n=n, ntri=ntri, state5=st[:n], area=ar[:n], tris=tr[:ntri], parent=pa[:n],
                vert_tris=[adj[off[i]:off[i + 1]] for i in range(n)])


def ref_remesh_lists(moved5, target5, tris, vert_tris, omega=OMEGA):
    """The reference's regrid_points2 with explicit vert_tris lists."""
    m = np.ascontiguousarray(moved5, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(target5, dtype=np.float64).copy().reshape(-1)
    tr = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    off = np.zeros(len(vert_tris) + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(v) for v in vert_tris])
    adj = np.ascontiguousarray(np.concatenate(vert_tris) if len(vert_tris) else np.zeros(0), dtype=np.int32)
    rc = ref().ref_regrid_csr(m.size // 5, m, t, tr.size // 3, tr, off, adj, omega)
    return t.reshape(-1, 5), rc


def ref_write_state(path, state5, area):
    """The reference's per-step state lines appended to `path`, written by
    oracle/_ref/ref_write_state (its stream statement restated in a small
    program of its own); None when that program was not built."""
    import subprocess, tempfile
    exe = os.path.join(HERE, "_ref", "ref_write_state")
    if not os.path.exists(exe):
        return None
    s = np.ascontiguousarray(state5, dtype=np.float64).reshape(-1, 5)
    rows = np.concatenate([s, np.ascontiguousarray(area, dtype=np.float64)[:, None]], axis=1)
    with tempfile.NamedTemporaryFile(suffix=".f64", delete=False) as f:
        f.write(np.ascontiguousarray(rows).tobytes())
        raw = f.name
    try:
        return subprocess.run([exe, raw, str(path)], check=False).returncode
    finally:
        os.unlink(raw)


def ref_read_points(run_dir, n, ntri, cap):
    """The reference's read_points run from `run_dir`: (state5, tris, off, adj)."""
    s = np.zeros((n, 5))
    t = np.zeros((ntri, 3), dtype=np.int32)
    off = np.zeros(n + 1, dtype=np.int32)
    adj = np.zeros(cap, dtype=np.int32)
    rc = ref().ref_read_points(str(run_dir).encode(), n, ntri, s.reshape(-1), t.reshape(-1), off, adj, cap)
    assert rc == 0, rc
    return s, t, off, adj[:off[-1]].copy()

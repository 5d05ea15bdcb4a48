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
    R.ref_regrid.argtypes = [i64, _D, _D, i64, _I, C.c_double]
    R.ref_regrid.restype = C.c_int
    R.ref_regrid_range.argtypes = [i64, _D, _D, i64, _I, C.c_double, i64, i64]
    R.ref_regrid_range.restype = C.c_int


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


def remesh(moved5, target5, tris, omega=OMEGA, use_ref=False, rows=None):
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
    bad = lib().orc_remesh(n, m, t, ntri, tr, omega, C.byref(fb))
    return t.reshape(n, 5), fb.value, bad

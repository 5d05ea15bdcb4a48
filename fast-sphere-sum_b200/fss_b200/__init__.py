"""fss_b200 -- ctypes front end of ``libfss.so`` (the C ABI in include/fss.h).

The product path is the CUDA library; this module only marshals numpy
arrays.  There is no CPU fallback: if ``libfss.so`` is missing or has no GPU,
the calls raise.

Mirrors the reference's interface (cygnari/fast-sphere-sum,
Old-BVE-code/rhs_eval.h:47 ``rhs_func(modify, curr_state, area, omega,
config1)``): state arrays are (N, 5) float64 ``[x, y, z, zeta, tracer]`` and
``rhs`` returns ``modify`` in the same layout.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfss.so")
CSRC = os.path.join(os.path.dirname(HERE), "csrc")

OMEGA = 2.0 * np.pi
PREC_FP64, PREC_MIXED = 0, 1
METHOD_DIRECT, METHOD_TREECODE = 0, 1
ASSIGN_COMPLETE, ASSIGN_REFERENCE = 0, 1
LIST_DUAL, LIST_LEAF = 0, 1
REBUILD_AUTO, REBUILD_STATIC, REBUILD_RESORT = 0, 1, 2
STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "NOMEM", 4: "TIMEOUT", 5: "TREE", 6: "STATE",
          7: "UNSUPPORTED", 8: "CAPACITY"}


class FssError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fss error {STATUS.get(code, code)}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32), ("method", C.c_int32),
                ("tree_levels", C.c_int32), ("leaf_target", C.c_int32), ("degree", C.c_int32),
                ("theta", C.c_double), ("many_count", C.c_int32), ("assign_mode", C.c_int32),
                ("list_mode", C.c_int32), ("use_graph", C.c_int32), ("src_parts", C.c_int32),
                ("block_threads", C.c_int32), ("targets_per_thread", C.c_int32), ("autotune", C.c_int32),
                ("rebuild", C.c_int32), ("cluster_targets", C.c_int32), ("wait_limit_us", C.c_int32),
                ("reserved", C.c_int32 * 3)]


class ShardInfo(C.Structure):
    _fields_ = [("rank", C.c_int32), ("nranks", C.c_int32), ("unit_level", C.c_int32), ("pad", C.c_int32),
                ("units", C.c_int64), ("unit_lo", C.c_int64), ("unit_hi", C.c_int64), ("target_lo", C.c_int64),
                ("target_hi", C.c_int64), ("cost_total", C.c_double), ("cost_own", C.c_double)]


class TreeInfo(C.Structure):
    _fields_ = [("tree_levels", C.c_int32), ("leaf_count", C.c_int32), ("degree", C.c_int32),
                ("n_proxy", C.c_int32), ("n_pairs", C.c_int64), ("n_list_entries", C.c_int64),
                ("n_items", C.c_int64), ("n_tiles", C.c_int64), ("unassigned", C.c_int64), ("pp_interactions", C.c_double),
                ("pc_interactions", C.c_double), ("block_threads", C.c_int32),
                ("targets_per_thread", C.c_int32), ("src_parts", C.c_int32), ("target_clusters", C.c_int32),
                ("cp_interactions", C.c_double), ("cc_interactions", C.c_double),
                ("lane_pairs_leaf", C.c_double), ("lane_pairs_cluster", C.c_double),
                ("max_degree", C.c_int32), ("max_cluster_points", C.c_int32)]


def build():
    """Compile libfss.so for sm_100a (nvcc cross-compiles without a GPU)."""
    import subprocess
    subprocess.run(["make", "-s", "-j8", "-C", CSRC], check=True)


_lib = None
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_i64 = C.c_int64

# every symbol include/fss.h declares
SYMBOLS = ["fss_config_init", "fss_create", "fss_destroy", "fss_last_error", "fss_set_stream",
           "fss_set_particles", "fss_rebuild_tree", "fss_rhs", "fss_rhs_direct", "fss_rhs_treecode",
           "fss_rk4_step", "fss_rk4_step_host", "fss_get_state", "fss_rhs_current", "fss_remesh", "fss_remesh_current", "fss_get_tree_info",
           "fss_get_tree", "fss_set_leaf_params", "fss_profile_enable", "fss_profile_read",
           "fss_work_per_rhs", "fss_icos_counts", "fss_icos_grid", "fss_area_init",
           "fss_vorticity_rh4_ref", "fss_vorticity_rh_vortices", "fss_tree_traverse", "fss_interp_nodes",
           "fss_tree_geometry", "fss_rhs_direct_noalloc", "fss_mlp_create", "fss_mlp_destroy",
           "fss_mlp_param_count", "fss_mlp_init", "fss_mlp_set_params", "fss_mlp_get_params", "fss_mlp_set_data",
           "fss_mlp_gradient", "fss_mlp_train", "fss_mlp_predict", "fss_selector_class_table", "fss_selector_features",
           "fss_select_classes",
           "fss_selector_apply", "fss_ensemble_create", "fss_ensemble_destroy", "fss_ensemble_set_stream",
           "fss_ensemble_add", "fss_ensemble_build", "fss_ensemble_rk4_step", "fss_ensemble_get_state",
           "fss_ensemble_info", "fss_ensemble_time_pairs", "fss_amr_create", "fss_amr_destroy", "fss_amr_counts", "fss_amr_refine",
           "fss_amr_get_mesh", "fss_amr_remesh", "fss_amr_refine_current", "fss_remesh_lists", "fss_state_csv_append",
           "fss_point_count_append", "fss_output_name", "fss_state_bin_append", "fss_state_bin_read",
           "fss_read_points_csv", "fss_read_tris_csv", "fss_read_vert_tris_csv", "fss_test_hold_tile", "fss_test_hold_stage", "fss_test_resort_mode", "fss_get_stream", "fss_shard_partition", "fss_shard_set", "fss_shard_get_info",
           "fss_shard_stage", "fss_shard_combine", "fss_version"]

NOALLOC_MAX_PARTICLES = 262144  # FSS_NOALLOC_MAX_PARTICLES in include/fss.h


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FssError(7, f"{LIB_PATH} is not built (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    L.fss_config_init.argtypes = [P(Config)]
    L.fss_config_init.restype = None
    L.fss_create.argtypes = [P(Config), P(_vp)]
    L.fss_destroy.argtypes = [_vp]
    L.fss_destroy.restype = None
    L.fss_last_error.argtypes = [_vp]
    L.fss_last_error.restype = C.c_char_p
    L.fss_set_stream.argtypes = [_vp, _vp]
    L.fss_set_particles.argtypes = [_vp, _i64, _D, _D]
    L.fss_rebuild_tree.argtypes = [_vp]
    for nm in ("fss_rhs", "fss_rhs_direct", "fss_rhs_treecode"):
        getattr(L, nm).argtypes = [_vp, _D, _D, C.c_double, _D, _vp]
    L.fss_rk4_step.argtypes = [_vp, C.c_double, C.c_double, C.c_int32]
    L.fss_rk4_step_host.argtypes = [_vp, _vp, C.c_double, C.c_double, C.c_int32]
    L.fss_get_state.argtypes = [_vp, _D]
    L.fss_rhs_current.argtypes = [_vp, C.c_double, _D, _vp]
    _I32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    L.fss_remesh.argtypes = [_i64, _D, _D, _i64, _I32, C.c_double, C.POINTER(_i64), C.POINTER(_i64)]
    L.fss_remesh_current.argtypes = [_vp, _i64, _vp, C.c_double, C.POINTER(_i64), C.POINTER(_i64)]
    L.fss_get_tree_info.argtypes = [_vp, P(TreeInfo)]
    L.fss_get_tree.argtypes = [_vp, _vp, _vp, _vp, _i64]
    L.fss_set_leaf_params.argtypes = [_vp, C.c_int32, _I, _D]
    L.fss_profile_enable.argtypes = [_vp, C.c_int32]
    L.fss_profile_read.argtypes = [_vp, C.c_char_p, C.c_int32, _vp, _vp, C.c_int32, P(C.c_int32)]
    L.fss_work_per_rhs.argtypes = [_vp, P(C.c_double), P(C.c_double)]
    L.fss_icos_counts.argtypes = [C.c_int32, P(_i64), P(_i64)]
    L.fss_icos_grid.argtypes = [C.c_int32, _D, _I]
    L.fss_area_init.argtypes = [_i64, _D, _i64, _I, _D]
    L.fss_vorticity_rh4_ref.argtypes = [_i64, _D]
    L.fss_vorticity_rh_vortices.argtypes = [_i64, _D, _vp, C.c_double, C.c_int32, C.c_double, C.c_uint64]
    L.fss_tree_traverse.argtypes = [C.c_int32, C.c_double, C.c_int32, _I, _vp, _i64, P(_i64)]
    L.fss_interp_nodes.argtypes = [C.c_int32, _D, _D]
    L.fss_tree_geometry.argtypes = [C.c_int32, _D]
    L.fss_rhs_direct_noalloc.argtypes = [_i64, _vp, _vp, C.c_double, _vp, _vp]
    L.fss_ensemble_create.argtypes = [P(Config), P(_vp)]
    L.fss_ensemble_destroy.argtypes = [_vp]
    L.fss_ensemble_destroy.restype = None
    L.fss_ensemble_set_stream.argtypes = [_vp, _vp]
    L.fss_ensemble_add.argtypes = [_vp, _i64, _D, _D, P(C.c_int32)]
    L.fss_ensemble_build.argtypes = [_vp]
    L.fss_ensemble_rk4_step.argtypes = [_vp, C.c_double, C.c_double, C.c_int32]
    L.fss_ensemble_get_state.argtypes = [_vp, C.c_int32, _D]
    L.fss_ensemble_info.argtypes = [_vp, P(C.c_int32), P(_i64), P(C.c_double), P(_i64)]
    L.fss_ensemble_time_pairs.argtypes = [_vp, C.c_int32, P(C.c_double)]
    L.fss_amr_create.argtypes = [_i64, _i64, _I32, _vp, _i64, _i64, C.c_int32, P(_vp)]
    L.fss_amr_destroy.argtypes = [_vp]
    L.fss_amr_destroy.restype = None
    L.fss_amr_counts.argtypes = [_vp, P(_i64), P(_i64)]
    L.fss_amr_refine.argtypes = [_vp, P(_i64), _D, _D, C.c_double, C.c_double]
    L.fss_amr_get_mesh.argtypes = [_vp, _vp, _vp, _vp]
    L.fss_amr_remesh.argtypes = [_vp, _D, _D, C.c_double, P(_i64), P(_i64)]
    L.fss_amr_refine_current.argtypes = [_vp, _vp, C.c_double, C.c_double, C.c_double, P(_i64)]
    L.fss_remesh_lists.argtypes = [_i64, _D, _D, _i64, _I32, _I32, _I32, C.c_double, P(_i64), P(_i64)]
    L.fss_state_csv_append.argtypes = [C.c_char_p, _i64, _D, _D]
    L.fss_point_count_append.argtypes = [C.c_char_p, _i64]
    L.fss_output_name.argtypes = [C.c_char_p, _i64, _i64, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  _i64]
    L.fss_state_bin_append.argtypes = [C.c_char_p, _i64, _D, _D]
    L.fss_state_bin_read.argtypes = [C.c_char_p, _i64, _i64, _vp, _vp, P(_i64)]
    L.fss_read_points_csv.argtypes = [C.c_char_p, _i64, _D]
    L.fss_read_tris_csv.argtypes = [C.c_char_p, _i64, _I32]
    L.fss_read_vert_tris_csv.argtypes = [C.c_char_p, C.c_char_p, _i64, _I32, _I32, _i64]
    L.fss_version.restype = C.c_char_p
    L.fss_test_hold_tile.argtypes = [_vp, C.c_int32]
    L.fss_test_hold_stage.argtypes = [_vp, C.c_int32]
    L.fss_test_resort_mode.argtypes = [_vp, C.c_int32]
    L.fss_get_stream.argtypes = [_vp, P(_vp)]
    L.fss_shard_partition.argtypes = [_i64, _D, C.c_int32, np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
    L.fss_shard_set.argtypes = [_vp, C.c_int32, C.c_int32]
    L.fss_shard_get_info.argtypes = [_vp, P(ShardInfo)]
    L.fss_shard_stage.argtypes = [_vp, C.c_int32, _vp]
    L.fss_shard_combine.argtypes = [_vp, C.c_int32, C.c_double, C.c_double, _vp]
    _lib = L
    return L


def _check(rc, ctx=None):
    if rc != 0:
        msg = lib().fss_last_error(ctx).decode()
        raise FssError(rc, msg)


# ------------------------------------------------------------------ inputs

def icos_grid(level):
    """Level-`level` icosahedral vertices (icos_init order) and faces."""
    nv, nf = _i64(), _i64()
    _check(lib().fss_icos_counts(level, C.byref(nv), C.byref(nf)))
    xyz = np.zeros((nv.value, 3))
    faces = np.zeros((nf.value, 3), dtype=np.int32)
    _check(lib().fss_icos_grid(level, xyz.reshape(-1), faces.reshape(-1)))
    return xyz, faces


def area_init(state5, faces):
    s = np.ascontiguousarray(state5, dtype=np.float64)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    area = np.zeros(s.shape[0])
    _check(lib().fss_area_init(s.shape[0], s.reshape(-1), f.shape[0], f.reshape(-1), area))
    return area


RH_AMP = 7.848e-6 * 86400.0  # w = K of the Rossby-Haurwitz wave, per day


def remesh(moved5, target5, tris, omega=OMEGA):
    """remesh.h regrid_points2 (fss_remesh): (new target state, fallback
    count, not-found count)."""
    m = np.ascontiguousarray(moved5, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(target5, dtype=np.float64).copy().reshape(-1)
    tr = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    fb, bad = _i64(), _i64()
    _check(lib().fss_remesh(m.size // 5, m, t, tr.size // 3, tr, omega, C.byref(fb), C.byref(bad)))
    return t.reshape(-1, 5), fb.value, bad.value


def make_state(level, field="rh4_ref", n_vortex=0, seed=1, amp=RH_AMP, width=0.1):
    """(state5 (N,5), area (N,)) on the level-`level` icosahedral grid.

    field 'rh4_ref': the reference's rossby_haurwitz_4 (vorticity_functions.h:13).
    field 'rh_vortices': RH R=4 wave (w = K = amp) + n_vortex seeded Gaussian vortices.
    field 'gauss_ref': the reference's gauss_vortex (vorticity_functions.h:26-45:
    4 pi exp(-16 |c - x|^2) about colatitude pi/2 - pi/20, mean removed;
    tracer 2 + latitude), in numpy (not bit-exact with the reference).
    """
    xyz, faces = icos_grid(level)
    s = np.zeros((xyz.shape[0], 5))
    s[:, :3] = xyz
    area = area_init(s, faces)
    if field == "rh4_ref":
        _check(lib().fss_vorticity_rh4_ref(s.shape[0], s.reshape(-1)))
    elif field == "gauss_ref":
        xyz = s[:, :3]
        c = np.array([np.cos(np.pi / 20), 0.0, np.sin(np.pi / 20)])
        z = 4 * np.pi * np.exp(-16 * np.sum((c - xyz) ** 2, axis=1))
        s[:, 3] = z - np.sum(z * area) / (4 * np.pi)
        s[:, 4] = 2 + (np.pi / 2 - np.arctan2(np.hypot(xyz[:, 0], xyz[:, 1]), xyz[:, 2]))
    elif field == "rh_vortices":
        _check(lib().fss_vorticity_rh_vortices(s.shape[0], s.reshape(-1), area.ctypes.data_as(_vp), amp,
                                               n_vortex, width, seed))
    else:
        raise ValueError(field)
    return s, area


def tree_traverse(tree_levels, theta, many_count, counts):
    """fast_rhs.h:16 tree_traverse on per-face counts (host): pairs (P, 7)."""
    cnt = np.ascontiguousarray(counts, dtype=np.int32)
    npairs = _i64()
    rc = lib().fss_tree_traverse(tree_levels, theta, many_count, cnt, None, 0, C.byref(npairs))
    if rc not in (0, 8):
        _check(rc)
    pairs = np.zeros((max(npairs.value, 1), 7), dtype=np.int32)
    _check(lib().fss_tree_traverse(tree_levels, theta, many_count, cnt, pairs.ctypes.data_as(_vp), npairs.value,
                                   C.byref(npairs)))
    return pairs[:npairs.value]


def interp_nodes(degree):
    """(nodes (K, 3) barycentric, vinv (K, K)) of the degree-n proxy set."""
    K = (degree + 1) * (degree + 2) // 2
    nodes = np.zeros((K, 3))
    vinv = np.zeros((K, K))
    _check(lib().fss_interp_nodes(degree, nodes.reshape(-1), vinv.reshape(-1)))
    return nodes, vinv


def tree_geometry(tree_levels):
    """Circumcentre + circumradius per face, levels 0..tree_levels-1 concatenated."""
    nf = sum(20 * 4 ** l for l in range(tree_levels))
    ti = np.zeros((nf, 4))
    _check(lib().fss_tree_geometry(tree_levels, ti.reshape(-1)))
    return ti


# ------------------------------------------------------------------ context

class Context:
    """One problem on one GPU.  Keyword arguments set fss_config fields."""

    def __init__(self, **kw):
        L = lib()
        cfg = Config()
        L.fss_config_init(C.byref(cfg))
        for k, v in kw.items():
            if not hasattr(cfg, k):
                raise TypeError(f"unknown config field {k}")
            setattr(cfg, k, v)
        self.cfg = cfg
        h = _vp()
        _check(L.fss_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            lib().fss_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc):
        _check(rc, self.h)

    def set_stream(self, stream_handle):
        self._c(lib().fss_set_stream(self.h, stream_handle))

    def set_particles(self, state5, area):
        s = np.ascontiguousarray(state5, dtype=np.float64)
        a = np.ascontiguousarray(area, dtype=np.float64)
        self._c(lib().fss_set_particles(self.h, s.shape[0], s.reshape(-1), a))
        self.n = s.shape[0]

    def rebuild_tree(self):
        self._c(lib().fss_rebuild_tree(self.h))

    def _rhs(self, fn, state5, area, omega, psi):
        s = np.ascontiguousarray(state5, dtype=np.float64)
        a = np.ascontiguousarray(area, dtype=np.float64)
        out = np.zeros_like(s)
        p = np.zeros(s.shape[0]) if psi else None
        self._c(fn(self.h, s.reshape(-1), a, omega, out.reshape(-1), p.ctypes.data_as(_vp) if psi else None))
        return (out, p) if psi else out

    def rhs(self, state5, area, omega=OMEGA, psi=False):
        """rhs_eval.h:47 rhs_func: modify (N,5) [and psi (N,)]."""
        return self._rhs(lib().fss_rhs, state5, area, omega, psi)

    def rhs_direct(self, state5, area, omega=OMEGA, psi=False):
        return self._rhs(lib().fss_rhs_direct, state5, area, omega, psi)

    def rhs_treecode(self, state5, area, omega=OMEGA, psi=False):
        return self._rhs(lib().fss_rhs_treecode, state5, area, omega, psi)

    def remesh_current(self, tris=None, omega=OMEGA):
        """remesh.h regrid_points2 on the device state, onto the positions
        given to set_particles; returns (fallback count, not-found count).
        tris=None reuses the triangles of the previous call."""
        fb, bad = _i64(), _i64()
        if tris is None:
            self._c(lib().fss_remesh_current(self.h, 0, None, omega, C.byref(fb), C.byref(bad)))
            return fb.value, bad.value
        t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
        self._c(lib().fss_remesh_current(self.h, t.size // 3, t.ctypes.data_as(_vp), omega, C.byref(fb),
                                         C.byref(bad)))
        return fb.value, bad.value

    def amr_refine_current(self, amr, vorticity_tol=0.2, circulation_tol=0.0025, omega=OMEGA):
        """amr() on the context's particles (they must be the mesh's points),
        new midpoints projected, the new set taken; returns the new count."""
        pc = _i64()
        self._c(lib().fss_amr_refine_current(self.h, amr.h, vorticity_tol, circulation_tol, omega, C.byref(pc)))
        self.n = pc.value
        return pc.value

    def rhs_current(self, omega=OMEGA, psi=False):
        out = np.zeros((self.n, 5))
        p = np.zeros(self.n) if psi else None
        self._c(lib().fss_rhs_current(self.h, omega, out.reshape(-1), p.ctypes.data_as(_vp) if psi else None))
        return (out, p) if psi else out

    def rk4_step(self, dt, omega=OMEGA, nsteps=1):
        self._c(lib().fss_rk4_step(self.h, dt, omega, nsteps))

    def rk4_step_host(self, state5, dt, omega=OMEGA, nsteps=1):
        """In place on a C-contiguous float64 (N,5) array (may be pinned)."""
        assert state5.dtype == np.float64 and state5.flags.c_contiguous
        self._c(lib().fss_rk4_step_host(self.h, state5.ctypes.data_as(_vp), dt, omega, nsteps))
        return state5

    def rk4_step_host_ptr(self, ptr, dt, omega=OMEGA, nsteps=1):
        self._c(lib().fss_rk4_step_host(self.h, ptr, dt, omega, nsteps))

    def get_state(self):
        out = np.zeros((self.n, 5))
        self._c(lib().fss_get_state(self.h, out.reshape(-1)))
        return out

    def tree_info(self):
        ti = TreeInfo()
        self._c(lib().fss_get_tree_info(self.h, C.byref(ti)))
        return {k: getattr(ti, k) for k, _ in TreeInfo._fields_}

    def get_tree(self):
        """(loc[levels, N], counts, pairs[P, 7]) in the reference's formats."""
        ti = self.tree_info()
        TL = ti["tree_levels"]
        nf = sum(20 * 4 ** l for l in range(TL))
        loc = np.zeros((TL, self.n), dtype=np.int32)
        counts = np.zeros(nf, dtype=np.int32)
        pairs = np.zeros((ti["n_pairs"], 7), dtype=np.int32)
        self._c(lib().fss_get_tree(self.h, loc.ctypes.data_as(_vp), counts.ctypes.data_as(_vp),
                                   pairs.ctypes.data_as(_vp), ti["n_pairs"]))
        return loc, counts, pairs

    def set_leaf_params(self, degree, theta):
        d = np.ascontiguousarray(degree, dtype=np.int32)
        t = np.ascontiguousarray(theta, dtype=np.float64)
        self._c(lib().fss_set_leaf_params(self.h, d.size, d, t))

    def profile(self, on=True):
        self._c(lib().fss_profile_enable(self.h, 1 if on else 0))

    def profile_read(self):
        names = C.create_string_buffer(4096)
        ms = np.zeros(64)
        ln = np.zeros(64, dtype=np.int64)
        cnt = C.c_int32()
        self._c(lib().fss_profile_read(self.h, names, 4096, ms.ctypes.data_as(_vp), ln.ctypes.data_as(_vp), 64,
                                       C.byref(cnt)))
        nm = names.value.decode().split("\n")[:cnt.value]
        return {n: (float(ms[i]), int(ln[i])) for i, n in enumerate(nm)}

    def work_per_rhs(self):
        a, b = C.c_double(), C.c_double()
        self._c(lib().fss_work_per_rhs(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def stream_handle(self):
        """The cudaStream_t the context launches on (an int)."""
        h = _vp()
        self._c(lib().fss_get_stream(self.h, C.byref(h)))
        return h.value or 0

    def shard(self, rank, nranks):
        """Make this context rank `rank` of `nranks` of one sharded problem
        (fss_shard_set; nranks = 0 undoes it)."""
        self._c(lib().fss_shard_set(self.h, rank, nranks))

    def shard_info(self):
        i = ShardInfo()
        self._c(lib().fss_shard_get_info(self.h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in ShardInfo._fields_ if k != "pad"}

    def shard_stage(self, stage, exchange):
        """Stage `stage` for this rank's targets into the exchange buffer (a
        device pointer, or a tensor with data_ptr())."""
        ptr = exchange if isinstance(exchange, int) else exchange.data_ptr()
        self._c(lib().fss_shard_stage(self.h, stage, ptr))

    def shard_combine(self, stage, dt, exchange, omega=OMEGA):
        ptr = exchange if isinstance(exchange, int) else exchange.data_ptr()
        self._c(lib().fss_shard_combine(self.h, stage, dt, omega, ptr))

    def test_hold_tile(self, block=0):
        """Test hook: the next evaluation's target-leaf pair block `block`
        withholds its first source tile, so that its bounded waits run out
        (fss_test_hold_tile)."""
        self._c(lib().fss_test_hold_tile(self.h, block))

    def test_hold_stage(self, which=0):
        """Test hook: block 0 of the next evaluation's proxy-charge (0) or
        cluster-coefficient (1) launch withholds the bulk copy of its matrix,
        so that its bounded wait runs out (fss_test_hold_stage)."""
        self._c(lib().fss_test_hold_stage(self.h, which))

    def test_resort_mode(self, mode=0):
        """Test hook: the per-step re-sort by partition of the old order (0,
        the default) or by the radix key sort (1) (fss_test_resort_mode)."""
        self._c(lib().fss_test_resort_mode(self.h, mode))


def shard_partition(cost, nranks):
    """Contiguous unit ranges of near-equal cost (host only): bounds[r] ..
    bounds[r + 1] for rank r."""
    cost = np.ascontiguousarray(cost, dtype=np.float64)
    b = np.zeros(nranks + 1, dtype=np.int64)
    _check(lib().fss_shard_partition(cost.size, cost, nranks, b))
    return b


def rhs_direct_noalloc(n, state5_dev_ptr, area_dev_ptr, out5_dev_ptr, stream_handle=None, omega=OMEGA):
    """fss_rhs_direct_noalloc on caller-owned device buffers (raw pointers);
    asynchronous on the given stream.  Raises FssError on a bad size."""
    _check(lib().fss_rhs_direct_noalloc(n, state5_dev_ptr, area_dev_ptr, omega, out5_dev_ptr, stream_handle))


def remesh_lists(moved5, target5, tris, vt_off, vt_adj, omega=OMEGA):
    """regrid_points2 with explicit vert_tris lists (CSR), tried in list
    order (fss_remesh_lists): (new target state, fallback count, not-found
    count)."""
    m = np.ascontiguousarray(moved5, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(target5, dtype=np.float64).copy().reshape(-1)
    tr = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    off = np.ascontiguousarray(vt_off, dtype=np.int32)
    adj = np.ascontiguousarray(vt_adj if len(vt_adj) else np.zeros(1), dtype=np.int32)
    fb, bad = _i64(), _i64()
    _check(lib().fss_remesh_lists(m.size // 5, m, t, tr.size // 3, tr, off, adj, omega, C.byref(fb), C.byref(bad)))
    return t.reshape(-1, 5), fb.value, bad.value


# ------------------------------------------------------------------ files

def output_name(point_count, init_cond, use_fast, tree_levels=1, use_amr=False, use_mpi=False, use_remesh=False,
                time_steps=1):
    """The reference's <name> of output_<name>.csv / point_counts_<name>.csv."""
    buf = C.create_string_buffer(256)
    _check(lib().fss_output_name(buf, 256, point_count, init_cond.encode(), int(use_fast), tree_levels,
                                 int(use_amr), int(use_mpi), int(use_remesh), time_steps))
    return buf.value.decode()


def state_csv_append(path, state5, area):
    s = np.ascontiguousarray(state5, dtype=np.float64)
    _check(lib().fss_state_csv_append(str(path).encode(), s.shape[0], s.reshape(-1),
                                      np.ascontiguousarray(area, dtype=np.float64)))


def point_count_append(path, n):
    _check(lib().fss_point_count_append(str(path).encode(), n))


def state_bin_append(path, state5, area):
    s = np.ascontiguousarray(state5, dtype=np.float64)
    _check(lib().fss_state_bin_append(str(path).encode(), s.shape[0], s.reshape(-1),
                                      np.ascontiguousarray(area, dtype=np.float64)))


def state_bin_read(path, step):
    """(state5, area) of step `step` of a binary state file."""
    n = _i64()
    rc = lib().fss_state_bin_read(str(path).encode(), step, 0, None, None, C.byref(n))
    if rc not in (0, 8):
        _check(rc)
    s = np.zeros((n.value, 5))
    a = np.zeros(n.value)
    _check(lib().fss_state_bin_read(str(path).encode(), step, n.value, s.ctypes.data_as(_vp), a.ctypes.data_as(_vp),
                                    C.byref(n)))
    return s, a


def read_points_csv(path, n):
    """x, y, z, zeta of the reference's <N>points_rh4.csv (tracer left 0)."""
    s = np.zeros((n, 5))
    _check(lib().fss_read_points_csv(str(path).encode(), n, s.reshape(-1)))
    return s


def read_tris_csv(path, ntri):
    t = np.zeros((ntri, 3), dtype=np.int32)
    _check(lib().fss_read_tris_csv(str(path).encode(), ntri, t.reshape(-1)))
    return t


def read_vert_tris_csv(lists_path, counts_path, n, cap):
    """The reference's vert_tris lists as CSR (off[n + 1], adj)."""
    off = np.zeros(n + 1, dtype=np.int32)
    adj = np.zeros(max(cap, 1), dtype=np.int32)
    _check(lib().fss_read_vert_tris_csv(str(lists_path).encode(), str(counts_path).encode(), n, off, adj, cap))
    return off, adj[:off[-1]].copy()


AMR_VORTICITY_TOL, AMR_CIRCULATION_TOL = 0.2, 0.0025  # amr.h:14-15


class Amr:
    """amr.h amr on a device-resident triangle mesh (fss_amr_*): refine()
    appends points to host arrays with room for max_count points; mesh()
    returns (tris, corner_keys, parent_verts); remesh() is regrid_points2 on
    this mesh with the vert_tris lists amr() leaves."""

    def __init__(self, tris, n, max_count, max_tris, parent_verts=None, device=0):
        t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
        pv = None if parent_verts is None else np.ascontiguousarray(parent_verts, dtype=np.int32).reshape(-1)
        self.h = _vp()
        self.max_count = max_count
        _check(lib().fss_amr_create(n, t.size // 3, t, None if pv is None else pv.ctypes.data_as(_vp), max_count,
                                    max_tris, device, C.byref(self.h)))

    def counts(self):
        n, nt = _i64(), _i64()
        _check(lib().fss_amr_counts(self.h, C.byref(n), C.byref(nt)))
        return n.value, nt.value

    def refine(self, state5, area, vorticity_tol=AMR_VORTICITY_TOL, circulation_tol=AMR_CIRCULATION_TOL):
        """(state5, area) of the current points -> (new state5, new area)."""
        n = state5.shape[0]
        st = np.zeros((self.max_count, 5)); st[:n] = state5
        ar = np.zeros(self.max_count); ar[:n] = area
        pc = _i64(n)
        _check(lib().fss_amr_refine(self.h, C.byref(pc), st.reshape(-1), ar, vorticity_tol, circulation_tol))
        return st[:pc.value].copy(), ar[:pc.value].copy()

    def mesh(self):
        n, nt = self.counts()
        tris = np.zeros((nt, 3), dtype=np.int32)
        keys = np.zeros((nt, 3), dtype=np.uint64)
        par = np.zeros((n, 2), dtype=np.int32)
        _check(lib().fss_amr_get_mesh(self.h, tris.ctypes.data_as(_vp), keys.ctypes.data_as(_vp),
                                      par.ctypes.data_as(_vp)))
        return tris, keys, par

    def remesh(self, moved5, target5, omega=OMEGA):
        m = np.ascontiguousarray(moved5, dtype=np.float64)
        t = np.ascontiguousarray(target5, dtype=np.float64).copy()
        fb, bad = _i64(), _i64()
        _check(lib().fss_amr_remesh(self.h, m.reshape(-1), t.reshape(-1), omega, C.byref(fb), C.byref(bad)))
        return t, fb.value, bad.value

    def close(self):
        if self.h:
            lib().fss_amr_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """Independent problems of uneven size advanced together (mixed-precision
    treecode): one persistent pair-kernel launch per RK stage for all members,
    one CUDA graph per RK4 step."""

    def __init__(self, **kw):
        L = lib()
        cfg = Config()
        L.fss_config_init(C.byref(cfg))
        for k, v in kw.items():
            if not hasattr(cfg, k):
                raise TypeError(f"unknown config field {k}")
            setattr(cfg, k, v)
        h = _vp()
        _check(L.fss_ensemble_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.sizes = []

    def close(self):
        if getattr(self, "h", None):
            lib().fss_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle):
        _check(lib().fss_ensemble_set_stream(self.h, stream_handle))

    def add(self, state5, area):
        s = np.ascontiguousarray(state5, dtype=np.float64)
        a = np.ascontiguousarray(area, dtype=np.float64)
        m = C.c_int32()
        _check(lib().fss_ensemble_add(self.h, s.shape[0], s.reshape(-1), a, C.byref(m)))
        self.sizes.append(s.shape[0])
        return m.value

    def build(self):
        _check(lib().fss_ensemble_build(self.h))

    def rk4_step(self, dt, omega=OMEGA, nsteps=1):
        _check(lib().fss_ensemble_rk4_step(self.h, dt, omega, nsteps))

    def get_state(self, member):
        out = np.zeros((self.sizes[member], 5))
        _check(lib().fss_ensemble_get_state(self.h, member, out.reshape(-1)))
        return out

    def time_pairs(self, reps=3):
        """Device ms of one persistent pair launch (mean of `reps`)."""
        ms = C.c_double()
        _check(lib().fss_ensemble_time_pairs(self.h, reps, C.byref(ms)))
        return ms.value

    def info(self):
        m, n, w = C.c_int32(), _i64(), _i64()
        inter = C.c_double()
        _check(lib().fss_ensemble_info(self.h, C.byref(m), C.byref(n), C.byref(inter), C.byref(w)))
        return {"members": m.value, "particles": n.value, "interactions_per_rhs": inter.value, "work_items": w.value}


def version():
    return lib().fss_version().decode()

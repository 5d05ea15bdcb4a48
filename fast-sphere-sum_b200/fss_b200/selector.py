"""Learned per-leaf interpolation degree and MAC for the treecode.

For each target leaf, the selector chooses one of 12 classes (n, theta) from
{4, 6, 8, 10} x {0.5, 0.6, 0.7}. It picks the classes with the fewest
interactions that keep the velocity error below a relative-L2 tolerance.
The network is a 16-64-64-12 MLP with BF16 weights and FP32 accumulation.
It is trained and run by the library's own kernels (``fss_mlp_*``). It
predicts log10(e_l(c) / U) for every leaf l and class c, where e_l is the
L2 velocity error over the leaf's particles and U the RMS speed. Labels come
from the treecode itself: for each class, every leaf runs that class in
mixed precision, and the result is compared with the FP64 direct sum on the
GPU.

    python -m fss_b200.selector gen   --out sel_data.npz [--fields 24] [--clusters]
    python -m fss_b200.selector train --data sel_data.npz --out selector_weights.npz
    python -m fss_b200.selector eval  --weights selector_weights.npz --level 8 --seed 999 [--clusters]

Two networks: one for target-leaf evaluation (every far source summed at
the particles, per-leaf traversal) and one for target clusters (the
reference's cp/cc types; the per-leaf choices are carried up to the faces
of a dual traversal), each trained on labels of its own mode.  The trained
weights used by default sit beside this file (``selector_weights.npz``,
``selector_weights_clusters.npz``); they carry the feature standardisation
and the training record.
"""
import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import (FssError, LIST_DUAL, LIST_LEAF, METHOD_DIRECT, METHOD_TREECODE, PREC_FP64, PREC_MIXED, Context, RH_AMP,
               _check, lib, make_state)

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "selector_weights.npz")
WEIGHTS_CLUSTERS = os.path.join(HERE, "selector_weights_clusters.npz")
NCLS, NFEAT = 12, 16


def class_table(clusters=False):
    """(degrees, thetas) of the 12 classes, c = 3 i + j: n = 4 + 2i, theta =
    0.5 + 0.1 j for target-leaf evaluation; n = 6 + 2i, theta = 0.7 + 0.1 j
    with target clusters."""
    n0, t0 = (6, 0.7) if clusters else (4, 0.5)
    return [n0 + 2 * (c // 3) for c in range(NCLS)], [t0 + 0.1 * (c % 3) for c in range(NCLS)]


DEGREES, THETAS = class_table(False)
FLOOR = 1e-12  # labels below this relative error carry no information
_vp = C.c_void_p


def _setup():
    L = lib()
    if getattr(L, "_sel_ready", False):
        return L
    P = C.POINTER
    L.fss_mlp_create.argtypes = [C.c_int32, P(_vp)]
    L.fss_mlp_destroy.argtypes = [_vp]
    L.fss_mlp_destroy.restype = None
    L.fss_mlp_param_count.restype = C.c_int32
    L.fss_mlp_init.argtypes = [_vp, C.c_uint64]
    L.fss_mlp_set_params.argtypes = [_vp, _vp]
    L.fss_mlp_get_params.argtypes = [_vp, _vp]
    L.fss_mlp_set_data.argtypes = [_vp, C.c_int64, _vp, _vp, _vp]
    L.fss_mlp_gradient.argtypes = [_vp, _vp, P(C.c_double)]
    L.fss_mlp_train.argtypes = [_vp, C.c_int32, C.c_int32, C.c_double, C.c_uint64, _vp]
    L.fss_mlp_predict.argtypes = [_vp, C.c_int64, _vp, _vp]
    L.fss_selector_features.argtypes = [_vp, _vp, _vp, P(C.c_double)]
    L.fss_select_classes.argtypes = [C.c_int64, C.c_int32, _vp, _vp, C.c_double, _vp]
    L.fss_selector_class_table.argtypes = [C.c_int32, _vp, _vp]
    L.fss_selector_apply.argtypes = [_vp, _vp, _vp, _vp, C.c_double, C.c_double, _vp]
    L._sel_ready = True
    return L


def _p(a):
    return a.ctypes.data_as(_vp)


class MLP:
    """The selector network on one GPU (owns an fss_mlp)."""

    def __init__(self, device=0, params=None, seed=1):
        L = _setup()
        h = _vp()
        _check(L.fss_mlp_create(device, C.byref(h)))
        self.h = h
        self.nparams = L.fss_mlp_param_count()
        if params is not None:
            self.set_params(params)
        else:
            _check(L.fss_mlp_init(self.h, seed))

    def close(self):
        if getattr(self, "h", None):
            lib().fss_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        _check(lib().fss_mlp_set_params(self.h, _p(p)))

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        _check(lib().fss_mlp_get_params(self.h, _p(p)))
        return p

    def set_data(self, x, t, mask=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32)
        self._keep = (x, t, m)
        _check(lib().fss_mlp_set_data(self.h, x.shape[0], _p(x), _p(t), None if m is None else _p(m)))

    def gradient(self):
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_double()
        _check(lib().fss_mlp_gradient(self.h, _p(g), C.byref(loss)))
        return g, loss.value

    def train(self, epochs, batch=4096, lr=1e-3, seed=0):
        losses = np.zeros(epochs)
        _check(lib().fss_mlp_train(self.h, epochs, batch, lr, seed, _p(losses)))
        return losses

    def predict(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], NCLS), dtype=np.float32)
        _check(lib().fss_mlp_predict(self.h, x.shape[0], _p(x), _p(y)))
        return y


def unpack(p):
    """(W1, b1, W2, b2, W3, b3) views of a flat parameter vector."""
    o = 0
    out = []
    for shape in ((64, 16), (64,), (64, 64), (64,), (12, 64), (12,)):
        k = int(np.prod(shape))
        out.append(np.asarray(p[o:o + k]).reshape(shape))
        o += k
    return out


# ------------------------------------------------------------------ data

def features(ctx):
    """(features (nleaf, 16), costs (nleaf, 12), U) of a built treecode context."""
    L = _setup()
    info = ctx.tree_info()
    nleaf = info["leaf_count"]
    f = np.zeros((nleaf, NFEAT), dtype=np.float32)
    k = np.zeros((nleaf, NCLS))
    u = C.c_double()
    _check(L.fss_selector_features(ctx.h, _p(f), _p(k), C.byref(u)), ctx.h)
    return f, k, u.value


def leaf_of(ctx):
    loc, _, _ = ctx.get_tree()
    return loc[-1]


def field(level, seed, n_vortex, amp_scale=1.0):
    s, a = make_state(level, "rh_vortices", n_vortex=n_vortex, seed=seed, amp=RH_AMP * amp_scale)
    return s, a


def default_weights(clusters):
    return WEIGHTS_CLUSTERS if clusters else WEIGHTS


def label_field(s, a, device=0, clusters=False):
    """Features, costs and per-class log errors of every leaf of one field
    (target-leaf evaluation, or target clusters with `clusters`)."""
    with Context(method=METHOD_DIRECT, precision=PREC_FP64, device=device) as d:
        d.set_particles(s, a)
        uref = d.rhs(s, a)[:, :3]
    U = float(np.sqrt(np.mean(np.sum(uref ** 2, 1))))
    y = None
    X = K = None
    degrees, thetas = class_table(clusters)
    for c in range(NCLS):
        with Context(method=METHOD_TREECODE, precision=PREC_MIXED, list_mode=LIST_DUAL if clusters else LIST_LEAF,
                     cluster_targets=int(clusters), degree=degrees[c], theta=thetas[c], device=device) as ctx:
            ctx.set_particles(s, a)
            if X is None:
                X, K, _ = features(ctx)
                leaf = leaf_of(ctx)
                nleaf = X.shape[0]
                y = np.zeros((nleaf, NCLS))
            u = ctx.rhs(s, a)[:, :3]
        e2 = np.bincount(leaf, weights=np.sum((u - uref) ** 2, 1), minlength=nleaf)
        y[:, c] = np.log10(np.sqrt(e2) / U + FLOOR)
    counts = np.bincount(leaf, minlength=X.shape[0])
    return X, y, K, counts


def generate(out, fields, seed0=100, levels=(7, 8), device=0, log=print, clusters=False):
    """Training set from `fields` seeded fields alternating over `levels`."""
    rng = np.random.default_rng(seed0)
    Xs, Ys, Ks, Ns, meta = [], [], [], [], []
    t0 = time.time()
    for i in range(fields):
        level = levels[i % len(levels)]
        nv = int(rng.integers(4, 33))
        amp = float(rng.uniform(0.95, 1.05))
        seed = seed0 + i
        s, a = field(level, seed, nv, amp)
        X, y, K, cnt = label_field(s, a, device, clusters)
        keep = cnt > 0
        Xs.append(X[keep]); Ys.append(y[keep]); Ks.append(K[keep]); Ns.append(cnt[keep])
        meta.append(dict(level=level, seed=seed, n_vortex=nv, amp_scale=amp, leaves=int(keep.sum()),
                         clusters=bool(clusters)))
        log(f"field {i}: level {level} seed {seed} vortices {nv} leaves {int(keep.sum())} ({time.time() - t0:.0f}s)")
    np.savez_compressed(out, X=np.concatenate(Xs), Y=np.concatenate(Ys), K=np.concatenate(Ks),
                        N=np.concatenate(Ns), meta=json.dumps(meta))
    return out


def train(data, out, epochs=60, batch=4096, lr=2e-3, seed=0, holdout=0.1, device=0, log=print):
    d = np.load(data)
    X, Y = d["X"].astype(np.float32), d["Y"].astype(np.float32)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(X.shape[0])
    nh = int(holdout * X.shape[0])
    te, tr = perm[:nh], perm[nh:]
    mean = X[tr].mean(0)
    std = X[tr].std(0) + 1e-6
    Xn = (X - mean) / std
    m = MLP(device=device, seed=seed + 1)
    m.set_data(Xn[tr], Y[tr])
    losses = m.train(epochs, batch=batch, lr=lr, seed=seed)
    p = m.params()
    pred = m.predict(Xn[te])
    rmse = float(np.sqrt(np.mean((pred - Y[te]) ** 2)))
    log(f"train loss {losses[-1]:.4f} (per-sample sum over 12 outputs); holdout RMSE {rmse:.3f} decades")
    np.savez(out, params=p, mean=mean, std=std, losses=losses, holdout_rmse=rmse,
             record=json.dumps(dict(data=os.path.basename(data), rows=int(X.shape[0]), epochs=epochs, batch=batch,
                                    lr=lr, seed=seed, holdout=holdout)))
    m.close()
    return out


def load(path=WEIGHTS):
    w = np.load(path)
    return w["params"].astype(np.float32), w["mean"].astype(np.float32), w["std"].astype(np.float32)


def apply(ctx, tol=1e-6, safety=2.0, weights=None, device=0):
    """Choose per-leaf (n, theta) for `ctx` and switch it to per-leaf lists
    (with target clusters, when the context has them: the network of that
    mode).  Returns the class index of every leaf."""
    L = _setup()
    params, mean, std = load(weights or default_weights(bool(ctx.cfg.cluster_targets)))
    m = MLP(device=device, params=params)
    nleaf = ctx.tree_info()["leaf_count"]
    choice = np.zeros(nleaf, dtype=np.int32)
    try:
        _check(L.fss_selector_apply(ctx.h, m.h, _p(mean), _p(std), tol, safety, _p(choice)), ctx.h)
    finally:
        m.close()
    return choice


def select(pred, cost, budget):
    pred = np.ascontiguousarray(pred, dtype=np.float64)
    cost = np.ascontiguousarray(cost, dtype=np.float64)
    choice = np.zeros(pred.shape[0], dtype=np.int32)
    _check(_setup().fss_select_classes(pred.shape[0], pred.shape[1], _p(pred), _p(cost), budget, _p(choice)))
    return choice


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("gen")
    g.add_argument("--out", default="sel_data.npz")
    g.add_argument("--fields", type=int, default=24)
    g.add_argument("--seed", type=int, default=100)
    g.add_argument("--clusters", action="store_true")
    t = sub.add_parser("train")
    t.add_argument("--data", default="sel_data.npz")
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--epochs", type=int, default=60)
    t.add_argument("--lr", type=float, default=2e-3)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=None)
    e.add_argument("--clusters", action="store_true")
    e.add_argument("--level", type=int, default=8)
    e.add_argument("--seed", type=int, default=999)
    e.add_argument("--tol", type=float, default=1e-6)
    e.add_argument("--safety", type=float, default=2.0)
    a = ap.parse_args(argv)
    if a.cmd == "gen":
        generate(a.out, a.fields, a.seed, clusters=a.clusters)
    elif a.cmd == "train":
        train(a.data, a.out, epochs=a.epochs, lr=a.lr)
    else:
        print(json.dumps(evaluate(a.weights or default_weights(a.clusters), a.level, a.seed, a.tol, a.safety,
                                  clusters=a.clusters)))


def evaluate(weights, level, seed, tol=1e-6, safety=2.0, n_vortex=32, device=0, clusters=False):
    """Interactions and error of the selector against fixed n=8, theta=0.7
    (both with target clusters when `clusters`)."""
    s, a = field(level, seed, n_vortex)
    with Context(method=METHOD_DIRECT, precision=PREC_FP64, device=device) as d:
        d.set_particles(s, a)
        uref = d.rhs(s, a)[:, :3]
    nref = np.linalg.norm(uref)
    out = {}
    def work(i):
        return i["pp_interactions"] + i["pc_interactions"] + i["cp_interactions"] + i["cc_interactions"]

    with Context(method=METHOD_TREECODE, precision=PREC_MIXED, degree=8, theta=0.7, cluster_targets=int(clusters),
                 device=device) as c:
        c.set_particles(s, a)
        u = c.rhs(s, a)[:, :3]
        out["fixed"] = dict(rel_l2=float(np.linalg.norm(u - uref) / nref), interactions=work(c.tree_info()))
    with Context(method=METHOD_TREECODE, precision=PREC_MIXED, list_mode=LIST_LEAF, cluster_targets=int(clusters),
                 device=device) as c:
        c.set_particles(s, a)
        choice = apply(c, tol=tol, safety=safety, weights=weights, device=device)
        u = c.rhs(s, a)[:, :3]
        out["learned"] = dict(rel_l2=float(np.linalg.norm(u - uref) / nref), interactions=work(c.tree_info()),
                              classes=np.bincount(choice, minlength=NCLS).tolist())
    out["interaction_ratio"] = out["fixed"]["interactions"] / out["learned"]["interactions"]
    return out


if __name__ == "__main__":
    main()

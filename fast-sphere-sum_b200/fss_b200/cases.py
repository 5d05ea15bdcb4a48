"""Run one fixed case of the library (for profiling and quick checks).

    python -m fss_b200.cases rhs  --level 8 --precision mixed [--repeat 2]
    python -m fss_b200.cases rk4  --level 8 --precision mixed --steps 2 [--learned]
    python -m fss_b200.cases direct --level 6 --precision mixed
    python -m fss_b200.cases ensemble --members 64 --steps 20
    python -m fss_b200.cases mlp --samples 2097152 --epochs 2

The mlp case: the selector network (16 -> 64 -> 64 -> 12) trained by the
library's own kernels on seeded synthetic rows (about the size of the
per-leaf error label set, 2M rows), then run forward on all rows.

The ensemble case: members on icosahedral levels drawn uniformly from 5-8,
each an RH R=4 wave with a seeded +-5% amplitude perturbation and 4-16
Gaussian vortices; mixed-precision BLTC n=8, theta=0.7; one CUDA graph per
RK4 step for all members.

--learned: the learned per-leaf (degree, theta) choice (tolerance 1e-6,
safety 2) and the autotuned block shape (--block N: that shape instead),
with target clusters (the reference's cp/cc types) unless --no-clusters.

Inputs: icosahedral grid of the given level, RH4 wave + seeded vortices.
Prints one line with the wall time; exits non-zero on any library error.
"""
import argparse
import time

import numpy as np

from . import (METHOD_DIRECT, METHOD_TREECODE, PREC_FP64, PREC_MIXED, RH_AMP, Context, Ensemble, make_state)


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["rhs", "rk4", "direct", "ensemble", "mlp"])
    p.add_argument("--samples", type=int, default=2097152)
    p.add_argument("--epochs", type=int, default=2)
    p.add_argument("--members", type=int, default=64)
    p.add_argument("--seed", type=int, default=100)
    p.add_argument("--level", type=int, default=8)
    p.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--degree", type=int, default=8)
    p.add_argument("--theta", type=float, default=0.7)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--repeat", type=int, default=2)
    p.add_argument("--vortices", type=int, default=32)
    p.add_argument("--no-graph", action="store_true")
    p.add_argument("--learned", action="store_true")
    p.add_argument("--clusters", action="store_true", help="target clusters with fixed degree/theta")
    p.add_argument("--no-clusters", action="store_true")
    p.add_argument("--block", type=int, default=0,
                   help="pair-kernel block threads (no autotuning: the only pair launches before the steps are "
                        "the two of the selector's one right-hand side)")
    a = p.parse_args(argv)
    prec = PREC_MIXED if a.precision == "mixed" else PREC_FP64
    if a.case == "ensemble":
        return ensemble_case(a)
    if a.case == "mlp":
        return mlp_case(a)
    s, area = make_state(a.level, "rh_vortices", n_vortex=a.vortices, seed=2)
    method = METHOD_DIRECT if a.case == "direct" else METHOD_TREECODE
    t0 = time.perf_counter()
    extra = dict(list_mode=1, autotune=0 if a.block else 1) if a.learned else {}
    if a.block:
        extra["block_threads"] = a.block
    if (a.learned and not a.no_clusters) or a.clusters:
        extra["cluster_targets"] = 1
    with Context(method=method, precision=prec, degree=a.degree, theta=a.theta,
                 use_graph=0 if a.no_graph else 1, **extra) as ctx:
        ctx.set_particles(s, area)
        if a.learned:
            from . import selector
            selector.apply(ctx, tol=1e-6, safety=2.0)
        if a.case == "rk4":
            ctx.rk4_step(0.01, nsteps=a.steps)
            out = ctx.get_state()
        else:
            for _ in range(a.repeat):
                out = ctx.rhs(s, area)
        info = ctx.tree_info()
    assert np.all(np.isfinite(out))
    alg_leaf = info["pp_interactions"] + info["pc_interactions"]
    alg_cl = info["cp_interactions"] + info["cc_interactions"]
    print(f"case={a.case} level={a.level} n={s.shape[0]} precision={a.precision} "
          f"items={info['n_items']} block={info['block_threads']} "
          f"pairs_leaf={alg_leaf:.4g} lane_pairs_leaf={info['lane_pairs_leaf']:.4g} "
          f"pairs_cluster={alg_cl:.4g} lane_pairs_cluster={info['lane_pairs_cluster']:.4g} "
          f"wall={time.perf_counter() - t0:.3f}s")


def ensemble_case(a):
    import json
    rng = np.random.default_rng(a.seed)
    t0 = time.perf_counter()
    with Ensemble(degree=a.degree, theta=a.theta) as ens:
        levels = []
        for m in range(a.members):
            level = int(rng.integers(5, 9))
            nv = int(rng.integers(4, 17))
            amp = float(rng.uniform(0.95, 1.05))
            s, area = make_state(level, "rh_vortices", n_vortex=nv, seed=a.seed + m, amp=RH_AMP * amp)
            ens.add(s, area)
            levels.append(level)
        ens.build()
        t_build = time.perf_counter() - t0
        info = ens.info()
        ens.rk4_step(0.01, nsteps=1)
        _ = ens.get_state(0)                       # sync
        t1 = time.perf_counter()
        ens.rk4_step(0.01, nsteps=a.steps)
        out = ens.get_state(0)
        dt = time.perf_counter() - t1
    assert np.all(np.isfinite(out))
    print(json.dumps(dict(case="ensemble", members=a.members, levels=np.bincount(levels, minlength=9)[5:].tolist(),
                          particles=info["particles"], work_items=info["work_items"],
                          interactions_per_rhs=info["interactions_per_rhs"], steps=a.steps,
                          wall_s=dt, steps_per_s=a.steps / dt,
                          pairs_per_s=4 * a.steps * info["interactions_per_rhs"] / dt, build_s=t_build)))


def mlp_case(a):
    from . import selector
    rng = np.random.default_rng(a.seed)
    x = rng.standard_normal((a.samples, 16)).astype(np.float32)
    t = np.tanh(x[:, :12] * x[:, 4:]).astype(np.float32)
    net = selector.MLP(params=None, seed=a.seed)
    try:
        t0 = time.perf_counter()
        net.set_data(x, t)
        losses = net.train(a.epochs, batch=4096, lr=1e-3, seed=a.seed)
        y = net.predict(x)
        dt = time.perf_counter() - t0
    finally:
        net.close()
    assert np.all(np.isfinite(losses)) and np.all(np.isfinite(y))
    print(f"case=mlp samples={a.samples} epochs={a.epochs} loss={losses[-1]:.4e} wall={dt:.3f}s")


if __name__ == "__main__":
    main()

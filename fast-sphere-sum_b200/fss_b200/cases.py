"""Run one fixed case of the library (for profiling and quick checks).

    python -m fss_b200.cases rhs  --level 8 --precision mixed [--repeat 2]
    python -m fss_b200.cases rk4  --level 8 --precision mixed --steps 2
    python -m fss_b200.cases direct --level 6 --precision mixed

Inputs: icosahedral grid of the given level, RH4 wave + seeded vortices.
Prints one line with the wall time; exits non-zero on any library error.
"""
import argparse
import time

import numpy as np

from . import (METHOD_DIRECT, METHOD_TREECODE, PREC_FP64, PREC_MIXED, Context, make_state)


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["rhs", "rk4", "direct"])
    p.add_argument("--level", type=int, default=8)
    p.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--degree", type=int, default=8)
    p.add_argument("--theta", type=float, default=0.7)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--repeat", type=int, default=2)
    p.add_argument("--vortices", type=int, default=32)
    p.add_argument("--no-graph", action="store_true")
    a = p.parse_args(argv)
    prec = PREC_MIXED if a.precision == "mixed" else PREC_FP64
    s, area = make_state(a.level, "rh_vortices", n_vortex=a.vortices, seed=2)
    method = METHOD_DIRECT if a.case == "direct" else METHOD_TREECODE
    t0 = time.perf_counter()
    with Context(method=method, precision=prec, degree=a.degree, theta=a.theta,
                 use_graph=0 if a.no_graph else 1) as ctx:
        ctx.set_particles(s, area)
        if a.case == "rk4":
            ctx.rk4_step(0.01, nsteps=a.steps)
            out = ctx.get_state()
        else:
            for _ in range(a.repeat):
                out = ctx.rhs(s, area)
        info = ctx.tree_info()
    assert np.all(np.isfinite(out))
    print(f"case={a.case} level={a.level} n={s.shape[0]} precision={a.precision} "
          f"items={info['n_items']} wall={time.perf_counter() - t0:.3f}s")


if __name__ == "__main__":
    main()

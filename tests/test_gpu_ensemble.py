"""Ensemble: uneven members advanced together by one persistent pair-kernel
launch per RK stage must reproduce each member run on its own, bit for bit
(same work lists, same summation order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ensemble_matches_members_run_alone(fss):
    specs = [(4, 1, 4), (5, 2, 8), (3, 3, 2), (5, 4, 16), (4, 5, 6)]
    fields = [fss.make_state(level, "rh_vortices", n_vortex=nv, seed=seed) for level, seed, nv in specs]
    with fss.Ensemble(degree=8, theta=0.7) as ens:
        for s, a in fields:
            ens.add(s, a)
        ens.build()
        info = ens.info()
        assert info["members"] == len(specs) and info["particles"] == sum(len(s) for s, _ in fields)
        ens.rk4_step(0.01, nsteps=3)
        got = [ens.get_state(m) for m in range(len(fields))]
    for (s, a), g in zip(fields, got):
        with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, degree=8, theta=0.7,
                         block_threads=160, src_parts=1) as ctx:
            ctx.set_particles(s, a)
            ctx.rk4_step(0.01, nsteps=3)
            ref = ctx.get_state()
        assert np.array_equal(g, ref)
        assert np.abs(g[:, :3] - s[:, :3]).max() > 0  # particles moved


def test_ensemble_tracks_fp64_direct(fss):
    s, a = fss.make_state(5, "rh_vortices", n_vortex=8, seed=7)
    with fss.Ensemble() as ens:
        ens.add(s, a)
        ens.add(*fss.make_state(4, "rh_vortices", n_vortex=4, seed=8))
        ens.build()
        ens.rk4_step(0.01, nsteps=5)
        got = ens.get_state(0)
    with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_FP64) as d:
        d.set_particles(s, a)
        d.rk4_step(0.01, nsteps=5)
        ref = d.get_state()
    disp = ref[:, :3] - s[:, :3]
    assert np.linalg.norm(got[:, :3] - ref[:, :3]) / np.linalg.norm(disp) < 2e-6

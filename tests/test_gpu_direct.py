"""Direct sum on the GPU against the FP64 oracle (rhs_eval.h:15-56)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("level", [3, 4])
def test_direct_fp64_matches_oracle(fss, oracle, level):
    s, a = fss.make_state(level, "rh4_ref")
    ref = oracle.rhs_direct(s, a)
    with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_FP64) as ctx:
        ctx.set_particles(s, a)
        out = ctx.rhs(s, a)
    # FP64 with |x - y|^2 / 2 in place of 1 - x.y: agreement to ~1e-13
    assert rel_l2(out[:, :3], ref[:, :3]) < 1e-11
    assert np.max(np.abs(out[:, :3] - ref[:, :3])) < 1e-10 * np.max(np.abs(ref[:, :3]))
    assert rel_l2(out[:, 3], ref[:, 3]) < 1e-11          # dzeta/dt = -2 omega u_z
    assert np.all(out[:, 4] == 0.0)                       # tracer rate


@pytest.mark.parametrize("level", [3, 5])
def test_direct_mixed_matches_oracle(fss, oracle, level):
    s, a = fss.make_state(level, "rh_vortices", n_vortex=8, seed=1)
    with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        out = ctx.rhs(s, a)
    rows = np.arange(0, s.shape[0], max(1, s.shape[0] // 2048))
    ref = oracle.rhs_direct_rows(s, a, rows)
    # FP32 interactions with Kahan-compensated accumulation
    assert rel_l2(out[rows, :3], ref) < 1e-6


def test_direct_stream_function(fss, oracle):
    s, a = fss.make_state(4, "rh_vortices", n_vortex=4, seed=3)
    rows = np.arange(0, s.shape[0], 5)
    ref = oracle.stream_rows(s, a, rows)
    for prec, tol in ((fss.PREC_FP64, 1e-11), (fss.PREC_MIXED, 1e-6)):
        with fss.Context(method=fss.METHOD_DIRECT, precision=prec) as ctx:
            ctx.set_particles(s, a)
            out, psi = ctx.rhs(s, a, psi=True)
        assert rel_l2(psi[rows], ref) < tol, prec


def test_direct_parts_and_shapes_agree(fss, oracle):
    """Source-list splits and block shapes change only the summation order."""
    s, a = fss.make_state(4, "rh4_ref")
    ref = oracle.rhs_direct(s, a)
    for parts in (1, 3, 7):
        for bt in (0, 192, 288):
            with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_MIXED, src_parts=parts,
                             block_threads=bt) as ctx:
                ctx.set_particles(s, a)
                out = ctx.rhs(s, a)
            assert rel_l2(out[:, :3], ref[:, :3]) < 1e-6, (parts, bt)


def test_direct_ragged_sizes(fss, oracle):
    """Particle counts that are not multiples of any tile size."""
    s, a = fss.make_state(3, "rh4_ref")
    for n in (2, 3, 37, 129, 257, 601):
        ss, aa = s[:n].copy(), a[:n].copy()
        ref = oracle.rhs_direct(ss, aa)
        with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_FP64) as ctx:
            ctx.set_particles(ss, aa)
            out = ctx.rhs(ss, aa)
        assert rel_l2(out[:, :3], ref[:, :3]) < 1e-11, n


def test_rhs_repeat_deterministic(fss):
    s, a = fss.make_state(4, "rh4_ref")
    with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_MIXED) as ctx:
        ctx.set_particles(s, a)
        o1 = ctx.rhs(s, a)
        o2 = ctx.rhs(s, a)
    assert np.array_equal(o1, o2)

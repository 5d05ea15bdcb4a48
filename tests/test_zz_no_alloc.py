"""fss_rhs_direct_noalloc: the direct sum for callers that cannot allocate
device memory (real-time loops where cudaMalloc/cudaFree could stall the
device; plugins whose host application owns the device memory budget).

The caller owns every buffer (here torch tensors stand in for the caller's
memory).  The entry point must agree with the FP64 oracle (rhs_eval.h:15-56)
and with the allocating fss_rhs_direct to the mixed-precision tolerance used
throughout the tests, on two calls in a row that share its fixed scratch
array; it must take no device memory once its module is loaded; and it must
refuse sizes beyond its limit.  This file is collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_allocating_entry_on_two_calls(fss):
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    fields = [fss.make_state(5, "rh_vortices", n_vortex=8, seed=1),
              fss.make_state(4, "rh4_ref")]        # a smaller second call: stale scratch must not leak
    for state, area in fields:
        n = state.shape[0]
        with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_MIXED) as ctx:
            ctx.set_particles(state, area)
            expect = ctx.rhs_direct(state, area)
        s_d = torch.from_numpy(state).to(dev)
        a_d = torch.from_numpy(area).to(dev)
        out = torch.full((n, 5), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        fss.rhs_direct_noalloc(n, s_d.data_ptr(), a_d.data_ptr(), out.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_l2(got[:, :3], expect[:, :3]) < 1e-6
        assert rel_l2(got[:, 3], expect[:, 3]) < 1e-6
        assert np.all(got[:, 4] == 0.0)


def test_noalloc_matches_oracle_and_takes_no_memory(fss, oracle):
    import torch
    dev = torch.device("cuda", 0)
    state, area = fss.make_state(4, "rh_vortices", n_vortex=8, seed=5)
    n = state.shape[0]
    want = oracle.rhs_direct(state, area)
    s_d = torch.from_numpy(state).to(dev)
    a_d = torch.from_numpy(area).to(dev)
    outs = [torch.full((n, 5), float("nan"), dtype=torch.float64, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    fss.rhs_direct_noalloc(n, s_d.data_ptr(), a_d.data_ptr(), outs[0].data_ptr(), None)  # loads the module
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    fss.rhs_direct_noalloc(n, s_d.data_ptr(), a_d.data_ptr(), outs[1].data_ptr(), None)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0
    for o in outs:
        got = o.cpu().numpy()
        assert rel_l2(got[:, :3], want[:, :3]) < 1e-6
        assert rel_l2(got[:, 3], want[:, 3]) < 1e-6
    assert np.array_equal(outs[0].cpu().numpy(), outs[1].cpu().numpy())


def test_noalloc_rejects_sizes_beyond_its_limit(fss):
    import torch
    dev = torch.device("cuda", 0)
    small = torch.zeros(16, dtype=torch.float64, device=dev)
    n = fss.NOALLOC_MAX_PARTICLES + 1
    with pytest.raises(fss.FssError) as e:
        fss.rhs_direct_noalloc(n, small.data_ptr(), small.data_ptr(), small.data_ptr(), None)
    assert e.value.code == 8 and "scratch" in str(e.value)
    with pytest.raises(fss.FssError):
        fss.rhs_direct_noalloc(1, small.data_ptr(), small.data_ptr(), small.data_ptr(), None)

"""One problem sharded over several GPUs, one process per GPU.

Every rank holds the whole state and the same tree and evaluates the
right-hand side for its own targets (fss_shard_set); per RK stage the ranks
sum one exchange buffer (N x 4 float64 on the device: a rank's own rows hold
its velocity sums, every other row -0.0) with one all-reduce, after which
every rank advances all particles identically.  This replaces the
reference's per-stage state replication over MPI (mpi_utils.h:6-26
sync_state_direct / sync_state_fast after fast_sum_mpi.cpp:322-338 and
direct_sum_mpi.cpp:74-82 split the targets).

The collective belongs to the caller: ``allreduce(tensor)`` sums a tensor
over the ranks in place (torch.distributed.all_reduce over NCCL on GPUs,
over gloo on CPUs); the driver below only orders the calls.
"""
import numpy as np

from . import OMEGA


def exchange_buffer(ctx, device):
    """The exchange buffer of a sharded context: a torch tensor (N, 4)."""
    import torch
    return torch.empty((ctx.n, 4), dtype=torch.float64, device=device)


def torch_allreduce(group=None):
    """Sum over the ranks of a torch.distributed process group."""
    import torch.distributed as dist

    def f(t):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return f


def rk4_steps(ctx, exchange, dt, nsteps=1, allreduce=None, omega=OMEGA):
    """`nsteps` RK4 steps of a sharded context: per stage its own targets,
    one all-reduce of `exchange` (a torch tensor on the context's device),
    then the combine for every particle.  The all-reduce is issued on the
    stream the context launches on, so that it follows the stage's kernels
    and precedes the combine.  With allreduce=None the buffer is used as it
    is (one rank)."""
    on_device = getattr(exchange, "is_cuda", False)
    if on_device:
        import torch
        ctx_stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=exchange.device)
    for _ in range(nsteps):
        for stage in (1, 2, 3, 4):
            ctx.shard_stage(stage, exchange)
            if allreduce is not None:
                if on_device:
                    with torch.cuda.stream(ctx_stream):
                        allreduce(exchange)
                else:
                    allreduce(exchange)
            ctx.shard_combine(stage, dt, exchange, omega)


def owned_rows_exact(full, lo, hi):
    """The exchange form of rows [lo, hi) of `full` (N x 4): those rows, -0.0
    elsewhere (numpy; the reference semantics of the device buffer)."""
    out = np.full_like(full, -0.0)
    out[lo:hi] = full[lo:hi]
    return out

"""Benchmark: RK4 steps/s of the barotropic-vorticity treecode on B200.

Headline workload: 655,362 particles (icosahedral level 8), Rossby-Haurwitz
R=4 wave + 32 seeded Gaussian vortices, mixed-precision treecode (FP32
interactions with Kahan accumulation, FP64 RK4 / renormalisation /
interpolation weights) with the learned per-leaf degree/MAC and target
clusters, particles re-sorted into their current leaves every step,
dt = 0.01 day.  Beside it: the plain FP64 BLTC (n = 8, theta = 0.7) on the
same GPU (the ratio's denominator) and the FP64 treecode with the headline's
algorithm, the velocity error of each against the FP64 direct sum, an
end-to-end number through the C ABI with host buffers, the pair kernel's
roofline, and the reference's CPU direct sum timed on this host's cores.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Output: one JSON line of details (tree, per-kernel rooflines, every arm, the
reference's CPU fast sum, remesh, AMR, the 64-member ensemble), then the
headline JSON line, short and last (value, rel-L2 against the FP64 direct
sum, the ratio to the plain FP64 BLTC, e2e, roofline, clocks).

With N > 1 (torchrun) every rank runs an independent replica;
value = all ranks' steps / max-over-ranks time.  The reference arm
(--impl reference) builds its inputs with the oracle alone and never loads
the product library.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fast-sphere-sum_b200"))

METRIC = "RK4 steps/s, N=655,362: mixed+learned BLTC vs FP64 plain @ rel-L2≤1e-6"
UNIT = "steps/s"
FLOPS_PER_PAIR = 23  # algorithmic flops of one velocity pair interaction
DT = 0.01


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--level", type=int, default=8)
    p.add_argument("--degree", type=int, default=8)
    p.add_argument("--theta", type=float, default=0.7)
    p.add_argument("--vortices", type=int, default=32)
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-remesh", action="store_true")
    p.add_argument("--no-amr", action="store_true")
    p.add_argument("--no-ensemble", action="store_true")
    p.add_argument("--shard", action="store_true",
                   help="one problem split over the ranks (strong scaling; one all-reduce of N x 32 B per RK "
                        "stage) instead of one replica per rank")
    p.add_argument("--members", type=int, default=64, help="ensemble members (levels 5-8)")
    p.add_argument("--cpu-sample", type=int, default=2048, help="targets in one CPU-baseline sample")
    p.add_argument("--tol", type=float, default=1e-6, help="selector: relative L2 velocity error target")
    p.add_argument("--safety", type=float, default=1.5, help="selector: predicted-error safety factor")
    p.add_argument("--fixed", action="store_true", help="headline arm without the learned selector")
    p.add_argument("--no-clusters", action="store_true",
                   help="headline arm without target clusters (far sources summed at the target particles)")
    p.add_argument("--sweep", action="store_true",
                   help="instead of the headline line: mixed-precision BLTC at fixed n in {6,8,10} x theta in "
                        "{0.5,0.7}, one JSON line each (errors vs the FP64 direct sum, steps/s)")
    return p.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def max_over_ranks(x, ws):
    """The largest x over the ranks (a GPU tensor under NCCL, a CPU one under
    gloo)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(steps, seconds, ws):
    """Whole-job steps/s of ws replicas that each ran `steps` steps, timed by
    the slowest rank's `seconds` (every rank passes its own time)."""
    return ws * steps / max_over_ranks(seconds, ws)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """SM clock, power and clock-event reasons sampled through NVML every
    10 ms in a background thread while the timed region runs."""

    BITS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, dev):
        self.dev = dev
        self.rows = []
        self.h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self.nv = pynvml
            # match the CUDA device to its NVML handle by PCI location
            # (integers from both sides; no string/pointer conversions)
            prop = torch.cuda.get_device_properties(dev)
            want = (int(prop.pci_domain_id), int(prop.pci_bus_id), int(prop.pci_device_id))
            for i in range(pynvml.nvmlDeviceGetCount()):
                h = pynvml.nvmlDeviceGetHandleByIndex(i)
                pci = pynvml.nvmlDeviceGetPciInfo(h)
                if (int(pci.domain), int(pci.bus), int(pci.device)) == want:
                    self.h = h
                    break
            self.max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.h = None

    def _reasons(self):
        f = getattr(self.nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(self.nv, "nvmlDeviceGetCurrentClocksThrottleReasons")
        return f(self.h)

    def _run(self):
        while not self.stop:
            try:
                self.rows.append((self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM),
                                  self.nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0, self._reasons()))
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        import threading
        self.stop = False
        if self.h is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self.stop = True
        if self.h is not None:
            self.t.join()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = np.array([r[0] for r in self.rows], dtype=float)
        load = sm[sm > 0.5 * self.max] if (sm > 0.5 * self.max).any() else sm
        reasons = sorted({nm for r in self.rows for b, nm in self.BITS.items() if r[2] & b})
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": float(self.max), "reasons": reasons,
                "power_w_max": float(max(r[1] for r in self.rows)), "samples": len(self.rows),
                "source": "NVML, 10 ms"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def profiled_traffic(name):
    """Per-launch DRAM bytes of a kernel from its committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{name}.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


def time_steps(ctx, stream, steps, flush):
    """Sum of per-step device times (CUDA events on the launch stream); the
    L2 is flushed between steps, outside the timed intervals."""
    import torch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            ctx.rk4_step(DT, nsteps=1)
            b.record(stream)
    stream.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs) / 1e3


def make_arm(fss, state, area, stream, prec, args, dev, clusters=False):
    """Fixed degree/theta treecode; tree depth, source split and block shape
    chosen by the autotuner."""
    ctx = fss.Context(method=fss.METHOD_TREECODE, precision=prec, degree=args.degree, theta=args.theta,
                      cluster_targets=int(clusters), device=dev, autotune=2)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_particles(state, area)
    return ctx


def auto_tree_levels(n, leaf_target=64, max_levels=8):
    """The library's automatic depth: the smallest whose mean leaf holds at
    least leaf_target particles (fixed for the learned arm, whose network
    was trained on leaves of that size)."""
    ll = 0
    while ll + 1 < max_levels and n / (20.0 * 4 ** (ll + 1)) >= leaf_target:
        ll += 1
    return ll + 1


def make_learned_arm(fss, state, area, stream, args, dev, clusters=True):
    """Mixed precision with the learned per-leaf (degree, theta) (with target
    clusters: carried up to the faces of a dual traversal); block shape and
    source split chosen by the autotuner on the learned lists (the tree
    depth stays the automatic one, on which the selector's network was
    trained)."""
    from fss_b200 import selector
    ctx = fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, list_mode=fss.LIST_LEAF,
                      cluster_targets=int(clusters), degree=args.degree, theta=args.theta, device=dev, autotune=2,
                      tree_levels=auto_tree_levels(state.shape[0]))
    ctx.set_stream(stream.cuda_stream)
    ctx.set_particles(state, area)
    choice = selector.apply(ctx, tol=args.tol, safety=args.safety, device=dev)
    return ctx, np.bincount(choice, minlength=selector.NCLS).tolist()


def run_sweep(fss, state, area, stream, flush, dev, args, u_ref):
    """Mixed-precision BLTC (FP32 interactions, Kahan sums, FP64 RK4 and
    renormalisation; far sources summed at the target particles) at each
    fixed (degree, theta): relative L2 and max velocity error against the
    FP64 direct sum over all targets and over 4,096 seeded sample targets
    (seed 7), and RK4 steps/s timed like the headline arm.  One JSON line
    per setting."""
    import copy
    n = state.shape[0]
    rows = np.sort(np.random.default_rng(7).choice(n, min(4096, n), replace=False))

    def errs(u, v):
        return (float(np.linalg.norm(u - v) / np.linalg.norm(v)),
                float(np.max(np.linalg.norm(u - v, axis=1)) / np.max(np.linalg.norm(v, axis=1))))

    for degree in (6, 8, 10):
        for theta in (0.5, 0.7):
            a = copy.copy(args)
            a.degree, a.theta = degree, theta
            ctx = make_arm(fss, state, area, stream, fss.PREC_MIXED, a, dev)
            try:
                u = ctx.rhs(state, area)[:, :3]
                l2, mx = errs(u, u_ref)
                l2s, mxs = errs(u[rows], u_ref[rows])
                warm(ctx, stream, args.warmup)
                t = time_steps(ctx, stream, args.steps, flush)
                inter, _ = ctx.work_per_rhs()
                info = ctx.tree_info()
            finally:
                ctx.close()
            print(json.dumps({"sweep": "mixed-precision BLTC, fixed degree/theta", "level": args.level,
                              "n_particles": n, "degree": degree, "theta": theta,
                              "tree_levels": info["tree_levels"], "rel_l2": l2, "rel_max": mx,
                              "rel_l2_sample4096": l2s, "rel_max_sample4096": mxs,
                              "steps_per_s": args.steps / t, "ms_per_step": 1e3 * t / args.steps,
                              "interactions_per_rhs": inter, "interactions_per_s": 4 * inter * args.steps / t,
                              "reference": "FP64 direct sum on the GPU, all targets"}), flush=True)


def warm(ctx, stream, w):
    for _ in range(w):
        ctx.rk4_step(DT, nsteps=1)
    stream.synchronize()


def cpu_reference_sample(state, area, sample, seed=7):
    """Reference direct sum (its own BVE_gfunc/slice/vec_add, row-range
    partition of direct_sum_mpi.cpp) on `sample` seeded targets, all cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    use_ref = O.ref() is not None
    rows = np.sort(np.random.default_rng(seed).choice(state.shape[0], sample, replace=False))
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    O.rhs_direct_rows(state, area, rows, threads=threads, use_ref=use_ref)
    dt = time.perf_counter() - t0
    n = state.shape[0]
    t_rhs = dt * n / sample
    return {"value": 1.0 / (4.0 * t_rhs), "unit": UNIT, "cores": threads,
            "kind": "reference" if use_ref else "port",
            "sample": f"reference direct sum rhs_direct_sum/BVE_gfunc (oracle/_ref) on {sample} seeded targets x "
                      f"{n} sources, {threads} threads, {dt:.2f} s; scaled by N/sample to one RHS, x4 per RK4 step"}


def remesh_measure(fss, ctx, state, area, level, stream, reps=5):
    """The remesh step as the reference's time loop uses it (new_dynamics.cpp
    213-217: after every RK4 step the moved particles are regridded onto the
    grid with remesh.h regrid_points2).  From the grid state: one RK4 step,
    then fss_remesh (host buffers, the drop-in; host wall clock, copies
    included) and fss_remesh_current (device-resident), both checked bit for
    bit against the reference's own regrid_points2 on the same input
    (oracle/_ref, one thread, timed), and `reps` RK4 steps each followed by
    fss_remesh_current (steps/s with remeshing every step)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    _, tris = fss.icos_grid(level)
    ctx.set_particles(state, area)
    ctx.rk4_step(DT, nsteps=1)
    moved = ctx.get_state()
    target = moved.copy()
    target[:, :3] = state[:, :3]
    fss.remesh(moved, target, tris)              # warm
    t0 = time.perf_counter()
    got, fb, bad = fss.remesh(moved, target, tris)
    wall_ms = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    ctx.remesh_current(tris)
    cur_ms = 1e3 * (time.perf_counter() - t0)
    got_dev = ctx.get_state()
    stream.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        ctx.rk4_step(DT, nsteps=1)
        ctx.remesh_current()  # the triangles of the previous call
    stream.synchronize()
    loop_s = time.perf_counter() - t0
    out = {"workload": "one RK4 step from the grid, then regrid onto the grid (the reference's use_remesh loop)",
           "points": int(moved.shape[0]), "triangles": int(tris.shape[0]), "fallback": fb, "not_found": bad,
           "wall_ms_host_buffers": wall_ms, "h2d_d2h_bytes": int(2 * moved.nbytes + target.nbytes),
           "wall_ms_device_resident_first_call": cur_ms, "rk4_plus_remesh_steps_per_s": reps / loop_s}
    if O.ref() is not None:
        # the reference is O(triangles) per point outside its adjacent
        # triangles: time it on a contiguous row range from a seeded start,
        # doubled until it runs ~2 s, and scale by N / rows
        n = moved.shape[0]
        lb, k, el = int(np.random.default_rng(11).integers(0, n // 2)), 1, 0.0
        while True:
            t0 = time.perf_counter()
            ref, _, rc = O.remesh(moved, target, tris, use_ref=True, rows=(lb, min(n, lb + k)))
            el = time.perf_counter() - t0
            if el >= 2.0 or lb + k >= n or rc != 0:
                break
            k *= 2
        ub = min(n, lb + k)
        out["cpu_reference_ms"] = 1e3 * el * n / (ub - lb)
        out["cpu_reference"] = (f"remesh.h regrid_points2 (oracle/_ref), 1 thread, rows {lb}..{ub} "
                                f"({el:.2f} s), scaled by N/rows")
        out["bit_exact_vs_reference_rows"] = bool(
            rc == 0 and np.array_equal(got[lb:ub].view(np.uint64), ref[lb:ub].view(np.uint64))
            and np.array_equal(got_dev[lb:ub].view(np.uint64), ref[lb:ub].view(np.uint64)))
    return out


def cpu_reference_fast(fss, level=6):
    """The reference's own fast sum (rhs_eval.h:34 rhs_fast_sum, oracle/_ref)
    at its only working setting (degree 2, theta 0.7, many_count 10, 4 tree
    levels) on the level-`level` grid of the headline field.  Its set-up
    (icosahedron_init, interp_init, points_assign, tree_traverse: once per run
    in the reference's loop) and one evaluation (what rhs_func does per call)
    are timed apart, on one thread and split over the host cores the way
    fast_sum_mpi.cpp splits it over MPI ranks (top-level target faces per
    rank, at most 20); the relative L2 velocity error is against the FP64
    direct sum (the oracle, all host threads).  Level 8 is out of reach on the
    host in minutes (its pair traversal is quadratic in the queue)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if O.ref() is None:
        return None
    s, a = fss.make_state(level, "rh_vortices", n_vortex=32, seed=2)
    n = s.shape[0]
    threads = max(1, min(20, os.cpu_count() or 1))
    out1, outp, t = np.zeros(5 * n), np.zeros(5 * n), np.zeros(3)
    rc = O.ref().ref_rhs_fast_timed(n, s.reshape(-1), a, O.OMEGA, 4, 0.7, 10, 2, threads, out1, outp.ctypes.data, t)
    ref = O.rhs_direct(s, a)
    u = out1.reshape(n, 5)[:, :3]
    return {"kind": "reference", "function": "rhs_fast_sum (oracle/_ref)", "level": level, "n": int(n),
            "tree_levels": 4, "degree": 2, "theta": 0.7, "many_count": 10, "rc": int(rc),
            "setup_ms": 1e3 * float(t[0]), "ms_per_rhs_1_thread": 1e3 * float(t[1]),
            "threads": threads, "partition": "fast_sum_mpi.cpp top-level target faces per rank, ranks as threads",
            "ms_per_rhs": 1e3 * float(t[2]), "steps_per_s": 1.0 / (4 * float(t[2])),
            "threads_equal_1_thread": bool(np.array_equal(out1, outp)),
            "rel_l2": float(np.linalg.norm(u - ref[:, :3]) / np.linalg.norm(ref[:, :3]))}


def amr_measure(fss, level=5, reps=3):
    """amr.h amr as the reference's -a loop calls it, on the reference's
    Gaussian vortex (level-`level` grid, the reference's tolerances 0.2 and
    0.0025; max_count of level + 2): fss_amr_refine (host buffers, host wall
    clock with the copies, a fresh mesh per repetition), then
    fss_amr_remesh on the refined mesh rotated by 0.005 rad; beside it the
    reference's own amr() on the same input (oracle/_ref, one thread, timed)
    and a bit-for-bit comparison of points and triangles."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    state, area = fss.make_state(level, "gauss_ref")
    _, tris = fss.icos_grid(level)
    n = state.shape[0]
    mc = 10 * 4 ** (level + 2) + 2
    times = []
    for r in range(reps + 1):
        with fss.Amr(tris, n, mc, 4 * mc) as amr:
            t0 = time.perf_counter()
            st, ar = amr.refine(state, area)
            if r:
                times.append(1e3 * (time.perf_counter() - t0))
            if r == reps:
                t_new, _, _ = amr.mesh()
                grid = st.copy()
                grid[:, :3] /= np.linalg.norm(grid[:, :3], axis=1, keepdims=True)
                c, sn = np.cos(0.005), np.sin(0.005)
                moved = grid.copy()
                moved[:, :3] = grid[:, :3] @ np.array([[c, -sn, 0], [sn, c, 0], [0, 0, 1]]).T
                amr.remesh(moved, grid)  # builds the adjacency
                t0 = time.perf_counter()
                _, fb, nf = amr.remesh(moved, grid)
                rm_ms = 1e3 * (time.perf_counter() - t0)
    # the reference's -a loop on the device: RK4 step, then amr() on the
    # context's particles (new points projected, tree and lists rebuilt)
    loop_steps = 5
    with fss.Amr(tris, n, mc, 4 * mc) as amr2, \
            fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, autotune=0) as ctx2:
        ctx2.set_particles(state, area)
        t0 = time.perf_counter()
        for _ in range(loop_steps):
            ctx2.rk4_step(DT, nsteps=1)
            n_loop = ctx2.amr_refine_current(amr2)
        loop_s = time.perf_counter() - t0
    out = {"workload": f"amr() on the Gaussian vortex, level {level} grid, tolerances 0.2 / 0.0025",
           "rk4_plus_amr_steps_per_s": loop_steps / loop_s, "rk4_plus_amr_points_after": int(n_loop),
           "points_in": int(n), "points_out": int(st.shape[0]), "triangles_out": int(t_new.shape[0]),
           "wall_ms_host_buffers": float(np.median(times)),
           "remesh_after_amr_ms_host_buffers": rm_ms, "remesh_fallback": fb, "remesh_not_found": nf}
    if O.ref() is not None:
        t0 = time.perf_counter()
        R = O.ref_amr(state, area, tris, mc)
        out["cpu_reference_ms"] = 1e3 * (time.perf_counter() - t0)
        out["cpu_reference"] = "amr.h amr (oracle/_ref), 1 thread"
        out["bit_exact_vs_reference"] = bool(R["n"] == st.shape[0] and np.array_equal(R["tris"], t_new)
                                             and np.array_equal(R["state5"].view(np.uint64), st.view(np.uint64)))
    return out


def kernel_rooflines(prof, steps, n, up_bytes, peaks):
    """HBM roofline of the memory-bound ranges with the algorithmic byte
    units of the scope table: upward pass = N 16 B read per level + K (4 +
    12) B per proxy (per RHS, from fss_work_per_rhs); tree build (the
    per-step re-sort) = N (24 + 8 + 16) B + 2 N 12 B per radix pass executed
    (none: the re-sort partitions the old order instead of sorting); RK4
    combine = N (5 x 8 x (1 + 4) + 5 x 8 + 16) B per step.  The
    downward pass has no byte unit (FP64, latency-bound): time only.  Times
    from the kernel-level pass (events around every launch)."""
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    src = "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
    out = []

    def add(name, ms, nbytes, per):
        gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else None
        out.append({"kernel": name, "bound": "hbm", "bytes": nbytes, "per": per, "ms": ms, "achieved": gbs,
                    "peak": hbm, "unit": "GB/s", "frac": (gbs / hbm) if gbs else None, "peak_source": src})

    up_ms = sum(prof[k][0] for k in ("upward_leaf", "upward_combine") if k in prof) / (4 * steps)
    if up_ms > 0:
        add("upward pass (k_up_leaf, k_up_sums, k_up_proxies)", up_ms, float(up_bytes), "RHS")
    if "resort" in prof:
        add("tree build: per-step re-sort (k_part_keys, k_part_scan, k_part_bucket, k_part_place, "
            "k_resort_commit)", prof["resort"][0] / steps, float(n) * (24 + 8 + 16), "step")
    if "epilogue" in prof:
        add("RK4 combine (k_epilogue, 4 per step)", prof["epilogue"][0] / steps,
            float(n) * (5 * 8 * 5 + 5 * 8 + 16), "step")
    if "downward" in prof:
        out.append({"kernel": "downward pass (k_down_coef, k_down_direct)", "bound": "latency",
                    "ms": prof["downward"][0] / (4 * steps), "per": "RHS"})
    return out


def main_reference(args, ws, rank):
    """The reference's own CPU implementation of the path, timed on this
    host's cores.  Its fast sum (rhs_fast_sum) cannot be set up at 655,362
    particles in minutes (its pair traversal is quadratic in the queue) and
    never reaches 1e-6, so the arm times its FP64 direct sum (rhs_direct_sum /
    BVE_gfunc, oracle/_ref) on a bounded sample per step: `cpu_sample` seeded
    target rows against all sources, scaled by N / rows to one RHS, x4 per RK4
    step.  The inputs are built by the oracle alone (icos_init, area_init and
    the seeded field), so the product library is never loaded here."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    state, area = O.rh_vortices_state(args.level, args.vortices, args.seed)
    n = state.shape[0]
    for _ in range(args.warmup):
        cpu_reference_sample(state, area, max(64, args.cpu_sample // 8))
    secs_extrapolated, timed = 0.0, 0.0
    cb = None
    for k in range(args.steps):
        t0 = time.perf_counter()
        cb = cpu_reference_sample(state, area, args.cpu_sample, seed=100 + k)
        timed += time.perf_counter() - t0
        secs_extrapolated += 1.0 / cb["value"]
    value = args.steps / secs_extrapolated
    cb["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "extrapolated": True,
            "samples": {"count": args.steps, "targets_per_sample": args.cpu_sample, "sources": int(n),
                        "timed_s": timed, "s_per_rhs_extrapolated": secs_extrapolated / (4 * args.steps),
                        "note": f"each 'step' is one sample of {args.cpu_sample} targets x {n} sources; "
                                f"ms_per_step is that sample scaled by N/rows x 4 RHS, not a step that ran"},
            "config": {"workload": f"BVE RHS RK4 step, {n} particles (icosahedral level {args.level}), "
                                   f"RH4 + {args.vortices} vortices; reference FP64 direct sum on host cores",
                       "n_particles": int(n),
                       "same_algorithm": False,
                       "why_direct": "the reference's treecode cannot be set up at this N in minutes and its "
                                     "degree-2 interpolation stays near 2e-1 rel-L2"},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_arm(ctx, stream, flush, args, ws):
    """(steps/s over all ranks, ms per step of the slowest rank) of an arm."""
    warm(ctx, stream, args.warmup)
    t = max_over_ranks(time_steps(ctx, stream, args.steps, flush), ws)
    return ws * args.steps / t, 1e3 * t / args.steps


def e2e_rhs_func(ctx, state, area, steps):
    """The reference's own call pattern (new_dynamics.cpp:170-229): per RK4
    step four fss_rhs calls with host buffers (state in, modify out) and the
    stage states combined and projected on the host, as rhs_func's caller
    does.  Host wall clock per step, after a synchronisation."""
    s = state.copy()
    dt, om = DT, 2 * np.pi

    def project(x, old_z):
        x[:, :3] /= np.linalg.norm(x[:, :3], axis=1, keepdims=True)
        x[:, 3] += -2 * om * (x[:, 2] - old_z)
        return x

    def step(s):
        k1 = ctx.rhs(s, area)
        i1 = s + dt / 2 * k1
        k2 = ctx.rhs(project(i1, i1[:, 2].copy()), area)
        i2 = s + dt / 2 * k2
        k3 = ctx.rhs(project(i2, i2[:, 2].copy()), area)
        i3 = s + dt * k3
        k4 = ctx.rhs(project(i3, i3[:, 2].copy()), area)
        out = s + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        return project(out, out[:, 2].copy())

    s = step(s)  # warm
    t0 = time.perf_counter()
    for _ in range(steps):
        s = step(s)
    wall = time.perf_counter() - t0
    return {"value": steps / wall, "unit": UNIT, "calls_per_step": 4,
            "h2d_bytes_per_step": int(4 * (state.nbytes + area.nbytes)), "d2h_bytes_per_step": int(4 * state.nbytes),
            "how": "four fss_rhs calls per RK4 step with host buffers (the reference's rhs_func call pattern, "
                   "new_dynamics.cpp:170-229), stage combine and projection on the host in NumPy; host wall clock"}


def ensemble_measure(fss, args, dev, stream, members=64, steps=20, seed=100):
    """The ensemble configuration: `members` problems on icosahedral levels
    drawn uniformly from 5-8 (10,242 - 655,362 particles each), each an RH R=4
    wave with a seeded +-5% amplitude perturbation and 4-16 Gaussian vortices;
    mixed-precision BLTC n = 8, theta = 0.7; one persistent pair launch per RK
    stage over the global (member, target leaf, source run) queue, one CUDA
    graph per RK4 step.  Device time of `steps` steps (CUDA events, L2 not
    flushed: the ensemble's working set is far larger than L2); the persistent
    launch timed alone for its FP32 fraction; member 0 against its own run."""
    rng = np.random.default_rng(seed)
    fields, levels = [], []
    for m in range(members):
        level = int(rng.integers(5, 9))
        nv = int(rng.integers(4, 17))
        amp = float(rng.uniform(0.95, 1.05))
        fields.append(fss.make_state(level, "rh_vortices", n_vortex=nv, seed=seed + m, amp=fss.RH_AMP * amp))
        levels.append(level)
    import torch
    t0 = time.perf_counter()
    with fss.Ensemble(degree=8, theta=0.7, device=dev) as ens:
        ens.set_stream(stream.cuda_stream)
        for s, a in fields:
            ens.add(s, a)
        ens.build()
        build_s = time.perf_counter() - t0
        info = ens.info()
        ens.rk4_step(DT, nsteps=1)  # capture + warm
        stream.synchronize()
        a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a_ev.record(stream)
            ens.rk4_step(DT, nsteps=steps)
            b_ev.record(stream)
        stream.synchronize()
        secs = a_ev.elapsed_time(b_ev) / 1e3
        pair_ms = ens.time_pairs(3)
        got0 = ens.get_state(0)
    s0, a0 = fields[0]
    with fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, degree=8, theta=0.7,
                     block_threads=160, src_parts=1, device=dev) as ctx:
        ctx.set_particles(s0, a0)
        ctx.rk4_step(DT, nsteps=1 + steps)
        ref0 = ctx.get_state()
    disp = ref0[:, :3] - s0[:, :3]
    inter = info["interactions_per_rhs"]
    peaks = load_peaks()
    fp32_peak = 148 * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    pair_tflops = FLOPS_PER_PAIR * inter / (pair_ms * 1e-3) / 1e12
    return {"workload": f"{members} members, icosahedral levels 5-8 drawn uniformly (seed {seed}), RH4 +-5% + 4-16 "
                        f"vortices, mixed-precision BLTC n=8 theta=0.7, {steps} RK4 steps",
            "members": members, "levels_5_6_7_8": np.bincount(levels, minlength=9)[5:].tolist(),
            "particles": info["particles"], "work_items": info["work_items"], "interactions_per_rhs": inter,
            "steps": steps, "device_s": secs, "steps_per_s": steps / secs,
            "interactions_per_s": 4 * steps * inter / secs, "build_s": build_s,
            "pair_launch_ms": pair_ms, "pair_launch_tflops": pair_tflops, "pair_launch_fp32_frac": pair_tflops / fp32_peak,
            "member0_vs_alone_rel_l2": float(np.linalg.norm(got0[:, :3] - ref0[:, :3]) / np.linalg.norm(disp)),
            "member0_bit_exact_vs_alone": bool(np.array_equal(got0, ref0))}


def main_shard(args, ws, rank, dev):
    """The headline arm split over the ranks: every rank builds the same tree
    and evaluates its own targets; per RK stage one all-reduce (sum) of the
    N x 4 float64 exchange buffer over NCCL.  Device time of K steps (CUDA
    events, L2 flushed between steps), max over ranks; value = steps / that
    time (strong scaling: the total work is fixed)."""
    import torch
    import fss_b200 as fss
    from fss_b200 import shard
    state, area = fss.make_state(args.level, "rh_vortices", n_vortex=args.vortices, seed=args.seed)
    n = state.shape[0]
    stream = torch.cuda.Stream(device=dev)   # every launch, the all-reduce and the events on it
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")
    from fss_b200 import selector as _sel
    ctx = fss.Context(method=fss.METHOD_TREECODE, precision=fss.PREC_MIXED, list_mode=fss.LIST_LEAF,
                      cluster_targets=1, degree=args.degree, theta=args.theta, device=dev, autotune=1)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_particles(state, area)
    _sel.apply(ctx, tol=args.tol, safety=args.safety, device=dev)
    ctx.shard(rank, ws)
    info = ctx.shard_info()
    ex = shard.exchange_buffer(ctx, f"cuda:{dev}")
    red = shard.torch_allreduce() if ws > 1 else None
    torch.cuda.synchronize()
    shard.rk4_steps(ctx, ex, DT, nsteps=args.warmup, allreduce=red)
    torch.cuda.synchronize()
    barrier(ws)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            shard.rk4_steps(ctx, ex, DT, nsteps=1, allreduce=red)
            b.record(stream)
    torch.cuda.synchronize()
    t = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs) / 1e3, ws)
    state_out = ctx.get_state()
    ctx.close()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": args.steps / t, "unit": UNIT, "n_gpus": ws,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
                          "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic",
                          "config": {"workload": f"BVE RK4 step, {n} particles (level {args.level}), learned "
                                                 f"mixed BLTC with target clusters, one problem split over {ws} "
                                                 f"ranks", "parallelism": f"sharded x{ws}",
                                     "exchange_bytes_per_stage": int(ex.numel() * 8),
                                     "unit_level": info["unit_level"], "units": info["units"],
                                     "rank0_cost_share": info["cost_own"] / max(info["cost_total"], 1.0)},
                          "finite": bool(np.all(np.isfinite(state_out)))}), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.shard and args.impl != "reference":
        import torch
        torch.cuda.set_device(local)
        main_shard(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        main_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    import fss_b200 as fss
    torch.cuda.set_device(local)
    dev = local
    state, area = fss.make_state(args.level, "rh_vortices", n_vortex=args.vortices, seed=args.seed)
    n = state.shape[0]
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")  # 256 MB > L2

    # accuracy reference: the FP64 direct sum on the GPU (checked against the
    # CPU oracle on 4,096 seeded targets at this size in tests/test_gpu_fullsize.py)
    with fss.Context(method=fss.METHOD_DIRECT, precision=fss.PREC_FP64, device=dev) as dctx:
        dctx.set_stream(stream.cuda_stream)
        dctx.set_particles(state, area)
        u_ref = dctx.rhs(state, area)[:, :3]

    if args.sweep:
        if rank == 0:
            run_sweep(fss, state, area, stream, flush, dev, args, u_ref)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    def rel_err(ctx):
        u = ctx.rhs(state, area)[:, :3]
        return float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)), float(
            np.max(np.linalg.norm(u - u_ref, axis=1)) / np.max(np.linalg.norm(u_ref, axis=1)))

    # ---------------- headline arm: mixed precision BLTC
    from fss_b200 import selector as _sel
    clusters = not args.no_clusters
    learned = (not args.fixed) and os.path.exists(_sel.default_weights(clusters))
    classes = None
    if learned:
        ctx, classes = make_learned_arm(fss, state, area, stream, args, dev, clusters)
    else:
        ctx = make_arm(fss, state, area, stream, fss.PREC_MIXED, args, dev, clusters)
    err_l2, err_max = rel_err(ctx)
    warm(ctx, stream, args.warmup)
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        t = time_steps(ctx, stream, args.steps, flush)
    torch.cuda.synchronize()
    barrier(ws)
    t_max = max_over_ranks(t, ws)
    value = replica_value(args.steps, t, ws)
    clocks = clk.summary()

    # kernel-level pass (events around every launch, no graph): shares and roofline
    ctx.profile(True)
    ctx.rk4_step(DT, nsteps=args.steps)
    prof = ctx.profile_read()
    ctx.profile(False)
    inter, up_bytes = ctx.work_per_rhs()
    pk = "pairs_mixed"
    pairs_ms = prof[pk][0] / (4 * args.steps)  # per RHS (target-leaf and target-cluster launches)
    launches_per_step = sum(v[1] for v in prof.values()) / args.steps
    total_ms = sum(v[0] for v in prof.values())
    peaks = load_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s, nominal at max SM clock
    achieved = FLOPS_PER_PAIR * inter / (pairs_ms * 1e-3) / 1e12
    traffic = profiled_traffic("pairs_mixed_level8")
    info = ctx.tree_info()
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": traffic,
                "kernel": "k_pairs (target-leaf + target-cluster launches of one RHS)", "kernel_ms": pairs_ms,
                "interactions_per_launch": inter, "flops_per_interaction": FLOPS_PER_PAIR,
                "peak_source": f"nominal FP32 148 SM x 128 lanes x 2 x {sm_max:.0f} MHz (MEASURED_PEAKS.json has no FP32 figure)"}
    roofline_detail = {"frac_at_sampled_clock": (achieved / (fp32_peak * clocks["sm_mhz"] / sm_max)) if clocks.get("sm_mhz") else None,
                       "kernel_shares": {k: round(v[0] / total_ms, 4) for k, v in prof.items()},
                       "upward_bytes_per_rhs": up_bytes,
                       "kernels": kernel_rooflines(prof, args.steps, n, up_bytes, peaks)}

    # ---------------- the other arms on the same GPU: the plain FP64 BLTC (the
    # ratio's denominator: fixed n, theta, far sources summed at the target
    # particles), the FP64 treecode with the headline's algorithm (target
    # clusters), and the mixed-precision treecode with target clusters at
    # fixed n = 8, theta = 0.7 (what the learned choice alone adds)
    fp64 = fp64c = fixc = None
    arms = []
    if not args.no_fp64:
        arms += [("fp64_plain", fss.PREC_FP64, False), ("fp64_same_algorithm", fss.PREC_FP64, True)]
    if learned:
        arms += [("mixed_fixed_clusters", fss.PREC_MIXED, clusters)]
    res = {}
    for name, prec, cl in arms:
        c2 = make_arm(fss, state, area, stream, prec, args, dev, clusters=cl)
        e2 = rel_err(c2)
        v2, ms2 = time_arm(c2, stream, flush, args, ws)
        ti = c2.tree_info()
        res[name] = {"value": v2, "ms_per_step": ms2, "rel_l2": e2[0], "rel_max": e2[1], "degree": args.degree,
                     "theta": args.theta, "target_clusters": cl, "precision": "fp64" if prec == fss.PREC_FP64 else "mixed",
                     "tuned": {"tree_levels": ti["tree_levels"], "src_parts": ti["src_parts"],
                               "block_threads": ti["block_threads"]}}
        c2.close()
    fp64, fp64c, fixc = res.get("fp64_plain"), res.get("fp64_same_algorithm"), res.get("mixed_fixed_clusters")

    # ---------------- end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.from_numpy(state.copy()).pin_memory()
        ptr = host.data_ptr()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for _ in range(args.warmup):
            ctx.rk4_step_host_ptr(ptr, DT, nsteps=1)
        with torch.cuda.stream(stream):
            for a, b in evs:
                flush.zero_()
                a.record(stream)
                ctx.rk4_step_host_ptr(ptr, DT, nsteps=1)  # H2D state, 4 stages, D2H state
                b.record(stream)
        stream.synchronize()
        te = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs) / 1e3, ws)
        e2e = {"value": ws * args.steps / te, "unit": UNIT, "h2d_bytes_per_step": int(state.nbytes),
               "d2h_bytes_per_step": int(state.nbytes)}

    e2e_rf = None
    if rank == 0 and ws == 1 and not args.no_e2e:
        e2e_rf = e2e_rhs_func(ctx, state, area, max(3, args.steps // 4))

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_reference_sample(state, area, args.cpu_sample)

    # the remesh step: one RK4 step from the grid, regridded back onto it
    remesh = None
    if rank == 0 and ws == 1 and not args.no_remesh:
        try:
            remesh = remesh_measure(fss, ctx, state, area, args.level, stream)
        except fss.FssError as e:  # too many points left their triangles in one step
            remesh = {"error": str(e)}
    ctx.close()

    cpu_fast = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            cpu_fast = cpu_reference_fast(fss)
        except Exception as e:  # a reported baseline only: its failure must not cost the line
            cpu_fast = {"error": f"{type(e).__name__}: {e}"}

    amr = None
    if rank == 0 and ws == 1 and not args.no_amr:
        amr = amr_measure(fss)

    ens = None
    if rank == 0 and ws == 1 and not args.no_ensemble:
        try:
            ens = ensemble_measure(fss, args, dev, stream, members=args.members)
        except fss.FssError as e:
            ens = {"error": str(e)}

    if rank == 0:
        workload = (f"BVE RK4 step (4 RHS), {n} particles (icosahedral level {args.level}), RH4 wave + "
                    f"{args.vortices} seeded vortices, mixed-precision BLTC "
                    f"({'learned per-leaf degree/theta' if learned else f'n={args.degree} theta={args.theta}'}"
                    f"{', target clusters' if clusters else ''}), particles re-sorted every step")
        # everything bulky first, on a line of its own ...
        detail = {"detail": "bench details (the headline is the next line)", "metric": METRIC,
                  "selector": (f"learned per-leaf (n, theta), tol {args.tol}, safety {args.safety}, "
                               f"classes (n, theta) {list(zip(*_sel.class_table(clusters)))}, "
                               f"class counts {classes}") if learned else "none (fixed degree/theta)",
                  "tree": info, "roofline_detail": roofline_detail, "arms": res,
                  "e2e_rhs_func": e2e_rf, "cpu_baseline": cpu, "cpu_reference_fast": cpu_fast,
                  "remesh": remesh, "amr": amr, "ensemble": ens}
        print(json.dumps(detail), flush=True)
        # ... then the headline, short and last
        short = lambda r: None if r is None else {k: r[k] for k in ("value", "ms_per_step", "rel_l2", "rel_max")}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "rel_l2": err_l2, "rel_max": err_max, "tol": args.tol,
                "ratio_vs_fp64_plain": (value / fp64["value"]) if fp64 else None,
                "fp64_plain": short(fp64),
                "ratio_vs_fp64_same_algorithm": (value / fp64c["value"]) if fp64c else None,
                "ratio_learned_vs_fixed_clusters": (value / fixc["value"]) if fixc else None,
                "mixed_fixed_clusters": short(fixc),
                "config": {"workload": workload, "n_particles": n, "tree_levels": info["tree_levels"],
                           "error_reference": "FP64 direct sum on the GPU, all targets",
                           "l2": "flushed between timed steps (256 MB write)",
                           "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
                "e2e": e2e,
                "e2e_rhs_func": None if e2e_rf is None else {"value": e2e_rf["value"], "unit": UNIT},
                "roofline": roofline,
                "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind")},
                "ensemble_steps_per_s": None if not ens or "error" in ens else ens["steps_per_s"],
                "interactions_per_s": inter * 4 * value,
                "gpu_launches": int(round(launches_per_step * args.steps)),
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

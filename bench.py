#!/usr/bin/env python
"""Benchmark: Krylov time to 1e-10 relative residual on the 128^3 7-point
Laplacian (n = 2,097,152, nnz = 14,581,760, CSR int32 / float64), PCG with
IC(0), x_true ~ U[-1,1] (seed 1), b = A x_true, x0 = 0.

One step = one complete mixed-precision refined PCG-IC(0) solve (FP32 inner
PCG with FP32 factors, FP64 residual / update / stopping norm) to true
relative residual <= 1e-10, inputs resident in HBM.  Also measured in the
same run: the plain FP64 GPU solve (for the mixed-vs-FP64 comparison), the
FP64 SpMV's fraction of the measured HBM peak, the dominant kernel's
roofline, the same solve end to end through the C ABI with host buffers,
and the reference's own CPU path (MTL4 compiled from its headers) on the
host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: replicas only (the triangular sweeps of IC(0) carry a global
dependency chain, so a single solve does not shard without changing the
preconditioner); each rank solves its own copy, value = max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mtl4-mirror_b200", "python"))

N_GRID = 128
METRIC = "Krylov time to 1e-10 rel residual (mixed vs FP64 GPU); SpMV % HBM peak"
WORKLOAD = "3-D 7-point Laplacian 128^3, PCG + IC(0), FP32 inner / FP64 refinement, rtol 1e-10"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic():
    """Per-launch DRAM bytes of kernels from the committed ncu summary
    (profiles/traffic.txt: '<key> <bytes per launch> ...' lines)."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        ok = [s for s in self.samples if len(s) >= 8]
        sm = [float(s[0]) for s in ok if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in ok if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in ok for k in range(4) if s[4 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def problem(M):
    A = M.laplacian3d(N_GRID)
    xt = M.uniform(A[0], 1)
    b = M.csr_mult(A, xt)
    return A, b


def reference_solver():
    """The reference's own CPU path: MTL4 compiled from its headers
    (oracle/_ref, OpenMP build, all host threads); the C restatement of it
    when that build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ref = oracle.available_reference(openmp=True)
    if ref is not None:
        return ref, "reference", ref.threads()
    return oracle.Restatement(), "port", 1


def time_reference_solve(ref, kind, A, b):
    t0 = time.perf_counter()
    r = ref.solve("cg", "ic0", A, b, rtol=1e-10, max_iter=2000)
    wall = time.perf_counter() - t0
    # the reference driver times the itl::cg call alone (factorisation apart)
    return (r["t_solve"] if kind == "reference" else wall), r["iterations"], r["t_factor"]


def run_reference_arm(args, rank):
    import mtlgpu as M
    if rank != 0:
        return
    A, b = problem(M)
    steps = max(1, args.steps)
    warm = max(0, min(args.warmup, 1))   # one warm-up solve: each step is seconds of CPU work
    ref, kind, cores = reference_solver()
    for _ in range(warm):
        time_reference_solve(ref, kind, A, b)
    ts, iters = [], None
    for _ in range(steps):
        t, iters, _ = time_reference_solve(ref, kind, A, b)
        ts.append(t)
    ms = 1e3 * sum(ts) / len(ts)
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "3-D 7-point Laplacian 128^3, itl::cg + itl::pc::ic_0 (FP64, the "
                               "reference's CPU path), rtol 1e-10", "n": A[0], "nnz": len(A[2])},
        "iterations": iters,
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": cores, "kind": kind,
                         "sample": f"full solve to 1e-10 ({iters} iterations) per step; "
                                   "ic_0 factorisation outside the timed call"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class Replicas:
    """Plumbing of the N-GPU run: one process per GPU, each solving its own
    replica of the workload (the single-system solve does not shard: see the
    design notes), a barrier around every timed region, and the slowest rank's
    time as the job's time.  `dist` is torch.distributed (or None for one
    process); `device` holds the all-reduce buffer (cuda:<local> with NCCL,
    cpu with gloo)."""

    def __init__(self, dist, device):
        self.dist, self.device = dist, device

    @property
    def rank(self):
        return self.dist.get_rank() if self.dist is not None else 0

    @property
    def world(self):
        return self.dist.get_world_size() if self.dist is not None else 1

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, v):
        if self.dist is None:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def aggregate(self, per_rank_units, ms):
        """Whole-job throughput: all ranks' units over the slowest rank's time."""
        return per_rank_units * self.world / (self.max_over_ranks(ms) / 1e3)

    def emit(self, line):
        """Only rank 0 prints the JSON line."""
        if self.rank == 0:
            print(json.dumps(line), flush=True)
            return True
        return False


def _local_ms(fn, reps, stream):
    """Mean ms of fn over reps with CUDA events on `stream` (one GPU)."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = [fn() for _ in range(reps)]
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, out


def batched_workload(M, ctx, stream):
    """512 independent random-graph Laplacians (n log-uniform in [1e3, 65536],
    average degree U[8, 32], shift 1e-2 mean degree, seed 3), b ~ N(0,1):
    one batched PCG to 1e-8 with Jacobi and IC(0), in FP64 and with FP32 inner
    solves refined in FP64."""
    systems, (n, rp, ci, v, off) = M.graph_batch(512, 1000, 65536, 8.0, 32.0, 1e-2, seed=3)
    b = M.normal(n, 3)
    dA = M.Csr(ctx, rp, ci, v)
    db, dx, dz = ctx.to_device(b), ctx.array(n), ctx.to_device(np.zeros(n))
    out = {"systems": 512, "n": int(n), "nnz": int(len(ci)), "rtol": 1e-8, "dtype": "f64"}
    for pc in ("diagonal", "ic0"):
        P = M.Pc(dA, pc)

        def run():
            ctx.xpay(dz, 0.0, dx)
            st, res = M.solve_batched(dA, P, off, dx, db, rtol=1e-8, max_iter=5000)
            assert st == M.OK, st
            return res
        run()
        ms, res = _local_ms(run, 2, stream)
        its = np.array([r.iterations for r in res[-1]])
        rel = max(r.true_resid / r.norm_r0 for r in res[-1])
        out[pc] = {"ms": ms, "iterations_max": int(its.max()),
                   "iterations_mean": float(its.mean()), "max_true_rel_residual": rel}
        P.close()
        # FP32 inner solves with FP64 refinement per system
        P = M.Pc(dA, pc, M.FP32)

        def run32():
            ctx.xpay(dz, 0.0, dx)
            st, res = M.solve_batched(dA, P, off, dx, db, rtol=1e-8, max_iter=5000,
                                      mode=M.SOLVE_MIXED)
            assert st == M.OK, st
            return res
        run32()
        ms, res = _local_ms(run32, 2, stream)
        its = np.array([r.iterations for r in res[-1]])
        rel = max(r.true_resid / r.norm_r0 for r in res[-1])
        out[pc + "_fp32_refined"] = {
            "ms": ms, "inner_iterations_max": int(its.max()),
            "outer_max": int(max(r.outer_iterations for r in res[-1])),
            "max_true_rel_residual": rel}
        P.close()
    dA.close()
    return out


def adjoint_workload(M, ctx, stream):
    """Differentiable solve on the 512 x 512 finite-volume operator (log-normal
    kappa, sigma 1, 8-cell correlation, seed 4): forward PCG-IC(0) solve,
    adjoint PCG-IC(0) solve with dL/dx = x - x_target, and the gradient on A's
    pattern, FP64 to 1e-10."""
    N = 512
    A = M.fv2d(N, 1.0, 8.0, 4)
    n, rp, ci, v = A
    c = (np.arange(N) + 0.5) / N - 0.5
    X, Y = np.meshgrid(c, c, indexing="ij")
    b = np.exp(-(X ** 2 + Y ** 2) / (2 * 0.1 ** 2)).ravel()
    dA = M.Csr(ctx, rp, ci, v)
    P = M.Pc(dA, "ic0")
    db, dx, dz = ctx.to_device(b), ctx.array(n), ctx.to_device(np.zeros(n))

    def forward():
        ctx.xpay(dz, 0.0, dx)
        st, res, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=20000)
        assert st == M.OK, st
        return res
    forward()
    x = dx.download()
    dg = ctx.to_device(0.01 * M.normal(n, 44) * -1.0)   # x - x_target = -0.01 N(0,1)
    dlam, grad = ctx.array(n), ctx.array(len(ci))

    def backward():
        ctx.xpay(dz, 0.0, dlam)
        st, res, _ = M.solve("cg", dA, P, dlam, dg, rtol=1e-10, max_iter=20000)
        assert st == M.OK, st
        dA.values_grad(dlam, dx, grad)
        return res
    backward()
    ms_f, rf = _local_ms(forward, 2, stream)
    ms_b, rb = _local_ms(backward, 2, stream)
    out = {"n": int(n), "nnz": int(len(ci)), "forward_ms": ms_f, "backward_ms": ms_b,
           "forward_iterations": rf[-1].iterations, "backward_iterations": rb[-1].iterations,
           "dtype": "f64", "rtol": 1e-10}
    P.close()
    dA.close()
    return out


def profile_case(case, grid, launches):
    """Runs one kernel of the path a few times on an N^3 Laplacian (for
    profiler captures): 'spmv' (FP64 y = A x), 'sweep64' / 'sweep32' (IC(0)
    lower sweep in FP64 / FP32)."""
    import mtlgpu as M
    A = M.laplacian3d(grid)
    n = A[0]
    ctx = M.Context(0)
    dA = M.Csr(ctx, *A[1:])
    if case == "spmv":
        dx, dy = ctx.to_device(M.uniform(n, 5)), ctx.array(n)
        for _ in range(launches):
            dA.spmv(dx, dy)
    else:
        prec = M.FP32 if case == "sweep32" else M.FP64
        dt = np.float32 if prec == M.FP32 else np.float64
        P = M.Pc(dA, "ic0", prec)
        r, z = ctx.to_device(np.ones(n, dt)), ctx.array(n, dt)
        for _ in range(launches):
            P.sweep(M.LOWER, r, z)
    ctx.synchronize()
    print(json.dumps({"profile_case": case, "grid": grid, "launches": launches}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mtlgpu", choices=["mtlgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and differentiable-solve measurements")
    ap.add_argument("--profile-case", choices=["spmv", "sweep64", "sweep32"])
    ap.add_argument("--grid", type=int, default=64)
    ap.add_argument("--launches", type=int, default=3)
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case, args.grid, args.launches)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch
    import mtlgpu as M

    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    reps = Replicas(dist, f"cuda:{local}")
    barrier = reps.barrier
    max_over_ranks = reps.max_over_ranks

    t_setup = time.perf_counter()
    A, b = problem(M)
    n, nnz = A[0], len(A[2])
    ctx = M.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    dA = M.Csr(ctx, *A[1:])
    t0 = time.perf_counter()
    P64 = M.Pc(dA, "ic0", M.FP64)
    ctx.synchronize()
    t_fac64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    P32 = M.Pc(dA, "ic0", M.FP32)
    ctx.synchronize()
    t_fac32 = time.perf_counter() - t0
    db = ctx.to_device(b)
    dx = ctx.array(n)
    dzero = ctx.to_device(np.zeros(n))
    setup_s = time.perf_counter() - t_setup

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        """Mean ms of fn over reps, CUDA events on the library's stream."""
        ctx.synchronize()
        barrier()
        e0, e1 = ev(), ev()
        e0.record(stream)
        out = [fn() for _ in range(reps)]
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1) / reps, out

    mixed_kw = dict(rtol=1e-10, max_iter=4000, mode=M.SOLVE_MIXED, inner_rtol=1e-6)
    fp64_kw = dict(rtol=1e-10, max_iter=2000)

    def solve_mixed():
        ctx.xpay(dzero, 0.0, dx)                # x0 = 0 on the device
        st, res, _ = M.solve("cg", dA, P32, dx, db, **mixed_kw)
        assert st == M.OK, st
        return res

    def solve_fp64():
        ctx.xpay(dzero, 0.0, dx)
        st, res, _ = M.solve("cg", dA, P64, dx, db, **fp64_kw)
        assert st == M.OK, st
        return res

    warm = max(3, args.warmup)
    for _ in range(warm):
        solve_mixed()
        solve_fp64()

    clocks = ClockSampler(local)
    clocks.start()
    steps = args.steps
    ms_mixed, res_mixed = timed(solve_mixed, steps)
    x_mixed = dx.download()
    ms_fp64, res_fp64 = timed(solve_fp64, steps)
    clk = clocks.stop()
    ms_mixed = max_over_ranks(ms_mixed)
    ms_fp64 = max_over_ranks(ms_fp64)
    true_rel = float(np.linalg.norm(b - M.csr_mult(A, x_mixed)) / np.linalg.norm(b))
    launches = int(sum(r.kernel_launches for r in res_mixed))

    # FP64 SpMV alone (matrix 175 MB > L2; y = A x)
    dy = ctx.array(n)
    dx.upload(M.uniform(n, 5))
    for _ in range(5):
        dA.spmv(dx, dy)
    ms_spmv, _ = timed(lambda: dA.spmv(dx, dy), 100)
    bytes_spmv = nnz * 12 + 4 * (n + 1) + 2 * n * 8
    peak, peak_kind = peaks()
    spmv_gbs = bytes_spmv / ms_spmv / 1e6

    # dominant kernel: the triangular sweep (FP32 in the mixed path).  Each
    # timed call also refills its output with the NaN-box sentinel (one
    # extra n*w write, a separate small kernel); achieved counts the
    # algorithmic bytes of the sweep only.
    L32 = P32.factor_info(M.LOWER)[0]
    r32 = ctx.to_device(np.ones(n, np.float32))
    z32 = ctx.array(n, np.float32)
    for _ in range(3):
        P32.sweep(M.LOWER, r32, z32)
    ms_sweep32, _ = timed(lambda: P32.sweep(M.LOWER, r32, z32), 20)
    bytes_sweep32 = L32 * (4 + 4) + 4 * (n + 1) + 2 * n * 4
    L64 = P64.factor_info(M.LOWER)[0]
    r64 = ctx.to_device(np.ones(n))
    z64 = ctx.array(n)
    ms_sweep64, _ = timed(lambda: P64.sweep(M.LOWER, r64, z64), 20)
    bytes_sweep64 = L64 * 12 + 4 * (n + 1) + 2 * n * 8
    traffic = read_traffic()

    # end to end through the C ABI with pinned host buffers, H2D/D2H inside
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.zeros(n, dtype=torch.float64).pin_memory()

    def e2e_step():
        hx.zero_()
        st, res = M.solve_host_ptrs("cg", dA, P32, hx.data_ptr(), hb.data_ptr(), **mixed_kw)
        assert st == M.OK, st
        return res

    e2e_step()
    ms_e2e, _ = timed(e2e_step, steps)
    ms_e2e = max_over_ranks(ms_e2e)

    line = {
        "metric": METRIC,
        "value": ms_mixed,
        "unit": "ms",
        "n_gpus": world,
        "steps": steps,
        "warmup": warm,
        "ms_per_step": ms_mixed,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "nnz": nnz, "index": "int32",
                   "l2": "inputs larger than L2 (matrix 175 MB + factors 2 x 100 MB)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "iterations": {"mixed_inner": res_mixed[-1].iterations,
                       "mixed_outer": res_mixed[-1].outer_iterations,
                       "fp64": res_fp64[-1].iterations},
        "true_rel_residual": true_rel,
        "fp64_ms": ms_fp64,
        "mixed_speedup_vs_fp64": ms_fp64 / ms_mixed,
        "spmv": {"ms": ms_spmv, "GBps": spmv_gbs, "hbm_frac": spmv_gbs / peak,
                 "bytes": bytes_spmv, "peak_kind": peak_kind},
        "roofline": {"kernel": "sweep_kernel<float,4> (IC(0) lower sweep, FP32)",
                     "bound": "hbm", "achieved": bytes_sweep32 / ms_sweep32 / 1e6,
                     "peak": peak, "unit": "GB/s",
                     "frac": bytes_sweep32 / ms_sweep32 / 1e6 / peak,
                     "traffic": traffic.get("sweep_f32_lower"),
                     "algorithmic_bytes": bytes_sweep32, "ms": ms_sweep32,
                     "peak_kind": peak_kind},
        "sweep_fp64": {"ms": ms_sweep64, "GBps": bytes_sweep64 / ms_sweep64 / 1e6,
                       "bytes": bytes_sweep64},
        "setup_s": {"total": setup_s, "ic0_fp64": t_fac64, "ic0_fp32": t_fac32},
        "e2e": {"value": ms_e2e, "unit": "ms", "h2d_bytes_per_step": 2 * n * 8,
                "d2h_bytes_per_step": n * 8},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if world == 1 and not args.no_extras:
        line["batched"] = batched_workload(M, ctx, stream)
        line["differentiable_solve"] = adjoint_workload(M, ctx, stream)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref, kind, cores = reference_solver()
        t, iters, tf = time_reference_solve(ref, kind, A, b)
        line["cpu_baseline"] = {
            "value": 1e3 * t, "unit": "ms", "cores": cores, "kind": kind,
            "sample": f"one full FP64 PCG-IC(0) solve to 1e-10 ({iters} iterations) of the same "
                      f"system; ic_0 factorisation excluded (timed separately: {tf:.3f} s)"}
    reps.emit(line)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

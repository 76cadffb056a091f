#!/usr/bin/env python
"""Benchmark: Krylov time to 1e-10 relative residual on the 128^3 7-point
Laplacian (n = 2,097,152, nnz = 14,581,760, CSR int32 / float64), PCG with
IC(0), x_true ~ U[-1,1] (seed 1), b = A x_true, x0 = 0.

One step = one complete mixed-precision refined PCG-IC(0) solve to a true
relative residual <= 1e-10, inputs resident in HBM: FP32 inner PCG (FP32
values, FP32 IC(0) factors applied with JACOBI_K Jacobi iterations per
triangle, FP32 vectors, compensated FP32 dots), FP64 residual, update and
stopping norm.  Also measured in the same run:
  * the plain FP64 GPU solve (exact level-scheduled triangular solves, the
    reference's iteration count) -- the mixed-vs-FP64 comparison -- and, for
    transparency, the mixed solve with exact sweeps and the FP64 solve with
    Jacobi-applied factors;
  * the FP64 SpMV on 128^3 (7-point) and 96^3 (27-point) against the
    measured HBM peak;
  * the dominant kernel's roofline;
  * config 3 (27-point convection-diffusion 96^3, BiCGSTAB + ILU(0), FP64
    and mixed);
  * the same mixed solve end to end through the C ABI with host buffers;
  * the reference's own CPU path (MTL4 compiled from its headers) on the host
    cores: its OpenMP and serial builds.

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
CD_GRID = 96
JACOBI_K = 1          # Jacobi iterations per triangle in the FP32 inner solves
INNER_RTOL = 1e-5     # largest reduction asked of one inner solve
METRIC = "Krylov time to 1e-10 rel residual (mixed vs FP64 GPU); SpMV % HBM peak"
WORKLOAD = ("3-D 7-point Laplacian 128^3, PCG + IC(0), FP32 inner (IC(0) applied by "
            f"{JACOBI_K} Jacobi iteration(s) per triangle) / FP64 refinement, rtol 1e-10")


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


def sell_index_bytes(rp, ci):
    """Bytes of column index per stored entry in the library's SELL-32 copies:
    2 (16-bit offsets from the row) when every entry lies within 32,767 of its
    row and MTLGPU_SELL_INDEX is not 32, else 4.  Factors of IC(0)/ILU(0) have
    a subset of the matrix's pattern, so the matrix decides for them too."""
    if os.environ.get("MTLGPU_SELL_INDEX", "") == "32" or len(ci) == 0:
        return 4
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.int64), np.diff(rp))
    return 2 if int(np.abs(ci.astype(np.int64) - rows).max()) <= 32767 else 4


def problem(M):
    A = M.laplacian3d(N_GRID)
    xt = M.uniform(A[0], 1)
    b = M.csr_mult(A, xt)
    return A, b


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_solver(flavour="omp"):
    """The reference's own CPU path: MTL4 compiled from its headers
    (oracle/_ref: 'omp' = the OpenMP build on all host threads, 'serial' = the
    default build); the C restatement of it when that build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ref = oracle.available_reference(flavour=flavour)
    if ref is not None:
        return ref, "reference", ref.threads() if flavour == "omp" else 1
    return oracle.Restatement(), "port", 1


def reference_problem(M, ref, grid=N_GRID, conv=False):
    """The workload built for the reference arm without the solver library:
    the seeded generators of libmtlgpu_fixtures, b = A x_true by the
    reference's own SpMV."""
    A = M.convdiff27(grid, 2) if conv else M.laplacian3d(grid)
    xt = M.uniform(A[0], 1)
    return A, ref.spmv(A, xt)


def time_reference_solve(ref, kind, A, b, method="cg", pc="ic0"):
    t0 = time.perf_counter()
    r = ref.solve(method, pc, A, b, rtol=1e-10, max_iter=2000)
    wall = time.perf_counter() - t0
    # the reference driver times the itl::cg call alone (factorisation apart)
    return (r["t_solve"] if kind == "reference" else wall), r["iterations"], r["t_factor"]


def run_reference_arm(args, rank):
    import mtlgpu as M   # seeded generators only (libmtlgpu_fixtures); no solver library
    if rank != 0:
        return
    ref, kind, cores = reference_solver("omp")
    A, b = reference_problem(M, ref)
    steps = max(1, args.steps)
    warm = max(0, min(args.warmup, 1))   # one warm-up solve: each step is seconds of CPU work
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
                         "cpu_model": cpu_model(),
                         "sample": f"full solve to 1e-10 ({iters} iterations) per step; "
                                   "ic_0 factorisation outside the timed call"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(M, A, b, A3, b3):
    """The reference's CPU path on the host cores (rank 0, N = 1): the full
    FP64 PCG-IC(0) solve (median of 5, OpenMP build; 1 run of the serial
    build), ic_0 factorisation (median of 5), one SpMV (mean over 1000 reps
    with OpenMP, 100 serial: the sparse_matrix_vector_timing.cpp protocol), and
    config 3's bicgstab + ilu_0 solve (OpenMP build)."""
    ref, kind, cores = reference_solver("omp")
    out = {"unit": "ms", "cores": cores, "kind": kind, "cpu_model": cpu_model(),
           "nproc": os.cpu_count()}
    time_reference_solve(ref, kind, A, b)   # warm-up
    runs = [time_reference_solve(ref, kind, A, b) for _ in range(5)]
    out["value"] = 1e3 * statistics.median(r[0] for r in runs)
    out["ic0_factor_ms"] = 1e3 * statistics.median(r[2] for r in runs)
    iters = runs[-1][1]
    x = M.uniform(A[0], 5)
    if kind == "reference":
        out["spmv_ms_omp"] = 1e3 * ref.spmv_time(A, x, 1000)   # seconds per product
    ser, skind, _ = reference_solver("serial")
    if skind == "reference":
        t, _, tf = time_reference_solve(ser, skind, A, b)
        out["serial_solve_ms"] = 1e3 * t
        out["serial_ic0_factor_ms"] = 1e3 * tf
        out["spmv_ms_serial"] = 1e3 * ser.spmv_time(A, x, 100)
    t3, it3, tf3 = time_reference_solve(ref, kind, A3, b3, "bicgstab", "ilu0")
    out["config3_bicgstab_ilu0_ms"] = 1e3 * t3
    out["config3_ilu0_factor_ms"] = 1e3 * tf3
    out["config3_iterations"] = it3
    # the reference's inserter on the same shuffled triplets (slot size 7, one
    # run): mtl::mat::inserter<compressed2D> from construction to destruction
    if kind == "reference":
        # config 4: the reference's itl::cg looped over the same 512 systems
        # (diagonal and ic_0, FP64 to 1e-8), one run each; solve and
        # factorisation times summed separately
        systems, (nb_, _, _, _, offb) = M.graph_batch(512, 1000, 65536, 8.0, 32.0, 1e-2, seed=3)
        bb = M.normal(nb_, 3)
        bat = {}
        for pc in ("diagonal", "ic0"):
            ts = tf = 0.0
            its = []
            for s_, As in enumerate(systems):
                rr = ref.solve("cg", pc, As, bb[offb[s_]:offb[s_ + 1]], rtol=1e-8, max_iter=5000)
                ts += rr["t_solve"]
                tf += rr["t_factor"]
                its.append(rr["iterations"])
            bat[pc] = {"solve_ms": 1e3 * ts, "factor_ms": 1e3 * tf, "iterations_max": max(its),
                       "iterations_mean": float(np.mean(its))}
        out["batched_512_systems"] = bat
        # the other Krylov methods on the same 48^3 system as the device leg
        Ak, bk = krylov_system(M)
        kr = {}
        for meth, pc, param, mx in KRYLOV_LEG:
            rr = ref.solve_krylov(meth, pc, Ak, bk, param=param, max_iter=mx, rtol=1e-8)
            kr[meth] = {"ms": 1e3 * rr["t_solve"], "iterations": rr["iterations"],
                        "err": rr["err"]}
        out["krylov_methods"] = kr
        _, r_, c_, v_ = assembly_triplets(M)
        ref.assemble(A[0], A[0], r_, c_, v_, slot_size=7)
        out["assembly_inserter_ms"] = 1e3 * ref.last_seconds
    out["sample"] = (f"full FP64 PCG-IC(0) solves to 1e-10 ({iters} iterations) of the same "
                     "system, median of 5 after 1 warm-up (OpenMP build, all host threads); "
                     "factorisation timed separately; SpMV 1000 reps (OpenMP) / 100 reps "
                     "(serial); config 3: one FP64 bicgstab + ilu_0 solve (OpenMP); config 4: "
                     "itl::cg over the 512 systems, one run each, diagonal and ic_0; the "
                     "other Krylov methods on 27-point 48^3, one run each; assembly: one "
                     "inserter run over the 14.6M shuffled triplets of the 128^3 matrix")
    return out


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

    def gather(self, obj):
        """Every rank's object, in rank order (all ranks take part)."""
        if self.dist is None:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def emit(self, line):
        """Only rank 0 prints the JSON line."""
        if self.rank == 0:
            print(json.dumps(line), flush=True)
            return True
        return False


def shard_systems(work, world):
    """Splits independent systems over `world` ranks by estimated work
    (longest first, each to the least-loaded rank; ties by index), so every
    rank solves its own share with no exchange between ranks.  Returns each
    rank's system indices, ascending."""
    order = sorted(range(len(work)), key=lambda s_: (-work[s_], s_))
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for s_ in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(s_)
        loads[r] += work[s_]
    return [sorted(p_) for p_ in parts]


def block_diag(systems, idx):
    """The block-diagonal CSR of systems[i] for i in idx: (n, rp, ci, v, offsets)."""
    sizes = [systems[i][0] for i in idx]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    rps, cis, vs = [np.zeros(1, np.int32)], [], []
    e = 0
    for k, i in enumerate(idx):
        n_, rp_, ci_, v_ = systems[i]
        rps.append(rp_[1:] + e)
        cis.append(ci_ + off[k])
        vs.append(v_)
        e += len(ci_)
    cat = (lambda a, dt: np.concatenate(a).astype(dt) if a else np.zeros(0, dt))
    return int(off[-1]), cat(rps, np.int32), cat(cis, np.int32), cat(vs, np.float64), off


def batched_sharded(M, reps, solve_share, seed=3):
    """Config 4 across ranks: the 512 systems split by stored entries
    (shard_systems), each rank solving its share with `solve_share(block
    diagonal matrix, rhs) -> (ms, iterations per system)`; the job's time is
    the slowest rank's, the rank results gathered to every rank."""
    systems, (n, _, _, _, off) = M.graph_batch(512, 1000, 65536, 8.0, 32.0, 1e-2, seed=seed)
    b = M.normal(n, seed)
    parts = shard_systems([len(sy[2]) for sy in systems], reps.world)
    mine = parts[reps.rank]
    A = block_diag(systems, mine)
    rhs = np.concatenate([b[off[i]:off[i + 1]] for i in mine]) if mine else np.zeros(0)
    ms, its = solve_share(A, rhs)
    every = reps.gather({"rank": reps.rank, "systems": mine, "iterations": list(its), "ms": ms})
    slowest = max(e["ms"] for e in every)
    covered = sorted(s_ for e in every for s_ in e["systems"])
    return {"systems": len(systems), "ranks": reps.world, "ms": slowest,
            "systems_per_s": len(systems) / (slowest / 1e3),
            "per_rank_ms": [e["ms"] for e in every],
            "per_rank_systems": [len(e["systems"]) for e in every],
            "all_systems_once": covered == list(range(len(systems)))}


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


def batched_workload(M, ctx, stream, peak):
    """512 independent random-graph Laplacians (n log-uniform in [1e3, 65536],
    average degree U[8, 32], shift 1e-2 mean degree, seed 3), b ~ N(0,1):
    batched PCG to 1e-8, FP64 and FP32 inner solves refined in FP64.  Jacobi,
    and IC(0) applied by JACOBI_K Jacobi iterations per triangle, run as one
    persistent launch (clusters taking systems from a work queue, shape
    autotuned on these systems); IC(0) with exact triangular solves runs the
    level-scheduled path.  Roofline: per system, iterations x (SpMV bytes +
    10 n vector words), summed, over the solve time."""
    systems, (n, rp, ci, v, off) = M.graph_batch(512, 1000, 65536, 8.0, 32.0, 1e-2, seed=3)
    b = M.normal(n, 3)
    dA = M.Csr(ctx, rp, ci, v)
    db, dx, dz = ctx.to_device(b), ctx.array(n), ctx.to_device(np.zeros(n))
    ns = np.diff(off).astype(np.int64)
    nnzs = np.array([len(sy[2]) for sy in systems], np.int64)
    out = {"systems": 512, "n": int(n), "nnz": int(len(ci)), "rtol": 1e-8}

    def run_case(P, mode, wsize):
        kw = dict(rtol=1e-8, max_iter=5000)
        if mode == "mixed":
            kw["mode"] = M.SOLVE_MIXED

        def run():
            ctx.xpay(dz, 0.0, dx)
            st, res = M.solve_batched(dA, P, off, dx, db, **kw)
            assert st == M.OK, st
            return res
        run()
        ms, res = _local_ms(run, 2, stream)
        its = np.array([r.iterations for r in res[-1]], np.int64)
        word = wsize
        per_it = nnzs * (4 + word) + 4 * (ns + 1) + 10 * word * ns
        byt = float((its * per_it).sum())
        rec = {"ms": ms, "iterations_max": int(its.max()), "iterations_mean": float(its.mean()),
               "max_true_rel_residual": max(r.true_resid / r.norm_r0 for r in res[-1]),
               "algorithmic_GB": byt / 1e9, "GBps": byt / ms / 1e6,
               "hbm_frac": byt / ms / 1e6 / peak}
        if mode == "mixed":
            rec["outer_max"] = int(max(r.outer_iterations for r in res[-1]))
        return rec

    P = M.Pc(dA, "diagonal")
    t0 = time.perf_counter()
    choice = M.batched_autotune(dA, P, off, dx, db, rtol=1e-8, max_iter=5000)
    out["autotune"] = {"ctas_per_large_system": (choice % 1000) // 100,
                       "lanes_per_row": choice % 100,
                       "single_cta_below_rows": choice // 1000,
                       "seconds": time.perf_counter() - t0}
    out["diagonal"] = run_case(P, "fp64", 8)
    P.close()
    P = M.Pc(dA, "diagonal", M.FP32)
    out["diagonal_fp32_refined"] = run_case(P, "mixed", 4)
    P.close()
    for prec, key, mode, w in ((M.FP64, "ic0_jacobi", "fp64", 8),
                               (M.FP32, "ic0_jacobi_fp32_refined", "mixed", 4)):
        P = M.Pc(dA, "ic0", prec)
        P.set_jacobi_sweeps(JACOBI_K)
        out[key] = run_case(P, mode, w)
        out[key]["jacobi_iterations_per_triangle"] = JACOBI_K
        P.close()
    P = M.Pc(dA, "ic0")
    out["ic0_exact_sweeps"] = run_case(P, "fp64", 8)
    P.close()
    dA.close()
    return out


def assembly_triplets(M, grid=N_GRID, seed=21):
    """The 128^3 7-point Laplacian as coordinate triplets in a seeded random
    order (the input of an unstructured assembly), and the matrix itself."""
    A = M.laplacian3d(grid)
    n, rp, ci, v = A
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
    perm = np.random.default_rng(seed).permutation(len(ci))
    return A, rows[perm], ci[perm], v[perm]


def assembly_workload(M, ctx, stream, peak):
    """Device assembly (mtlgpu_csr_assemble, the inserter's semantics) of the
    128^3 Laplacian from 14.6M shuffled triplets resident in HBM, to a
    ready-to-use matrix handle; and the device laplacian generator.
    Algorithmic bytes: triplets read once (4 + 4 + 8 B) and the CSR written
    once (nnz (4 + 8) + 4 (n + 1))."""
    A, r, c, v = assembly_triplets(M)
    n, rp, ci, vv = A
    dr, dc, dv = ctx.to_device(r), ctx.to_device(c), ctx.to_device(v)
    B = M.Csr.assemble(ctx, n, n, dr, dc, dv)
    got = B.download()
    identical = bool(np.array_equal(got[0], rp) and np.array_equal(got[1], ci)
                     and np.array_equal(got[2], vv))
    B.close()

    def asm():
        M.Csr.assemble(ctx, n, n, dr, dc, dv).close()
    ms, _ = _local_ms(asm, 3, stream)

    def gen():
        M.Csr.laplacian3d(ctx, N_GRID).close()
    gen()
    ms_gen, _ = _local_ms(gen, 3, stream)
    byt = len(r) * 16 + len(ci) * 12 + 4 * (n + 1)
    return {"workload": "128^3 7-point Laplacian from %d shuffled triplets (store updater)"
                        % len(r),
            "ms": ms, "GBps_algorithmic": byt / ms / 1e6, "hbm_frac": byt / ms / 1e6 / peak,
            "identical_to_generator": identical, "includes": "sort, fold, row starts and the "
            "handle's SpMV layout analysis", "laplacian3d_generate_ms": ms_gen}


KRYLOV_LEG = [("bicg", "identity", 0, 2000), ("cgs", "ilu0", 0, 2000),
              ("bicgstab_2", "ilu0", 0, 2000), ("bicgstab_ell", "ilu0", 4, 2000),
              ("tfqmr", "ilu0", 0, 2000), ("qmr", "ilu0", 0, 100), ("idr_s", "identity", 2, 4000),
              ("gmres", "ilu0", 30, 300)]
KRYLOV_GRID = 48


def krylov_system(M):
    A = M.convdiff27(KRYLOV_GRID, 2)
    return A, M.csr_mult(A, M.uniform(A[0], 1))


def krylov_workload(M, ctx, stream):
    """The other Krylov methods (mtlgpu_solve_krylov, FP64, exact ILU(0)
    triangular solves on the left where the method takes a preconditioner)
    on the 27-point convection-diffusion operator 48^3 (n = 110,592), rtol
    1e-8, x0 = 0: time per solve, iterations, true residual."""
    A, b = krylov_system(M)
    n = A[0]
    dA = M.Csr(ctx, *A[1:])
    P = M.Pc(dA, "ilu0")
    db, dx, dz = ctx.to_device(b), ctx.array(n), ctx.to_device(np.zeros(n))
    out = {"system": "27-point convection-diffusion %d^3, rtol 1e-8" % KRYLOV_GRID, "n": n}
    for meth, pc, param, mx in KRYLOV_LEG:
        L = P if pc == "ilu0" else None

        def run():
            ctx.xpay(dz, 0.0, dx)
            st, res, _ = M.solve_krylov(meth, dA, L, dx, db, param=param, max_iter=mx,
                                        rtol=1e-8)
            return st, res
        run()
        ms, rr = _local_ms(run, 2, stream)
        st, res = rr[-1]
        out[meth] = {"ms": ms, "status": st, "iterations": res.iterations, "param": param,
                     "pc_left": pc, "true_rel_residual": res.true_resid / np.linalg.norm(b),
                     "kernel_launches": res.kernel_launches}
    # the same solves with the ILU(0) factors applied by 2 Jacobi iterations
    # per triangle (another preconditioner application; methods that need the
    # adjoint apply or no preconditioner are left out)
    P.set_jacobi_sweeps(2)
    fast = {}
    for meth, pc, param, mx in KRYLOV_LEG:
        if pc != "ilu0" or meth == "qmr":
            continue

        def run():
            ctx.xpay(dz, 0.0, dx)
            st, res, _ = M.solve_krylov(meth, dA, P, dx, db, param=param, max_iter=mx,
                                        rtol=1e-8)
            return st, res
        run()
        ms, rr = _local_ms(run, 2, stream)
        st, res = rr[-1]
        fast[meth] = {"ms": ms, "status": st, "iterations": res.iterations,
                      "true_rel_residual": res.true_resid / np.linalg.norm(b)}
    out["ilu0_by_jacobi_k2"] = fast
    P.set_jacobi_sweeps(0)
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
           "dtype": "f64", "rtol": 1e-10, "pc": "IC(0), exact triangular solves"}
    x_ex, g_ex, l_ex = dx.download(), grad.download(), dlam.download()
    # the same FP64 solves with the IC(0) factors applied by k Jacobi
    # iterations per triangle: another preconditioner, the same gradients to
    # the solve tolerance
    for k in (1, 2):
        P.set_jacobi_sweeps(k)
        forward()
        backward()
        mf, rf = _local_ms(forward, 2, stream)
        mb, rb = _local_ms(backward, 2, stream)
        xk, gk, lk = dx.download(), grad.download(), dlam.download()
        rel = lambda a, b_: float(np.linalg.norm(a - b_) / np.linalg.norm(b_))
        out[f"jacobi_k{k}"] = {"forward_ms": mf, "backward_ms": mb,
                               "forward_iterations": rf[-1].iterations,
                               "backward_iterations": rb[-1].iterations,
                               "rel_diff_x": rel(xk, x_ex), "rel_diff_dL_db": rel(lk, l_ex),
                               "rel_diff_dL_dvals": rel(gk, g_ex)}
    P.set_jacobi_sweeps(0)
    P.close()
    dA.close()
    return out


def profile_case(case, grid, launches):
    """Runs one kernel (or one solve) of the path a few times on an N^3
    Laplacian, for profiler captures: 'spmv' (FP64 y = A x, SELL-32),
    'spmv32' (FP32), 'jacobi32' (FP32 IC(0) apply with JACOBI_K Jacobi
    iterations per triangle), 'sweep64' / 'sweep32' (exact IC(0) lower sweep),
    'mixed' (complete mixed solves of the headline configuration, for the
    launch list; the solves get an interrupt flag held at 0, which keeps
    their iterations in host-launched graphs: ncu lists every kernel of
    those, while the device-side loop's body graph is not profiled per
    kernel), 'mixed27' (the mixed BiCGSTAB + ILU(0) solve of the N^3
    27-point convection-diffusion system, seed 2), 'batched' (the 512-system
    batched Jacobi PCG, FP64), 'assemble' (device assembly of the N^3 Laplacian from shuffled triplets)."""
    import mtlgpu as M
    A = M.laplacian3d(grid)
    n = A[0]
    ctx = M.Context(0)
    dA = M.Csr(ctx, *A[1:])
    if case in ("spmv", "spmv32"):
        dt = np.float32 if case == "spmv32" else np.float64
        dx, dy = ctx.to_device(M.uniform(n, 5).astype(dt)), ctx.array(n, dt)
        for _ in range(launches):
            (dA.spmv_f32 if case == "spmv32" else dA.spmv)(dx, dy)
    elif case == "jacobi32":
        P = M.Pc(dA, "ic0", M.FP32)
        P.set_jacobi_sweeps(JACOBI_K)
        r, z = ctx.to_device(np.ones(n, np.float32)), ctx.array(n, np.float32)
        for _ in range(launches):
            P.apply_f32(r, z)
    elif case == "mixed":
        P = M.Pc(dA, "ic0", M.FP32)
        P.set_jacobi_sweeps(JACOBI_K)
        b = M.csr_mult(A, M.uniform(n, 1))
        dx, db = ctx.array(n), ctx.to_device(b)
        flag = np.zeros(1, np.int32)
        for _ in range(launches):
            dx.upload(np.zeros(n))
            st, res, _ = M.solve("cg", dA, P, dx, db, rtol=1e-10, max_iter=4000,
                                 mode=M.SOLVE_MIXED, inner_rtol=INNER_RTOL, interrupt=flag)
            assert st == M.OK, st
    elif case == "mixed27":
        A = M.convdiff27(grid, 2)
        n = A[0]
        dA.close()
        dA = M.Csr(ctx, *A[1:])
        P = M.Pc(dA, "ilu0", M.FP32)
        P.set_jacobi_sweeps(JACOBI_K)
        b = M.csr_mult(A, M.uniform(n, 1))
        dx, db = ctx.array(n), ctx.to_device(b)
        flag = np.zeros(1, np.int32)    # host-launched graphs, as for 'mixed'
        for _ in range(launches):
            dx.upload(np.zeros(n))
            st, res, _ = M.solve("bicgstab", dA, P, dx, db, rtol=1e-10, max_iter=4000,
                                 mode=M.SOLVE_MIXED, inner_rtol=INNER_RTOL, interrupt=flag)
            assert st == M.OK, st
    elif case == "assemble":
        Af, r, c, v = assembly_triplets(M, grid)
        nf = Af[0]
        dr, dc, dv = ctx.to_device(r), ctx.to_device(c), ctx.to_device(v)
        for _ in range(launches):
            M.Csr.assemble(ctx, nf, nf, dr, dc, dv).close()
    elif case == "batched":
        systems, (nb, rp, ci, v, off) = M.graph_batch(512, 1000, 65536, 8.0, 32.0, 1e-2,
                                                      seed=3)
        dB = M.Csr(ctx, rp, ci, v)
        P = M.Pc(dB, "diagonal")
        db, dx = ctx.to_device(M.normal(nb, 3)), ctx.array(nb)
        for _ in range(launches):
            dx.upload(np.zeros(nb))
            st, _ = M.solve_batched(dB, P, off, dx, db, rtol=1e-8, max_iter=5000)
            assert st == M.OK, st
    else:
        prec = M.FP32 if case == "sweep32" else M.FP64
        dt = np.float32 if prec == M.FP32 else np.float64
        P = M.Pc(dA, "ic0", prec)
        r, z = ctx.to_device(np.ones(n, dt)), ctx.array(n, dt)
        for _ in range(launches):
            P.sweep(M.LOWER, r, z)
    ctx.synchronize()
    print(json.dumps({"profile_case": case, "grid": grid, "launches": launches}))


def sweep_scan():
    """Exact IC(0) lower sweep (level-ordered ticket kernel) on N^3 7-point
    Laplacians, N = 64 .. 192: time per sweep with CUDA events (20 sweeps
    after 3 warm-ups), levels (3N - 2) and rows per level.  A least-squares
    line time/level = hop + row_cost * rows/level splits the per-level cost
    into the dependency hop and the row work."""
    import torch
    import mtlgpu as M
    os.environ["MTLGPU_SWEEP"] = "ticket"
    ctx = M.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device="cuda:0")
    rows = []
    for N in (64, 96, 128, 160, 192):
        A = M.laplacian3d(N)
        n = A[0]
        dA = M.Csr(ctx, *A[1:])
        for prec, dt, name in ((M.FP64, np.float64, "f64"), (M.FP32, np.float32, "f32")):
            P = M.Pc(dA, "ic0", prec)
            r, z = ctx.to_device(np.ones(n, dt)), ctx.array(n, dt)
            for _ in range(3):
                P.sweep(M.LOWER, r, z)
            ctx.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(20):
                P.sweep(M.LOWER, r, z)
            e1.record(stream)
            ctx.synchronize()
            ms = e0.elapsed_time(e1) / 20
            lev = P.factor_info(M.LOWER)[1]
            rec = {"N": N, "prec": name, "n": n, "levels": lev, "rows_per_level": n / lev,
                   "sweep_ms": ms, "us_per_level": 1e3 * ms / lev}
            rows.append(rec)
            print(json.dumps(rec), flush=True)
            P.close()
        dA.close()
    for name in ("f64", "f32"):
        pts = [(r["rows_per_level"], r["us_per_level"]) for r in rows if r["prec"] == name]
        xs, ys = np.array([p[0] for p in pts]), np.array([p[1] for p in pts])
        slope, hop = np.polyfit(xs, ys, 1)
        print(json.dumps({"fit": name, "hop_us": hop, "us_per_1000_rows": 1e3 * slope}),
              flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mtlgpu", choices=["mtlgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the config-3, batched and differentiable-solve measurements")
    ap.add_argument("--profile-case",
                    choices=["spmv", "spmv32", "jacobi32", "sweep64", "sweep32", "mixed",
                             "mixed27", "batched", "assemble"])
    ap.add_argument("--sweep-scan", action="store_true",
                    help="per-level cost of the exact sweep on 64^3 .. 192^3 grids")
    ap.add_argument("--grid", type=int, default=64)
    ap.add_argument("--launches", type=int, default=3)
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case, args.grid, args.launches)
        return
    if args.sweep_scan:
        sweep_scan()
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
    P32.set_jacobi_sweeps(JACOBI_K)
    ctx.synchronize()
    t_fac32 = time.perf_counter() - t0
    db = ctx.to_device(b)
    dx = ctx.array(n)
    dzero = ctx.to_device(np.zeros(n))
    setup_s = time.perf_counter() - t_setup

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed(fn, reps_):
        """Mean ms of fn over reps_, CUDA events on the library's stream."""
        ctx.synchronize()
        barrier()
        e0, e1 = ev(), ev()
        e0.record(stream)
        out = [fn() for _ in range(reps_)]
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1) / reps_, out

    mixed_kw = dict(rtol=1e-10, max_iter=4000, mode=M.SOLVE_MIXED, inner_rtol=INNER_RTOL)
    fp64_kw = dict(rtol=1e-10, max_iter=2000)

    def solver(P, kw, method="cg", dA_=dA, dx_=dx, db_=db, dzero_=dzero):
        def run():
            ctx.xpay(dzero_, 0.0, dx_)                # x0 = 0 on the device
            st, res, _ = M.solve(method, dA_, P, dx_, db_, **kw)
            assert st == M.OK, st
            return res
        return run

    solve_mixed = solver(P32, mixed_kw)
    solve_fp64 = solver(P64, fp64_kw)
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

    # transparency: which part of the gain is the approximate triangular solve
    P32.set_jacobi_sweeps(0)
    solve_mixed()
    ms_mixed_exact, res_mx = timed(solve_mixed, 2)
    P32.set_jacobi_sweeps(JACOBI_K)
    P64.set_jacobi_sweeps(JACOBI_K)
    solve_fp64()
    ms_fp64_jacobi, res_fj = timed(solve_fp64, 2)
    P64.set_jacobi_sweeps(0)

    peak, peak_kind = peaks()

    flush = torch.empty(64 << 20, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > L2

    def hold():
        """Holds the library's stream with a ~20 ms spin kernel, so that a
        loop of per-launch event pairs is queued in full before the GPU
        reaches it: a host slower than the kernels would otherwise leave
        idle gaps inside the event pairs."""
        with torch.cuda.stream(stream):
            torch.cuda._sleep(40_000_000)

    def cold_ms(fn, reps_):
        """Mean ms of fn with the 126 MB L2 flushed (256 MB written) before
        every launch; each launch bracketed by its own CUDA events on the
        library's stream."""
        evs = []
        ctx.synchronize()
        hold()
        with torch.cuda.stream(stream):
            for _ in range(reps_):
                flush.zero_()
                e0, e1 = ev(), ev()
                e0.record(stream)
                fn()
                e1.record(stream)
                evs.append((e0, e1))
        ctx.synchronize()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) / reps_

    def after_ms(fn, before, reps_):
        """Mean ms of fn launched right after before() (untimed), each fn
        bracketed by its own CUDA events on the library's stream: fn with
        the cache state the preceding kernels of the solve leave."""
        evs = []
        ctx.synchronize()
        hold()
        for _ in range(reps_):
            before()
            e0, e1 = ev(), ev()
            e0.record(stream)
            fn()
            e1.record(stream)
            evs.append((e0, e1))
        ctx.synchronize()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) / reps_

    def spmv_stats(dA_, n_, nnz_, ib_, reps_=100):
        # algorithmic bytes: 8-byte value + ib_-byte index per entry, the
        # slice offsets, x once and y once
        dxs, dys = ctx.to_device(M.uniform(n_, 5)), ctx.array(n_)
        for _ in range(5):
            dA_.spmv(dxs, dys)
        ms, _ = timed(lambda: dA_.spmv(dxs, dys), reps_)
        ms_cold = cold_ms(lambda: dA_.spmv(dxs, dys), 30)
        byt = nnz_ * (8 + ib_) + 4 * (n_ // 32 + 1) + 2 * n_ * 8
        return {"ms": ms, "GBps": byt / ms / 1e6, "hbm_frac": byt / ms / 1e6 / peak,
                "bytes": byt, "index_bytes": ib_, "peak_kind": peak_kind,
                "back_to_back": "mean of %d products back to back" % reps_,
                "cold": {"ms": ms_cold, "GBps": byt / ms_cold / 1e6,
                         "hbm_frac": byt / ms_cold / 1e6 / peak,
                         "how": "L2 flushed before each product, per-launch CUDA events"}}

    ib = sell_index_bytes(A[1], A[2])
    spmv = spmv_stats(dA, n, nnz, ib)

    # The mixed solve's kernels, timed alone on the same data (FP32).  Per
    # inner iteration the solve runs three: the direction product
    # (p = z + beta p, q = A p, p.q), the first L pass fused with the x / r
    # update, and the U pass with r.z; the first and the last are timed here
    # (the fused L pass has no entry point of its own; its share is in the
    # launch-list profile).  Algorithmic bytes: the product reads A's entries
    # (4-byte value + ib-byte index), the slice offsets, z and p once and
    # writes p and q; a Jacobi pass reads the factor's off-diagonal entries
    # (4-byte value + ib-byte index), v, D and the previous iterate once and
    # writes one vector.  The plain FP32 SpMV is timed for the record.
    nnz_off = P32.factor_info(M.LOWER)[0] - n
    bytes_pass = nnz_off * (4 + ib) + 4 * (n // 32 + 1) + 4 * n * 4
    r32 = ctx.to_device(np.ones(n, np.float32))
    z32 = ctx.array(n, np.float32)
    for _ in range(3):
        P32.apply_f32(r32, z32)
    ms_apply32, _ = timed(lambda: P32.apply_f32(r32, z32), 50)
    ms_pass = ms_apply32 / (2 * JACOBI_K)
    ms_pass_cold = cold_ms(lambda: P32.apply_f32(r32, z32), 30) / (2 * JACOBI_K)
    x32 = ctx.to_device(M.uniform(n, 5).astype(np.float32))
    y32 = ctx.array(n, np.float32)
    for _ in range(5):
        dA.spmv_f32(x32, y32)
    ms_spmv32, _ = timed(lambda: dA.spmv_f32(x32, y32), 100)
    bytes_spmv32 = nnz * 8 + 4 * (n // 32 + 1) + 2 * n * 4   # 4-byte indices in FP32
    p32, po32, q32, dpq = (ctx.to_device(M.uniform(n, 6).astype(np.float32)),
                           ctx.array(n, np.float32), ctx.array(n, np.float32), ctx.array(1))

    def direction():
        dA.cg_direction_product(M.FP32, x32, 0.5, p32, po32, q32, dpq)

    for _ in range(5):
        direction()
    # In the solve the product follows the IC(0) apply (L and U passes,
    # ~150 MB streamed): timed that way for the roofline; back to back (L2
    # keeps part of A between launches) and with L2 flushed, for the record.
    ms_dir32 = after_ms(direction, lambda: P32.apply_f32(r32, z32), 50)
    ms_dir32_b2b, _ = timed(direction, 100)
    ms_dir32_cold = cold_ms(direction, 30)
    bytes_dir32 = nnz * (4 + ib) + 4 * (n // 32 + 1) + 4 * n * 4
    traffic = read_traffic()

    # exact sweeps (the FP64 path's dominant kernel), for the record
    L64 = P64.factor_info(M.LOWER)[0]
    r64 = ctx.to_device(np.ones(n))
    z64 = ctx.array(n)
    for _ in range(3):
        P64.sweep(M.LOWER, r64, z64)
    ms_sweep64, _ = timed(lambda: P64.sweep(M.LOWER, r64, z64), 20)
    bytes_sweep64 = L64 * 12 + 4 * (n + 1) + 2 * n * 8

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

    dominant = {
        "jacobi_pass_kernel<float> (IC(0) U pass, r.z fused)": (ms_pass, bytes_pass,
                                                                 2 * JACOBI_K - 1,
                                                                 "jacobi_pass_f32"),
        "cg_pspmv_kernel<float> (p = z + beta p, q = A p, p.q)": (ms_dir32, bytes_dir32, 1,
                                                                   "cg_pspmv_f32"),
    }
    dom = max(dominant, key=lambda k: dominant[k][0] * dominant[k][2])
    d_ms, d_bytes, _, d_key = dominant[dom]
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
        "config": {"workload": WORKLOAD, "n": n, "nnz": nnz,
                   "index": "int32 CSR; SELL-32 column indices: %d bytes in the solve's "
                            "kernels and the FP64 SpMV, 4 in the plain FP32 SpMV" % ib,
                   "jacobi_iterations_per_triangle": JACOBI_K, "inner_rtol": INNER_RTOL,
                   "l2": "inputs larger than L2 (matrix 175 MB + factors 2 x 100 MB)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "iterations": {"mixed_inner": res_mixed[-1].iterations,
                       "mixed_outer": res_mixed[-1].outer_iterations,
                       "fp64": res_fp64[-1].iterations,
                       "mixed_exact_sweeps_inner": res_mx[-1].iterations,
                       "fp64_jacobi": res_fj[-1].iterations},
        "true_rel_residual": true_rel,
        "fp64_ms": ms_fp64,
        "mixed_speedup_vs_fp64": ms_fp64 / ms_mixed,
        "mixed_exact_sweeps_ms": ms_mixed_exact,
        "fp64_jacobi_sweeps_ms": ms_fp64_jacobi,
        "spmv": spmv,
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": d_bytes / d_ms / 1e6,
                     "peak": peak, "unit": "GB/s", "frac": d_bytes / d_ms / 1e6 / peak,
                     "traffic": traffic.get(d_key), "algorithmic_bytes": d_bytes,
                     "ms": d_ms, "peak_kind": peak_kind},
        "mixed_kernels": {"cg_pspmv_f32": {"ms": ms_dir32, "GBps": bytes_dir32 / ms_dir32 / 1e6,
                                           "how": "each launch right after an IC(0) apply, "
                                                  "as in the solve; per-launch CUDA events",
                                           "bytes": bytes_dir32, "launches_per_iteration": 1,
                                           "back_to_back_ms": ms_dir32_b2b,
                                           "cold_ms": ms_dir32_cold,
                                           "cold_GBps": bytes_dir32 / ms_dir32_cold / 1e6},
                          "jacobi_pass_f32": {"ms": ms_pass, "GBps": bytes_pass / ms_pass / 1e6,
                                              "bytes": bytes_pass,
                                              "launches_per_iteration": 2 * JACOBI_K - 1,
                                              "cold_ms": ms_pass_cold,
                                              "cold_GBps": bytes_pass / ms_pass_cold / 1e6},
                          "spmv_f32": {"ms": ms_spmv32, "GBps": bytes_spmv32 / ms_spmv32 / 1e6,
                                       "bytes": bytes_spmv32}},
        "sweep_fp64": {"ms": ms_sweep64, "GBps": bytes_sweep64 / ms_sweep64 / 1e6,
                       "bytes": bytes_sweep64, "levels": P64.factor_info(M.LOWER)[1]},
        "setup_s": {"total": setup_s, "ic0_fp64": t_fac64, "ic0_fp32": t_fac32},
        "e2e": {"value": ms_e2e, "unit": "ms", "h2d_bytes_per_step": 2 * n * 8,
                "d2h_bytes_per_step": n * 8},
        "gpu_launches": launches,
        "clocks": clk,
    }
    A3 = b3 = None
    if world > 1 and not args.no_extras:
        # config 4 sharded by systems: no data-path collective
        def solve_share(Ab, rhs):
            nb_, rp_, ci_, v_, off_ = Ab
            dB = M.Csr(ctx, rp_, ci_, v_)
            Pb = M.Pc(dB, "diagonal")
            dbb, dxb, dzb = ctx.to_device(rhs), ctx.array(nb_), ctx.to_device(np.zeros(nb_))

            def run():
                ctx.xpay(dzb, 0.0, dxb)
                st, res = M.solve_batched(dB, Pb, off_, dxb, dbb, rtol=1e-8, max_iter=5000)
                assert st == M.OK, st
                return res
            run()
            ms_, rr = timed(run, 2)
            Pb.close()
            dB.close()
            return ms_, [r_.iterations for r_ in rr[-1]]
        line["batched_sharded"] = batched_sharded(M, reps, solve_share)
    if world == 1 and not args.no_extras:
        A3, b3, line["config3"] = config3_workload(M, ctx, timed, solver, spmv_stats, peak)
        line["batched"] = batched_workload(M, ctx, stream, peak)
        line["differentiable_solve"] = adjoint_workload(M, ctx, stream)
        line["assembly"] = assembly_workload(M, ctx, stream, peak)
        line["krylov_methods"] = krylov_workload(M, ctx, stream)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if A3 is None:
            A3 = M.convdiff27(CD_GRID, 2)
            b3 = M.csr_mult(A3, M.uniform(A3[0], 1))
        line["cpu_baseline"] = cpu_baseline(M, A, b, A3, b3)
    reps.emit(line)
    if dist is not None:
        dist.destroy_process_group()


def config3_workload(M, ctx, timed, solver, spmv_stats, peak):
    """Config 3: 27-point convection-diffusion on 96^3 (seed 2), x_true ~
    U[-1,1] (seed 1), b = A x_true; BiCGSTAB + ILU(0) to 1e-10 in FP64 (exact
    triangular solves: the reference's iteration count) and mixed (FP32
    inner solve, ILU(0) applied by JACOBI_K Jacobi iterations per triangle,
    FP64 refinement)."""
    A = M.convdiff27(CD_GRID, 2)
    n, nnz = A[0], len(A[2])
    b = M.csr_mult(A, M.uniform(n, 1))
    dA = M.Csr(ctx, *A[1:])
    P64 = M.Pc(dA, "ilu0", M.FP64)
    P32 = M.Pc(dA, "ilu0", M.FP32)
    P32.set_jacobi_sweeps(JACOBI_K)
    db, dx, dz = ctx.to_device(b), ctx.array(n), ctx.to_device(np.zeros(n))
    kw = dict(dA_=dA, dx_=dx, db_=db, dzero_=dz)
    fp64 = solver(P64, dict(rtol=1e-10, max_iter=2000), "bicgstab", **kw)
    mixed = solver(P32, dict(rtol=1e-10, max_iter=4000, mode=M.SOLVE_MIXED,
                             inner_rtol=INNER_RTOL), "bicgstab", **kw)
    fp64()
    mixed()
    ms_fp64, r64 = timed(fp64, 2)
    ms_mixed, rmx = timed(mixed, 3)
    x = dx.download()
    out = {"workload": "27-point convection-diffusion 96^3, BiCGSTAB + ILU(0), rtol 1e-10",
           "n": n, "nnz": nnz, "mixed_ms": ms_mixed, "fp64_ms": ms_fp64,
           "mixed_speedup_vs_fp64": ms_fp64 / ms_mixed,
           "iterations": {"fp64": r64[-1].iterations, "mixed_inner": rmx[-1].iterations,
                          "mixed_outer": rmx[-1].outer_iterations},
           "true_rel_residual": float(np.linalg.norm(b - M.csr_mult(A, x)) / np.linalg.norm(b)),
           "jacobi_iterations_per_triangle": JACOBI_K,
           "spmv": spmv_stats(dA, n, nnz, sell_index_bytes(A[1], A[2]))}
    P32.close()
    P64.close()
    dA.close()
    return A, b, out


if __name__ == "__main__":
    main()

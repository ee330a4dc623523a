#!/usr/bin/env python
"""GLR benchmark: one "job" = one GLR build + a 16-RHS solve + a logdet.

Workload (config 2, the plain FP64 GPU configuration): 512^2 uniform grid on
[0,1]^2 (N = 262144), lumped mass, Z = L + 25 M (5-point Neumann
Laplacian), B = Gaussian (l = 0.005) x Wendland-C2 (rho = 0.015) kernel
matrix (~183 nnz/row), GLR rank 200 + oversample 20 (ell = 220, kept capped
at 200), q = 1, seed 0, Z-solve tolerance 1e-10; 16 N(0,1) right-hand sides
solved at c = 1 and logdet at c = 1.  Synthetic data generated from the
configuration's formulas (lgh_b200/problems.py).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Ours: each rank builds its own replica (the build does not shard on one
node here: replicas, weak scaling); inputs resident in HBM; W untimed jobs,
then K jobs between a barrier + synchronize, CUDA events on the library's
stream (the legacy default stream), max over ranks.  Also reported: the
same jobs end to end through the C ABI from pinned host buffers (e2e), the
per-kernel roofline of the dominant kernel from the library's live event
timing, per-RHS solve latency p50/p99, SM clocks sampled during the timed
region, a Poisson request stream through the request loop (serving), and
the CPU baseline (one complete job of the oracle on all host cores).

--impl reference: the reference's CPU path restated by the oracle
(oracle/), all host threads, same workload and metric; the K timed steps
together run complete jobs (each job cut into bounded pieces that are
spread evenly over the steps), so the steps' measured time is whole jobs.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "lgpsf-hessian_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

CONFIG = "c2"
NRHS = 16
SHIFT = 1.0
ZRTOL = 1e-10
ELL, RANK, QPOW, SEED = 220, 200, 1, 0
METRIC = "GLR jobs/s (build + 16-RHS solve + logdet)"
UNIT = "jobs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--serve-s", type=float, default=5.0)
    ap.add_argument("--serve-slots", type=int, default=64,
                    help="Z-solve columns in flight in the request loop")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the c3 / c4 / c5 sub-objects of the line")
    ap.add_argument("--serve-rates", default="",
                    help="comma-separated request rates for --config c5")
    ap.add_argument("--kernel-case", default="",
                    choices=["", "zsolve", "spmm", "build", "batch", "rows"],
                    help="run one device case and print the library's "
                         "per-kernel event timing (for ncu captures of "
                         "single kernels): zsolve = a blocked Z-solve of a "
                         "seeded N x width block, spmm = B times it, build "
                         "= one GLR build at ell = width")
    ap.add_argument("--kc-config", default="c2")
    ap.add_argument("--kc-width", type=int, default=220)
    ap.add_argument("--kc-rtol", type=float, default=1e-10)
    ap.add_argument("--kc-fp32", action="store_true")
    ap.add_argument("--kc-shifts", type=int, default=8,
                    help="batch case: shifts (log-spaced in [1e-3, 1e3])")
    ap.add_argument("--kc-rank", type=int, default=200,
                    help="batch case: ell (rank cap = ell - 20)")
    ap.add_argument("--kc-ranks", type=int, default=2,
                    help="rows case: row slabs, run as threads of this "
                         "process on one GPU (the ranks serialise on the "
                         "device, so the case measures the sharded "
                         "algorithm's extra work, not multi-GPU time)")
    ap.add_argument("--config", default="c2", choices=["c2", "c3", "c4", "c5"],
                    help="c2: the headline job (default); c3 / c4: the "
                         "mixed-precision 3D extend and the batched-shift "
                         "workloads, one JSON line each")
    return ap.parse_args()


def max_over_ranks(seconds, world, device):
    """The slowest rank's device-timed seconds (every rank calls this at
    the same point; one all-reduce of one double)."""
    if world <= 1:
        return seconds
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(cfg):
    return {"workload": "c2: 512^2 2D grid (N=%d), B Gaussian x Wendland "
                        "(%.1f nnz/row), Z = L + 25 M (5-point), ell=%d "
                        "(rank %d + oversample %d), q=%d, Z-solve rtol %g, "
                        "%d N(0,1) RHS at c=%g, logdet at c=%g"
                        % (cfg["N"], cfg["nnz_B"] / cfg["N"], ELL, RANK,
                           ELL - RANK, QPOW, ZRTOL, NRHS, SHIFT, SHIFT),
            "N": cfg["N"], "nnz_B": cfg["nnz_B"], "nnz_Z": cfg["nnz_Z"],
            "ell": ELL, "rank_cap": RANK, "q_power": QPOW, "seed": SEED,
            "zsolve": "blocked PCG, smoothed-aggregation V-cycle "
                      "preconditioner, rtol %g" % ZRTOL,
            "nrhs": NRHS, "shift": SHIFT,
            "l2": "inputs larger than L2 (ell-wide blocks 461 MB each)"}


# --------------------------------------------------------------------------
# CPU side: the oracle (the reference's replicated CPU path restated) on the
# host cores


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_job(cfg, oracle, nthreads, rhs):
    """One complete C2 job on the oracle, as a sequence of bounded pieces
    (a generator: each next() runs one piece).  The same job as the e2e
    arm: the prior with its multigrid set-up, the build (ell 220, rank cap
    200, q 1, check on; F-applies in waves of `nthreads` columns, one
    column per thread), the 16-RHS solve at c = 1 (column-parallel), the
    logdet.  Yields the logdet last."""
    B, Z = cfg["_orc_B"], cfg["_orc_Z"]
    pr = oracle.Prior(Z, cfg["mass"], ksp_rtol=ZRTOL, pc="amg")
    yield None
    o = oracle.opts_default(ell=ELL, q_power=QPOW, seed=SEED, trunc_rel=0.0,
                            check=1)
    b = oracle.Build(B, pr, o, cap=RANK, wave=nthreads)
    while b.step():
        yield None
    yield None
    g = b.finish()
    g.solve_block(SHIFT, rhs)
    yield g.logdet(SHIFT)


def reference_pieces(nthreads):
    """Pieces of one reference_job: prior, build, solve + logdet."""
    import oracle
    return 1 + oracle.build_pieces(ELL, QPOW, RANK, nthreads) + 1


def oracle_setup(cfg):
    import oracle
    nthreads = os.cpu_count() or 1
    oracle.set_threads(nthreads)
    if "_orc_B" not in cfg:
        cfg["_orc_B"] = oracle.Csr(cfg["B"]["rowptr"], cfg["B"]["colidx"],
                                   cfg["B"]["vals"])
        cfg["_orc_Z"] = oracle.Csr(cfg["Z"]["rowptr"], cfg["Z"]["colidx"],
                                   cfg["Z"]["vals"])
    rhs = np.asfortranarray(
        np.random.default_rng(7).standard_normal((cfg["N"], NRHS)))
    return oracle, nthreads, rhs


def _sample_note(nthreads):
    return ("oracle (the reference's replicated CPU path restated in C++, "
            "OpenBLAS), %d threads on %s: complete C2 jobs, each the prior "
            "with its smoothed-aggregation set-up, the build (F-applies of "
            "one column per thread, per-column CG rtol %g with the V-cycle "
            "PC in the role of the reference's CG + PCGAMG), the 16-RHS "
            "solve and the logdet" % (nthreads, cpu_model(), ZRTOL))


def cpu_baseline(cfg):
    """One complete job on the oracle, timed end to end (no sample, no
    extrapolation)."""
    oracle, nthreads, rhs = oracle_setup(cfg)
    t0 = time.perf_counter()
    for _ in reference_job(cfg, oracle, nthreads, rhs):
        pass
    job = time.perf_counter() - t0
    return dict(value=1.0 / job, unit=UNIT, cores=nthreads, kind="port",
                cpu_model=cpu_model(),
                sample=_sample_note(nthreads) + "; one job, %.1f s" % job)


def run_reference(args):
    """The reference arm: the oracle on all host threads, on the same
    workload.  The K timed steps run exactly J complete jobs, J = ceil(K /
    P) with P the pieces of one job, the pieces split evenly over the
    steps, so ms_per_step x K is the measured time of J whole jobs.  The
    W warm-up steps run the same share of pieces of a separate job that is
    then dropped."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from lgh_b200 import problems as P
    cfg = P.grid_problem(CONFIG)
    oracle, nthreads, rhs = oracle_setup(cfg)
    npc = reference_pieces(nthreads)
    K, W = args.steps, args.warmup
    J = -(-K // npc)
    bounds = [(k * J * npc) // K for k in range(K + 1)]

    def run_steps(nsteps, njobs, times):
        jobs = (reference_job(cfg, oracle, nthreads, rhs)
                for _ in range(njobs))
        it = (x for job in jobs for x in job)
        for k in range(nsteps):
            t0 = time.perf_counter()
            for _ in range(bounds[k + 1] - bounds[k]):
                next(it, None)
            if k == nsteps - 1 and times is not None:
                for _ in it:             # the last step drains what is left
                    pass
            if times is not None:
                times.append(time.perf_counter() - t0)

    run_steps(min(W, K), 1, None)        # warm-up share of a dropped job
    times = []
    run_steps(K, J, times)
    total = sum(times)
    v = J / total
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": K, "warmup": W,
            "ms_per_step": 1e3 * total / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (config formulas)", "config": workload(cfg),
            "jobs_timed": J, "pieces_per_job": npc,
            "step_note": "the %d timed steps run %d complete job(s), %d "
                         "pieces each, split evenly over the steps"
                         % (K, J, npc),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads,
                             "kind": "port", "cpu_model": cpu_model(),
                             "sample": _sample_note(nthreads)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# GPU side


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        # every rank runs the same replica work between collectives, so a
        # rank that waits this long has lost its peers
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    import lgh_b200 as L
    from lgh_b200 import problems as P

    L.load()
    cfg = P.grid_problem(CONFIG)
    N = cfg["N"]
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=ZRTOL))
    opts = L.glr_opts(ell=ELL, q_power=QPOW, seed=SEED, trunc_rel=0.0,
                      check=1)
    ex = L.exec_opts(rank_cap=RANK)
    rhs_h = np.random.default_rng(100 + rank).standard_normal((N, NRHS))
    rhs = L.DeviceBlock(N, NRHS, rhs_h)
    xout = L.DeviceBlock(N, NRHS)
    cs = np.array([SHIFT])
    Lb = L.load()

    # the previous job's object is released when the next job starts (in
    # the timed region), as a caller that builds one object per job does;
    # its blocks then come back from the library's allocation cache
    live = {}

    def job(timers=None):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        live.pop("g", None)
        g = L.Glr(B, pr, opts, exec=ex)
        live["g"] = g
        ev[1].record()
        L._chk(Lb.lgh_glr_solve_batch(g.h, 1, cs.ctypes.data_as(L.c_dbl_p),
                                      NRHS, rhs.ptr(), N, xout.ptr(), N),
               "lgh_glr_solve_batch")
        ev[2].record()
        ld = g.logdet(SHIFT)
        ev[3].record()
        if timers is not None:
            timers.append(ev)
        return g, ld

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        job()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    launches0 = Lb.lgh_launch_count()
    rt0 = L.runtime_counters()
    t_start, t_end = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    timers = []
    torch.cuda.nvtx.range_push("timed")
    t_start.record()
    for _ in range(args.steps):
        job(timers)
    t_end.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches = Lb.lgh_launch_count() - launches0
    rt1 = L.runtime_counters()
    runtime = {k: (rt1[k] - rt0[k]) / args.steps
               for k in ("allocs", "alloc_s", "frees", "free_s")}
    clk = clocks.stop()
    elapsed = max_over_ranks(t_start.elapsed_time(t_end) / 1e3, world,
                             "cuda")
    build_s = [ev[0].elapsed_time(ev[1]) / 1e3 for ev in timers]
    solve_s = [ev[1].elapsed_time(ev[2]) / 1e3 for ev in timers]
    g_last = live["g"]

    # per-kernel roofline: a separate, untimed pass of the same job with
    # the library's per-launch CUDA-event registry on (the registry adds an
    # event pair around every hot launch, so it stays off in the timed loop)
    L.kernel_timing(True)
    for _ in range(min(2, args.steps)):
        job()
    torch.cuda.synchronize()
    ktimes = L.kernel_timing_get()
    L.kernel_timing(False)
    stats = g_last.stats()
    report = g_last.report

    # per-RHS latency of the reference-form single solve (lgh_glr_solve)
    lat = []
    for j in range(NRHS):
        v = L.Vec(data=rhs_h[:, j])
        x = L.Vec(N)
        e0, e1 = torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        e0.record()
        L._chk(Lb.lgh_glr_solve(g_last.h, SHIFT, v.h, x.h), "lgh_glr_solve")
        e1.record()
        torch.cuda.synchronize()
        lat.append(e0.elapsed_time(e1))
    lat.sort()

    # solve residual against the GLR model operator H~(c) (one RHS, FP64 on
    # the host): H~ = Z M^{-1/2} (U Lam U^T + c I) M^{-1/2} Z
    x0 = xout.get()[:, 0]
    U = g_last.U()
    lam = g_last.eigs()
    ms = np.sqrt(cfg["mass"])
    t1 = P.csr_matvec(cfg["Z"], x0) / ms
    t2 = SHIFT * t1 + U @ (lam * (U.T @ t1))
    hx = P.csr_matvec(cfg["Z"], t2 / ms)
    rnorm = float(np.linalg.norm(hx - rhs_h[:, 0]))
    resid = rnorm / float(np.linalg.norm(rhs_h[:, 0]))

    def happly(v):
        a = P.csr_matvec(cfg["Z"], v) / ms
        a = SHIFT * a + U @ (lam * (U.T @ a))
        return P.csr_matvec(cfg["Z"], a / ms)

    v = np.random.default_rng(3).standard_normal(N)
    hnorm = 0.0
    for _ in range(12):                  # power estimate of ||H~||_2
        v = happly(v)
        hnorm = float(np.linalg.norm(v))
        v /= hnorm
    berr = rnorm / (hnorm * float(np.linalg.norm(x0))
                    + float(np.linalg.norm(rhs_h[:, 0])))
    del U

    # roofline of the dominant kernel (largest share of timed device time)
    dom = max(ktimes.items(), key=lambda kv: kv[1][0])
    name, (kms, kn, kbytes) = dom
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs")
    peak_note = "measured (MEASURED_PEAKS.json hbm_gbs)"
    if peak is None:
        peak, peak_note = 6650.0, "fallback 6.65 TB/s"
    achieved = (kbytes / kn) / (kms / kn / 1e3) / 1e9 if kn else None
    # DRAM bytes per launch: the ncu captures give DRAM / algorithmic bytes
    # for the kernel's launch kinds at C2 (profiles/traffic.json); scaled by
    # this run's algorithmic bytes per launch, whose launch widths differ
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            ent = json.load(f).get(name)
        if isinstance(ent, dict) and kn:
            traffic = ent["dram_per_algorithmic"] * kbytes / kn
        elif isinstance(ent, (int, float)):
            traffic = ent
    except (OSError, ValueError, KeyError):
        pass
    tot_ms = sum(v[0] for v in ktimes.values()) or 1.0
    kernels = {k: {"ms": round(v[0], 3), "launches": v[1],
                   "share": round(v[0] / tot_ms, 4),
                   "GBps": round((v[2] / v[1]) / (v[0] / v[1] / 1e3) / 1e9, 1)
                   if v[1] and v[0] > 0 else None}
               for k, v in ktimes.items() if v[1]}

    line = {"metric": METRIC, "value": world * args.steps / elapsed,
            "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (config formulas)",
            "config": workload(cfg),
            "replicas": world,
            "build_s": statistics.mean(build_s),
            "solves_per_s": NRHS / statistics.mean(solve_s),
            "solve_p50_ms": lat[len(lat) // 2],
            "solve_p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
            "solve_residual_model": resid,
            "solve_backward_error": berr,
            "kept": report["kept"], "lam_abs_max": report["lam_abs_max"],
            "next_abs": report["next_abs"], "resid_max": report["resid_max"],
            "zsolve_mean_col_iters": stats["zsolve_mean_col_iters"],
            "t_zsolve_s": stats["t_zsolve"], "t_spmm_s": stats["t_spmm"],
            "roofline": {"kernel": name, "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None,
                         "traffic": traffic, "peak_source": peak_note,
                         "bytes_per_launch": kbytes / kn if kn else None,
                         "launch_ms": kms / kn if kn else None},
            "kernels": kernels, "gpu_launches": launches, "clocks": clk,
            "host_per_job": dict(runtime, **{k: stats[k] for k in (
                "t_build", "t_sketch", "t_zsolve", "t_spmm", "t_orth",
                "t_eig", "t_check")})}

    if not args.no_mixed:
        line["mixed"] = run_mixed_job(args, B, pr, opts, N, g_last, rhs, xout,
                                      L, torch)
    if not args.no_serve:
        line["serving"] = run_serving(args, g_last, N, L)
    if not args.no_e2e:
        line["e2e"] = run_e2e(args, cfg, L, torch, world, dist)
    if rank == 0 and world == 1 and not args.no_configs:
        # the other configurations, one sub-object each (not the headline)
        del g_last
        timers.clear()
        live.clear()
        line["configs"] = {}
        for name, fn in (("c3", run_c3), ("c4", run_c4), ("c5", run_c5)):
            try:
                line["configs"][name] = fn(args)
            except Exception as e:          # reported, not fatal
                line["configs"][name] = {"error": repr(e)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(cfg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _sin_max(U1, U2):
    """Largest principal angle (sine) between two orthonormal column sets."""
    sv = np.linalg.svd(U2.T @ U1, compute_uv=False)
    return float(np.sqrt(max(0.0, 1.0 - float(np.min(sv)) ** 2)))


def accuracy_vs_fp64(g64, g32, x64, x32, c):
    """Errors of a mixed-precision result against the FP64 one on the same
    inputs: eigenvalues (relative to the largest, and per eigenvalue),
    the largest principal angle of the leading 20 eigenvectors, solve
    agreement, logdet relative difference."""
    l64, l32 = g64.eigs(), g32.eigs()
    k = min(len(l64), len(l32))
    d = np.abs(l32[:k] - l64[:k])
    kk = min(20, k)
    U64, U32 = g64.U()[:, :kk], g32.U()[:, :kk]
    ld64, ld32 = g64.logdet(c), g32.logdet(c)
    return {"kept_fp64": int(len(l64)), "kept_mixed": int(len(l32)),
            "eig_err_rel_max": float(d.max() / abs(l64[0])),
            "eig_err_rel_each": float(np.max(d / np.abs(l64[:k]))),
            "subspace_sin_top%d" % kk: _sin_max(U64, U32),
            "solve_rel_diff": float(np.linalg.norm(x32 - x64)
                                    / np.linalg.norm(x64)),
            "logdet_rel_diff": float(abs(ld32 - ld64) / abs(ld64))}


def run_mixed_job(args, B, pr, opts, N, g64, rhs, xout, L, torch):
    """The same job (build + 16-RHS solve + logdet) with LGH_PREC_MIXED:
    FP32 sketch blocks, F-applies and CholQR2 sweeps (FP64 accumulation),
    FP64 Rayleigh-Ritz; Z-solves with FP64 Krylov vectors and an FP32
    V-cycle, to the same Z tolerance.  Timed like the headline (CUDA events, W warm-up
    jobs), errors against the FP64 job's results."""
    Lb = L.load()
    ex = L.exec_opts(rank_cap=RANK, precision=L.PREC_MIXED)
    cs = np.array([SHIFT])
    xm = L.DeviceBlock(N, NRHS)
    x64 = xout.get()

    def job():
        g = L.Glr(B, pr, opts, exec=ex)
        L._chk(Lb.lgh_glr_solve_batch(g.h, 1, cs.ctypes.data_as(L.c_dbl_p),
                                      NRHS, rhs.ptr(), N, xm.ptr(), N),
               "lgh_glr_solve_batch")
        g.logdet(SHIFT)
        return g

    for _ in range(max(1, args.warmup - 2)):
        job()
    torch.cuda.synchronize()
    info0 = pr.info()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    bt, st = [], []
    g = None
    for _ in range(args.steps):
        evs[0].record()
        g = None             # the previous job's object goes first
        g = L.Glr(B, pr, opts, exec=ex)
        evs[1].record()
        L._chk(Lb.lgh_glr_solve_batch(g.h, 1, cs.ctypes.data_as(L.c_dbl_p),
                                      NRHS, rhs.ptr(), N, xm.ptr(), N),
               "lgh_glr_solve_batch")
        g.logdet(SHIFT)
        evs[2].record()
        torch.cuda.synchronize()
        bt.append(evs[0].elapsed_time(evs[1]) / 1e3)
        st.append(evs[1].elapsed_time(evs[2]) / 1e3)
    info1 = pr.info()
    acc = accuracy_vs_fp64(g64, g, x64, xm.get(), SHIFT)
    calls = info1["pc32_calls"] - info0["pc32_calls"]
    out = {"jobs_per_s": 1.0 / (statistics.mean(bt) + statistics.mean(st)),
           "build_s": statistics.mean(bt),
           "solves_per_s": NRHS / statistics.mean(st),
           "pc32_block_solves_per_job": calls / max(1, args.steps)}
    out.update(acc)
    return out


def run_serving(args, g, N, L, rate=None, window=None, slots=None):
    """Continuous batching through the request loop (lgh_server_*) on the
    built object: a seeded Poisson stream at --serve-rate requests/s for
    --serve-s seconds, 60/30/10 solve/sample/logdet, m ~ U{1..64} columns,
    shifts log-uniform in [1e-3, 1e3]; submit-to-done latency per request
    and completed columns per second (first submit to last completion)."""
    rng = np.random.default_rng(2024)
    rate = args.serve_rate if rate is None else rate
    window = args.serve_s if window is None else window
    slots = args.serve_slots if slots is None else slots
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window:
            break
        u = rng.random()
        kind = 0 if u < 0.6 else (1 if u < 0.9 else 2)
        m = int(rng.integers(1, 65))
        c = float(10.0 ** rng.uniform(-3, 3))
        arrivals.append((t, kind, m, c))
    mmax = max(m for _, k, m, _ in arrivals if k != 2)
    pool = np.asfortranarray(rng.standard_normal((N, mmax)))
    sv = L.Server(g, slots=slots)
    ids = []
    t_sub, late = 0.0, 0.0
    t0 = time.perf_counter()
    for ta, kind, m, c in arrivals:
        dt = ta - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        late = max(late, -dt)
        ts = time.perf_counter()
        ids.append(sv.submit(kind, c, None if kind == 2 else pool[:, :m]))
        t_sub += time.perf_counter() - ts
    lat = []
    for i in ids:
        lat.append(sv.wait(i, timeout=600.0)[1])
    t1 = time.perf_counter()
    st = sv.stats()
    sv.close()
    lat.sort()
    cols = sum(m for _, k, m, _ in arrivals if k != 2)
    return {"requests": len(arrivals), "offered_per_s": rate,
            "window_s": window, "slots": slots, "columns": cols,
            "columns_per_s": cols / (t1 - t0),
            "p50_ms": 1e3 * lat[len(lat) // 2],
            "p99_ms": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))],
            "max_ms": 1e3 * lat[-1], "ticks": st["ticks"],
            "loop_s": {k: round(st[k], 4) for k in (
                "t_admit_s", "t_tick_s", "t_harvest_s", "t_up_s",
                "t_down_s")},
            "client": {"span_s": round(t1 - t0, 3),
                       "submit_s": round(t_sub, 4),
                       "max_late_s": round(late, 4)},
            "harvests": st["harvests"],
            "occupancy": round(st["occupancy"], 3),
            "stage_mean_s": {k: round(st[k], 4) for k in (
                "wait_stage_s", "wait_admit_s", "run_s", "copy_out_s")},
            "mix": "60/30/10 solve/sample/logdet, m~U{1..64}, "
                   "c log-uniform [1e-3, 1e3]"}


def run_e2e(args, cfg, L, torch, world, dist):
    """The same jobs through the C ABI from pinned host buffers: every step
    uploads B, Z, mass (lgh_mat_create_csr from host arrays) and the 16
    right-hand sides, builds, solves, reads the solutions and the logdet
    back.  Timed with CUDA events + synchronize, max over ranks."""
    import ctypes
    N = cfg["N"]
    Lb = L.load()
    pin = {}
    for nm in ("B", "Z"):
        for k in ("rowptr", "colidx", "vals"):
            a = torch.from_numpy(np.ascontiguousarray(cfg[nm][k])).pin_memory()
            pin[nm + k] = a
    mass = torch.from_numpy(cfg["mass"].copy()).pin_memory()
    rhs = torch.from_numpy(np.random.default_rng(7).standard_normal(
        (NRHS, N))).pin_memory()
    xh = torch.empty((NRHS, N), dtype=torch.float64).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in pin.values()) \
        + mass.numel() * 8 + rhs.numel() * 8
    d2h = xh.numel() * 8 + 8
    opts = L.glr_opts(ell=ELL, q_power=QPOW, seed=SEED, trunc_rel=0.0,
                      check=1)
    ex = L.exec_opts(rank_cap=RANK)
    cs = np.array([SHIFT])

    def step():
        hB, hZ = ctypes.c_void_p(), ctypes.c_void_p()
        L._chk(Lb.lgh_mat_create_csr(N, pin["Browptr"].data_ptr(),
                                     pin["Bcolidx"].data_ptr(),
                                     pin["Bvals"].data_ptr(), 0,
                                     ctypes.byref(hB)), "create B")
        L._chk(Lb.lgh_mat_create_csr(N, pin["Zrowptr"].data_ptr(),
                                     pin["Zcolidx"].data_ptr(),
                                     pin["Zvals"].data_ptr(), 0,
                                     ctypes.byref(hZ)), "create Z")
        md = mass.to("cuda", non_blocking=True)
        vm = ctypes.c_void_p()
        L._chk(Lb.lgh_vec_create_with_array(N, md.data_ptr(),
                                            ctypes.byref(vm)), "mass")
        hp = ctypes.c_void_p()
        po = L.prior_opts(ksp_rtol=ZRTOL)
        L._chk(Lb.lgh_prior_create_mat(hZ, vm, ctypes.byref(po),
                                       ctypes.byref(hp)), "prior")
        hg = ctypes.c_void_p()
        rep = L.GlrReport()
        L._chk(Lb.lgh_glr_compute_ex(hB, hp, ctypes.byref(opts),
                                     ctypes.byref(ex), ctypes.byref(hg),
                                     ctypes.byref(rep)), "compute")
        rd = rhs.to("cuda", non_blocking=True)
        xd = torch.empty((NRHS, N), dtype=torch.float64, device="cuda")
        L._chk(Lb.lgh_glr_solve_batch(hg, 1, cs.ctypes.data_as(L.c_dbl_p),
                                      NRHS, rd.data_ptr(), N, xd.data_ptr(),
                                      N), "solve_batch")
        xh.copy_(xd, non_blocking=True)
        ld = Lb.lgh_glr_logdet(hg, SHIFT)
        Lb.lgh_glr_destroy(hg)
        Lb.lgh_prior_destroy(hp)
        Lb.lgh_vec_destroy(ctypes.byref(vm))
        Lb.lgh_mat_destroy(ctypes.byref(hB))
        Lb.lgh_mat_destroy(ctypes.byref(hZ))
        return ld

    step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    el = max_over_ranks(e0.elapsed_time(e1) / 1e3, world, "cuda")
    return {"value": world * args.steps / el, "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}


def _events(torch, k):
    return [torch.cuda.Event(enable_timing=True) for _ in range(k)]


def run_c3(args):
    """Config 3: 96^3 3D grid (N = 884736), Z = h L + 16 M (7-point),
    B Gaussian (0.012) x Wendland (0.025), a = 1 + sin sin sin / 2;
    lgh_glr_compute at ell = 200 then lgh_glr_extend by 200 (to 400), in
    mixed precision and in FP64 on the same inputs; build and extend
    seconds and the mixed-vs-FP64 errors.  One JSON line."""
    import torch
    import lgh_b200 as L
    from lgh_b200 import problems as P
    torch.cuda.set_device(0)
    cfg = P.grid_problem("c3")
    N = cfg["N"]
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=ZRTOL))
    opts = L.glr_opts(ell=200, q_power=1, seed=SEED, trunc_rel=0.0, check=1)
    rhs = np.random.default_rng(5).standard_normal(N)
    res = {}
    gs = {}
    for name, prec in (("mixed", L.PREC_MIXED), ("fp64", L.PREC_FP64)):
        ex = L.exec_opts(precision=prec)
        L.Glr(B, pr, L.glr_opts(ell=40, seed=SEED, check=0), exec=ex)  # warm
        ev = _events(torch, 3)
        ev[0].record()
        g = L.Glr(B, pr, opts, exec=ex)
        ev[1].record()
        g.extend(200)
        ev[2].record()
        torch.cuda.synchronize()
        res[name] = {"build_s": ev[0].elapsed_time(ev[1]) / 1e3,
                     "extend_s": ev[1].elapsed_time(ev[2]) / 1e3,
                     "kept": int(len(g.eigs()))}
        gs[name] = g
    x64 = gs["fp64"].solve(1.0, rhs)
    x32 = gs["mixed"].solve(1.0, rhs)
    res["mixed_vs_fp64"] = accuracy_vs_fp64(gs["fp64"], gs["mixed"], x64, x32,
                                            1.0)
    line = {"metric": "GLR build + extend seconds (ell 200 -> 400)",
            "value": res["mixed"]["build_s"] + res["mixed"]["extend_s"],
            "unit": "s", "higher_is_better": False, "n_gpus": 1,
            "dtype": "f32 blocks / f64 core (mixed)",
            "data": "synthetic (config formulas)",
            "config": {"workload": "c3: 96^3 3D grid (N=%d), B %.1f nnz/row, "
                                   "Z = h L + 16 M (7-point), ell 200 then "
                                   "extend 200, q=1, Z rtol %g"
                                   % (N, cfg["nnz_B"] / N, ZRTOL),
                       "N": N, "nnz_B": cfg["nnz_B"]},
            "results": res}
    return line


def run_c4(args):
    """Config 4: the C2 operator built once at ell = 420 (rank cap 400),
    then 64 shifts log-spaced in [1e-3, 1e3] x 256 N(0,1) right-hand sides
    through lgh_glr_solve_batch and lgh_glr_sample_batch (shift-independent
    Z-solves once, per-shift Woodbury combinations), and logdet at all 64
    shifts; FP64 and mixed.  Right-hand-side columns per second.  One JSON
    line."""
    import torch
    import lgh_b200 as L
    from lgh_b200 import problems as P
    torch.cuda.set_device(0)
    cfg = P.grid_problem(CONFIG)
    N = cfg["N"]
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=ZRTOL))
    cs = np.logspace(-3, 3, 64)
    m = 256
    R = L.DeviceBlock(N, m, np.random.default_rng(8).standard_normal((N, m)))
    Xo = L.DeviceBlock(N, m * len(cs))
    Lb = L.load()
    res = {}
    for name, prec in (("fp64", L.PREC_FP64), ("mixed", L.PREC_MIXED)):
        ex = L.exec_opts(precision=prec, rank_cap=400)
        g = L.Glr(B, pr, L.glr_opts(ell=420, seed=SEED, trunc_rel=0.0,
                                    check=0), exec=ex)
        csp = cs.ctypes.data_as(L.c_dbl_p)
        ld = np.empty_like(cs)
        # the first multi-shift call forms W = Z^{-1} M^{1/2} U once per
        # build (kept Z-solves); timed on its own and reported beside the
        # per-call throughput
        ew = _events(torch, 2)
        ew[0].record()
        L._chk(Lb.lgh_glr_solve_batch(g.h, 2, csp, 8, R.ptr(), N, Xo.ptr(),
                                      N), "warm")
        ew[1].record()
        torch.cuda.synchronize()
        w_s = ew[0].elapsed_time(ew[1]) / 1e3
        # the first call of the full shape tunes the combination's tile
        L._chk(Lb.lgh_glr_solve_batch(g.h, len(cs), csp, m, R.ptr(), N,
                                      Xo.ptr(), N), "tune")
        L._chk(Lb.lgh_glr_sample_batch(g.h, len(cs), csp, m, R.ptr(), N,
                                       Xo.ptr(), N), "tune")
        torch.cuda.synchronize()
        # three repetitions of each operation; the median is reported
        reps = {"s": [], "p": [], "l": []}
        for _ in range(3):
            ev = _events(torch, 4)
            ev[0].record()
            L._chk(Lb.lgh_glr_solve_batch(g.h, len(cs), csp, m, R.ptr(), N,
                                          Xo.ptr(), N), "solve_batch")
            ev[1].record()
            L._chk(Lb.lgh_glr_sample_batch(g.h, len(cs), csp, m, R.ptr(), N,
                                           Xo.ptr(), N), "sample_batch")
            ev[2].record()
            L._chk(Lb.lgh_glr_logdet_batch(g.h, len(cs), csp,
                                           ld.ctypes.data_as(L.c_dbl_p)),
                   "ld")
            ev[3].record()
            torch.cuda.synchronize()
            reps["s"].append(ev[0].elapsed_time(ev[1]) / 1e3)
            reps["p"].append(ev[1].elapsed_time(ev[2]) / 1e3)
            reps["l"].append(ev[2].elapsed_time(ev[3]))
        ts = float(np.median(reps["s"]))
        tp = float(np.median(reps["p"]))
        res[name] = {"kept": int(len(g.eigs())), "w_precompute_s": w_s,
                     "batch_info": g.batch_info(), "solve_s": ts,
                     "sample_s": tp,
                     "logdet_64_ms": float(np.median(reps["l"])),
                     "solve_cols_per_s": m * len(cs) / ts,
                     "sample_cols_per_s": m * len(cs) / tp,
                     "solve_s_each": [round(x, 4) for x in reps["s"]]}
        del g
    line = {"metric": "batched solve columns/s (64 shifts x 256 RHS)",
            "value": res["mixed"]["solve_cols_per_s"], "unit": "columns/s",
            "higher_is_better": True, "n_gpus": 1,
            "dtype": "f32 sweeps / f64 core (mixed); fp64 beside",
            "data": "synthetic (config formulas)",
            "config": {"workload": "c4: c2 operator, ell 420 (rank 400), "
                                   "64 shifts log-spaced [1e-3, 1e3] x 256 "
                                   "RHS, solve + sample + logdet",
                       "N": N},
            "results": res}
    return line


def run_c5(args):
    """Config 5: 128^3 3D grid (N = 2097152), Z = h L + 16 M, B Gaussian
    (0.01) x Wendland (0.02); GLR rank 500 (ell 520, rank cap 500) built in
    mixed precision and kept resident; then seeded Poisson request streams
    (60/30/10 solve/sample/logdet, m ~ U{1..64}, c log-uniform in
    [1e-3, 1e3]) through the request loop at each rate of --serve-rates;
    p50 / p99 latency and completed columns per second.  One JSON line."""
    import torch
    import lgh_b200 as L
    from lgh_b200 import problems as P
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    cfg = P.grid_problem("c5")
    t_gen = time.perf_counter() - t0
    N = cfg["N"]
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=ZRTOL))
    ex = L.exec_opts(precision=L.PREC_MIXED, rank_cap=500)
    ev = _events(torch, 2)
    ev[0].record()
    g = L.Glr(B, pr, L.glr_opts(ell=520, q_power=1, seed=SEED,
                                trunc_rel=0.0, check=0), exec=ex)
    ev[1].record()
    torch.cuda.synchronize()
    build_s = ev[0].elapsed_time(ev[1]) / 1e3
    rates = [float(r) for r in (args.serve_rates or "2,5,10").split(",")]
    sweep = [run_serving(args, g, N, L, rate=r, window=args.serve_s)
             for r in rates]
    line = {"metric": "served columns/s and p50/p99 request latency",
            "value": max(x["columns_per_s"] for x in sweep),
            "unit": "columns/s", "higher_is_better": True, "n_gpus": 1,
            "dtype": "f32 blocks / f64 core (mixed)",
            "data": "synthetic (config formulas)",
            "config": {"workload": "c5: 128^3 3D grid (N=%d), B %.1f nnz/row, "
                                   "ell 520 (rank 500), Poisson request "
                                   "streams at %s requests/s" % (
                                       N, cfg["nnz_B"] / N, rates),
                       "N": N, "nnz_B": cfg["nnz_B"]},
            "generate_s": t_gen, "build_s": build_s,
            "kept": int(len(g.eigs())), "sweep": sweep}
    return line


def rows_case(L, cfg, ell, rtol, nranks):
    """The build over row slabs against the one-rank build of the same
    operators: per-column PCG iterations (the rank-local block-Jacobi
    preconditioner against the global V-cycle), halo exchanges and bytes,
    all-reduce count, spectrum agreement, and the wall time with the ranks
    as threads sharing one GPU."""
    import threading
    N = cfg["N"]
    gopts = L.glr_opts(ell=ell, seed=0, trunc_rel=0.0)
    popts = L.prior_opts(ksp_rtol=rtol)
    pr = L.Prior(Z=L.Mat(cfg["Z"]), mass=cfg["mass"], opts=popts)
    t0 = time.time()
    g1 = L.Glr(L.Mat(cfg["B"]), pr, gopts)
    one = {"build_s": round(time.time() - t0, 3),
           "mean_col_iters": round(pr.info()["mean_col_iters"], 2)}
    lam1 = g1.eigs().copy()
    del g1, pr
    comms = L.local_rows_comms(nranks)
    res, errs = [None] * nranks, []

    def rank(r):
        try:
            a, b = L.shard_range(N, nranks, r)
            Bm = L.Mat(L.rows_slab(cfg["B"], a, b), rows=(N, comms[r]))
            Zm = L.Mat(L.rows_slab(cfg["Z"], a, b), rows=(N, comms[r]))
            p = L.Prior(Z=Zm, mass=cfg["mass"][a:b], opts=popts)
            g = L.Glr(Bm, p, gopts)
            res[r] = {"rows": b - a, "ghosts_B": Bm.rows_info()[2],
                      "ghosts_Z": Zm.rows_info()[2],
                      "halo_B": Bm.rows_traffic()[:2],
                      "halo_Z": Zm.rows_traffic()[:2],
                      "mean_col_iters": p.info()["mean_col_iters"],
                      "lam": g.eigs().copy()}
            del g, p, Bm, Zm
        except Exception as e:
            errs.append(repr(e))

    t0 = time.time()
    ts = [threading.Thread(target=rank, args=(r,)) for r in range(nranks)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    wall = time.time() - t0
    L.free_local_rows_comms(comms)
    if errs:
        raise RuntimeError(errs)
    lam = res[0]["lam"]
    return {"one_rank": one,
            "slabs": {"ranks": nranks, "wall_s_threads_one_gpu": round(wall, 3),
                      "mean_col_iters": round(res[0]["mean_col_iters"], 2),
                      "per_rank": [{k: v for k, v in r.items() if k != "lam"}
                                   for r in res],
                      "lam_max_abs_diff_rel": float(
                          np.abs(lam - lam1).max() / np.abs(lam1).max()),
                      "kept": int(len(lam))}}


def run_kernel_case(args):
    """One device case through the C ABI with the per-kernel event
    registry on; prints the wall time and each kernel's launches, time and
    achieved bandwidth (algorithmic bytes / event time)."""
    import lgh_b200 as L
    from lgh_b200 import problems as P
    L.load()
    cfg = P.grid_problem(args.kc_config)
    N, w = cfg["N"], args.kc_width
    L.kernel_timing(True)
    t0 = time.time()
    if args.kernel_case == "zsolve":
        Z = L.Mat(cfg["Z"])
        pr = L.Prior(Z=Z, mass=cfg["mass"],
                     opts=L.prior_opts(ksp_rtol=args.kc_rtol))
        X = np.random.default_rng(0).standard_normal((N, w))
        L.test_zsolve(pr, X, fp32=args.kc_fp32)
        info = pr.info()
    elif args.kernel_case == "spmm":
        B = L.Mat(cfg["B"])
        X = np.random.default_rng(0).standard_normal((N, w))
        L.test_spmm(B, X, fp32=args.kc_fp32)
        info = {}
    elif args.kernel_case == "batch":
        # many-shift batched solves (w right-hand sides, --kc-shifts
        # shifts) on an FP64 and a mixed object: the fused combination
        # kernels, timed per call after a tuning call and a graph capture
        import torch
        B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
        pr = L.Prior(Z=Z, mass=cfg["mass"],
                     opts=L.prior_opts(ksp_rtol=args.kc_rtol))
        ell = args.kc_rank
        cs = np.logspace(-3, 3, args.kc_shifts)
        R = L.DeviceBlock(N, w, np.random.default_rng(8).standard_normal(
            (N, w)))
        Xo = L.DeviceBlock(N, w * len(cs))
        Lb = L.load()
        info = {}
        for name, prec in (("fp64", L.PREC_FP64), ("mixed", L.PREC_MIXED)):
            g = L.Glr(B, pr, L.glr_opts(ell=ell, seed=0, trunc_rel=0.0,
                                        check=0),
                      exec=L.exec_opts(precision=prec, rank_cap=ell - 20))
            ts = []
            for _ in range(4):
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ev[0].record()
                L._chk(Lb.lgh_glr_solve_batch(
                    g.h, len(cs), cs.ctypes.data_as(L.c_dbl_p), w, R.ptr(),
                    N, Xo.ptr(), N), "solve_batch")
                ev[1].record()
                torch.cuda.synchronize()
                ts.append(ev[0].elapsed_time(ev[1]))
            info[name] = {"call_ms": [round(t, 3) for t in ts],
                          "batch": g.batch_info()}
            del g
    elif args.kernel_case == "rows":
        info = rows_case(L, cfg, w, args.kc_rtol, args.kc_ranks)
    else:
        B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
        pr = L.Prior(Z=Z, mass=cfg["mass"],
                     opts=L.prior_opts(ksp_rtol=args.kc_rtol))
        g = L.Glr(B, pr, L.glr_opts(ell=w, seed=0, trunc_rel=0.0))
        info = g.stats()
    dt = time.time() - t0
    print("case %s %s w=%d: %.3f s  %s" % (args.kernel_case, args.kc_config,
                                           w, dt, info))
    for k, (ms, n, by) in L.kernel_timing_get().items():
        if n:
            print("  %-24s launches %7d  %9.3f ms  %8.3f ms/launch  %7.1f "
                  "GB/s" % (k, n, ms, ms / n, by / n / (ms / n / 1e3) / 1e9))
    return 0


def main():
    args = parse()
    if args.kernel_case:
        return run_kernel_case(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.config in ("c3", "c4", "c5"):
        fn = {"c3": run_c3, "c4": run_c4, "c5": run_c5}[args.config]
        print(json.dumps(fn(args)), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""Benchmark: mode-solves/s of the batched 2D Helmholtz/Poisson
diagonalisation solve (duct's helm3d hot path) on B200.

Workload (one "step"): the four solves of one RK3/CN substep of the square
duct at my = mz = 129 (n = 127 interior points), 64 Fourier modes k = 0..63
with kx = 0.5 k (Lx = 4 pi): u, v, w Dirichlet with lambda = kx^2 + 2/(nu dt)
(nu = 1/2000, dt = 1e-3) and the pressure Poisson problem, Neumann with
lambda = kx^2 (kx = 0 singular, pinned as the reference does).  That is
256 mode-solves per step on seeded synthetic complex128 right-hand sides.

Arms:
* default: the device-resident batched solve (ductgpu_solve_fields_dev) with
  inputs in HBM, replayed from the library's CUDA graphs of the step (one per
  rotating input set); the per-kernel durations behind ``roofline`` come
  from a second run of the same steps with a CUDA event pair around every
  launch.  ``roofline.achieved`` counts the algorithm's flops (the
  reference's full n x n GEMMs, 4 n^3 a plane and pass); the flip-symmetric
  kernel executes half of them (``roofline.executed``), so its fraction of
  the DGEMM peak can read above 1.  ``e2e`` times the reference-facing host-array entry
  (ductgpu_helm3d_batch: H2D + solve + D2H of the four fields, copies
  overlapped with the solves) for the same work.
* ``--impl reference``: the reference's CPU algorithm (the oracle's
  restatement of helm3d/solvediag with the same LAPACK/BLAS calls) on all
  host cores; under torchrun rank 0 alone runs it and prints the line.

Several GPUs (``--gpus N`` under torchrun, one rank per GPU): replicas only
-- every rank solves its own copy of the step (no exchange: Fourier modes
are independent), ``value`` is all ranks' mode-solves over the slowest
rank's time (max over ranks), ``scaling`` weak.  NCCL carries the barrier
and the max on GPUs; without a GPU the same host logic runs over gloo.
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
sys.path.insert(0, ROOT)

METRIC = "mode-solves/s (batched 2D Helmholtz/Poisson diagonalisation solve)"
UNIT = "mode-solves/s"
WORKLOAD = "cfg1: square duct my=mz=129, 64 Fourier modes x 4 fields (u,v,w Dirichlet + pressure Neumann)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed", "int8"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-transforms", action="store_true")
    ap.add_argument("--no-dns", action="store_true", help="skip the config-4 DNS steps/s block")
    ap.add_argument("--dns-only", action="store_true",
                    help="only the config-4 DNS block (one GPU; with --dns-steps for short profiling runs)")
    ap.add_argument("--dns-steps", type=int, default=None, help="timed DNS steps (default: the config's 200)")
    ap.add_argument("--pass-kernel", default="auto",
                    choices=["auto", "staged-32", "staged-16", "register", "persist", "parity", "parity-queue"],
                    help="GEMM-pass kernel; auto runs the library's autotuner (profiling runs fix it, since "
                         "the autotuner's timing under a profiler is not the live one)")
    ap.add_argument("--transforms-only", action="store_true",
                    help="only the HBM-bound kernels (transyz, derivyz, transposes) on one GPU")
    return ap.parse_args()


def workload():
    from duct_b200 import synth
    c = synth.config("cfg1")
    m, nm = c["my"], c["nmodes"]
    xalp = c["alp"] * np.arange(nm)
    rhs = [synth.chebyshev_rhs(m, m, nm, seed=1 + i, ib=0) for i in range(len(c["fields"]))]
    return c, m, nm, xalp, rhs


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9
                          for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_setup(args, backend=None, timeout_s=120):
    """One process per GPU from the launcher's environment (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_ADDR/PORT).  NCCL on GPUs, gloo without one (the
    multi-rank host logic is tested that way on CPU); the timeout ends a
    collective that a departed rank never joins with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, v):
    """The slowest rank's time: every multi-GPU number is the max over ranks."""
    if pg is None:
        return v
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_rate(c, m, xalp, rhs, budget_s=10.0, max_iters=None):
    """The reference CPU algorithm (oracle restatement, same LAPACK/BLAS
    calls) on every host core: mode-solves/s over whole cfg1 batches."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_blas_threads(1)
    ops = O.Ops(m)
    nm = len(xalp)
    done, t0 = 0, time.perf_counter()
    it = 0
    while True:
        for (name, bound, lam), f in zip(c["fields"], rhs):
            O.helm3d(f, ops, bound, lam, xalp, nthreads=threads)
            done += nm
        it += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_iters and it >= max_iters):
            break
    return done / el, threads, done, el


def run_reference(args, world, rank):
    if rank != 0:
        return
    c, m, nm, xalp, rhs = workload()
    per_step = nm * len(c["fields"])
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_blas_threads(1)
    ops = O.Ops(m)

    def step():
        for (name, bound, lam), f in zip(c["fields"], rhs):
            O.helm3d(f, ops, bound, lam, xalp, nthreads=threads)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    v = per_step * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded splitmix64 Chebyshev-coefficient RHS)",
        "config": {"workload": WORKLOAD, "mode_solves_per_step": per_step},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "%d full cfg1 batches (%d mode-solves each)" % (args.steps, per_step)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local, pg):
    import duct_b200 as D
    c, m, nm, xalp, rhs = workload()
    n = m - 2
    nf = len(c["fields"])
    per_step = nm * nf
    ctx = D.Context(local)
    ctx.pseudomat(m)

    # two rotating input/output sets: 2 x 4 x 2 x 17 MB = 272 MB > 126 MB L2
    sets = []
    for s in range(2):
        fl = []
        for (name, bound, lam), f in zip(c["fields"], rhs):
            r = ctx.device_array(f.shape)
            o = ctx.device_array(f.shape)
            r.upload(f)
            fl.append(dict(rhs=r, sol=o, xalp=xalp, alambda=lam, ib=0, bound=bound))
        sets.append(fl)

    # the library's autotuner picks the GEMM-pass kernel for this batch
    names = {D.PASS_STAGED: "staged-32", D.PASS_STAGED16: "staged-16", D.PASS_REGISTER: "register",
             D.PASS_PERSIST: "persist", D.PASS_PARITY: "parity", D.PASS_PARITY_QUEUE: "parity-queue"}
    if args.pass_kernel == "auto":
        pass_id = ctx.autotune(sets[0], reps=5)
    else:
        pass_id = {v: k for k, v in names.items()}[args.pass_kernel]
        ctx.set_pass_kernel(pass_id)
    pass_kernel = names[pass_id]

    def timed(prec):
        # The step is replayed from CUDA graphs of the batched solve, one per
        # rotating input set (the library's path for a repeated substep);
        # direct calls if the precision's solve cannot be captured.
        try:
            graphs = [ctx.graph_create(sets[s], precision=prec) for s in range(2)]
        except D.DuctGPUError:
            graphs = None

        def step(i):
            if graphs:
                ctx.graph_launch(graphs[i % 2])
            else:
                ctx.solve_fields_dev(sets[i % 2], prec)

        for i in range(args.warmup):
            step(i)
        ctx.synchronize()
        barrier(pg)
        clocks = ClockSampler(local)
        clocks.start()
        ctx.event_record(0)
        for i in range(args.steps):
            step(i)
        ctx.event_record(1)
        ms = ctx.event_elapsed(0, 1)
        ctx.synchronize()
        clk = clocks.stop()
        ms = max_over_ranks(pg, ms)
        barrier(pg)
        # Kernel durations for the roofline: the same steps as direct calls
        # with a CUDA event pair around every launch (a second timed region;
        # the events add gaps between launches, so the step time above is
        # taken without them).
        ctx.profile(True)
        ctx.profile_reset()
        l0 = ctx.launch_count()
        ctx.event_record(0)
        for i in range(args.steps):
            ctx.solve_fields_dev(sets[i % 2], prec)
        ctx.event_record(1)
        ms_prof = ctx.event_elapsed(0, 1)
        ctx.synchronize()
        launches = ctx.launch_count() - l0
        prof = {k: ctx.profile_read(k) for k in (D.K_PASS_FP64, D.K_MIXED_GEMM, D.K_NEUMANN, D.K_WALLS, D.K_RESIDUAL)}
        ctx.profile(False)
        if graphs:
            for g in graphs:
                ctx.graph_destroy(g)
        barrier(pg)
        return ms / args.steps, launches, prof, clk, ms_prof, bool(graphs)

    want = ["fp64", "mixed", "int8"] if args.precision == "auto" else [args.precision]
    res = {}
    for name in want:
        prec = {"fp64": D.PREC_FP64, "mixed": D.PREC_MIXED, "int8": D.PREC_INT8}[name]
        ms_step, launches, prof, clk, ms_prof, graph = timed(prec)
        res[name] = dict(ms_step=ms_step, launches=launches, prof=prof, clk=clk, ms_prof=ms_prof,
                         graph=graph, value=world * per_step / (ms_step * 1e-3))
    # accuracy of the split paths against the FP64 passes on the same (full)
    # operators, which the split paths emulate; the flip-symmetric passes are
    # another decomposition of the operator (checked against the oracle by
    # tests/test_gpu_parity.py)
    ctx.set_pass_kernel(D.PASS_STAGED)
    acc8 = None
    if "int8" in res and "fp64" in res:
        ctx.solve_fields_dev(sets[0], D.PREC_FP64)
        ref8 = [f["sol"].download() for f in sets[0]]
        ctx.solve_fields_dev(sets[0], D.PREC_INT8)
        acc8 = {name: float(np.linalg.norm(f["sol"].download() - r) / np.linalg.norm(r))
                for (name, _, _), f, r in zip(c["fields"], sets[0], ref8)}
    acc = None
    if "mixed" in res and "fp64" in res:
        ctx.solve_fields_dev(sets[0], D.PREC_FP64)
        ref = [f["sol"].download() for f in sets[0]]
        ctx.solve_fields_dev(sets[0], D.PREC_MIXED)
        acc = {}
        for (name, bound, lam), f, r in zip(c["fields"], sets[0], ref):
            a = f["sol"].download()
            if bound == "n":          # singular kx=0 plane: compare modulo a constant
                a[:, :, 0] -= a[:, :, 0].mean()
                r = r.copy()
                r[:, :, 0] -= r[:, :, 0].mean()
            acc[name] = float(np.linalg.norm(a - r) / np.linalg.norm(r))
    ctx.set_pass_kernel(pass_id)
    best = max(res, key=lambda k: res[k]["value"])
    B = res[best]
    peak64, peak64_note = fp64_peak()
    peak16 = bf16_peak()
    roofs = {}
    for name, R in res.items():
        if name == "fp64":
            kms, kn = R["prof"][D.K_PASS_FP64]
            if pass_kernel == "parity-queue":
                # one launch runs the four flip-symmetric passes of the step
                he, ho = (n + 1) // 2, n // 2
                flops = 4 * 4.0 * n * (he * he + ho * ho) * per_step
                kname = "k_pass_fp64q (the four flip-symmetric passes in one persistent launch, FP64 DMMA m16n8k16)"
                traffic = None
            elif pass_kernel == "parity":
                # even and odd half blocks (ceil(n/2), floor(n/2)) on 2n real
                # columns per plane: the flops the flip-symmetric pass executes
                he, ho = (n + 1) // 2, n // 2
                flops = 4.0 * n * (he * he + ho * ho) * per_step
                # the library's rule: the warp-specialised persistent kernel
                # for half blocks of 32 / 64 rows and >= 6 16-line tiles per SM
                tiles = per_step * ((n + 15) // 16)
                if ((he + 31) // 32) * 32 <= 64 and tiles >= 6 * torch_sm_count():
                    kname = "k_pass_fp64w (flip-symmetric half blocks, warp-specialised persistent, FP64 DMMA m16n8k16)"
                    traffic = traffic_from_profile("k_pass_fp64w")
                else:
                    kname = "k_pass_fp64s (flip-symmetric half blocks, FP64 DMMA m16n8k16)"
                    traffic = traffic_from_profile("k_pass_fp64s")
            else:
                flops = 4.0 * n ** 3 * per_step          # n x n operator on 2n real columns per plane
                kname = "k_pass_fp64 (FP64 DMMA m16n8k16)"
                traffic = traffic_from_profile("k_pass_fp64")
            # algorithmic flops: the reference's full n x n GEMMs (4 n^3 a plane
            # and pass; a single-launch kernel runs four passes a launch)
            alg = 4.0 * n ** 3 * per_step * (4 if pass_kernel == "parity-queue" else 1)
            t_launch = (kms / kn) * 1e-3 if kn else None
            ach = alg / t_launch / 1e12 if kn else None
            exe = flops / t_launch / 1e12 if kn else None
            roofs[name] = {"bound": "tensor", "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                           "frac": (ach / peak64) if (ach and peak64) else None,
                           "flops_per_launch": alg,
                           "note": "algorithmic flops (the reference's full-operator GEMMs) over the kernel's "
                                   "event-timed launch; the flip-symmetric kernel executes half of them",
                           "executed": {"achieved": exe, "frac": (exe / peak64) if (exe and peak64) else None,
                                        "flops_per_launch": flops},
                           "traffic": traffic,
                           "kernel": kname, "peak_source": peak64_note,
                           "kernel_share_of_step": kms / R["ms_prof"]}
        elif name == "int8":
            kms, kn = R["prof"][D.K_MIXED_GEMM]
            # per launch: 28 slice products of the padded 128 x 128 operator
            # against 256 real columns (128 padded lines x re/im) per plane
            ops = 28 * 2.0 * 128 * 128 * 256 * per_step
            ach = ops / ((kms / kn) * 1e-3) / 1e12 if kn else None
            roofs[name] = {"bound": "tensor", "achieved": ach, "peak": 4500.0, "unit": "TOPS (int8)",
                           "frac": (ach / 4500.0) if ach else None,
                           "traffic": traffic_from_profile("k_pass_i8ws"),
                           "kernel": "k_pass_i8ws (tcgen05 kind::i8, 28 slice products, exact int32)",
                           "peak_source": "nominal dense int8 (no measured int8 peak on this pool)",
                           "fp64_equiv_tflops": (4.0 * n ** 3 * per_step) / ((kms / kn) * 1e-3) / 1e12 if kn else None,
                           "kernel_share_of_step": kms / R["ms_prof"]}
        else:
            kms, kn = R["prof"][D.K_MIXED_GEMM]
            flops = 10 * 4.0 * n ** 3 * per_step     # 10 BF16 slice products per pass
            ach = flops / ((kms / kn) * 1e-3) / 1e12 if kn else None
            roofs[name] = {"bound": "tensor", "achieved": ach, "peak": peak16, "unit": "TFLOP/s",
                           "frac": (ach / peak16) if (ach and peak16) else None,
                           "traffic": traffic_from_profile("k_pass_mixed"),
                           "kernel": "k_pass_mixed (tcgen05 kind::f16, BF16 slices)",
                           "peak_source": "measured cuBLAS bf16 burst (MEASURED_PEAKS.json)",
                           "kernel_share_of_step": kms / R["ms_prof"]}

    e2e = None
    if not args.no_e2e:
        prec = {"fp64": D.PREC_FP64, "mixed": D.PREC_MIXED, "int8": D.PREC_INT8}[best]
        e2e = measure_e2e(ctx, c, m, nm, xalp, rhs, prec, args, pg, world)

    hbm = transform_rates(ctx) if (rank == 0 and not args.no_transforms) else None
    cfg2 = uneven_rect_rate(ctx, args) if not args.no_transforms else None
    cfg4 = None
    if not args.no_dns and rank == 0:
        cfg4 = dns_cfg4(args, local, world == 1 and not args.no_cpu)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, threads, done, el = cpu_reference_rate(c, m, xalp, rhs, budget_s=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": "%d mode-solves (whole cfg1 batches) in %.1f s" % (done, el)}
        parity = parity_vs_oracle(ctx, c, m, xalp, rhs, sets, list(res), local)

    for fl in sets:
        for f in fl:
            f["rhs"].free()
            f["sol"].free()
    ctx.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": B["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": B["ms_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "mixed": "bf16-split+f64-refine", "int8": "int8-split (7x7 slices, exact int32)"}[best],
            "data": "synthetic (seeded splitmix64 Chebyshev-coefficient RHS)",
            "config": {"workload": WORKLOAD, "mode_solves_per_step": per_step,
                       "precision": best,
                       "parallelism": "replicas" if world > 1 else "1gpu",
                       "l2": "2 rotating input/output sets (272 MB) > 126 MB L2",
                       "pass_kernel": pass_kernel,
                       "step": ("CUDA-graph replay of ductgpu_solve_fields_dev (one graph per rotating set)"
                                if B["graph"] else "ductgpu_solve_fields_dev calls"),
                       "kernel_timing": "per-launch CUDA events in a second run of the same steps"},
            "gpu_launches": B["launches"],
            "roofline": roofs[best], "cpu_baseline": cpu, "e2e": e2e, "clocks": B["clk"],
            "paths": {k: {"value": v["value"], "ms_per_step": v["ms_step"], "roofline": roofs[k],
                          "gpu_launches": v["launches"], "graph": v["graph"]} for k, v in res.items()},
            "parity": parity,
            "mixed_rel_err_vs_fp64": acc,
            "int8_rel_err_vs_fp64": acc8,
            "hbm_kernels": hbm,
            "cfg2_uneven_rect_batch": cfg2,
            "cfg4_dns": cfg4,
        }
        print(json.dumps(line), flush=True)


def _errs(a, b):
    """Relative error of a against b: 2-norm over all points and max-norm
    (absolute where b is zero)."""
    d = (np.asarray(a) - np.asarray(b)).ravel()
    nb, mb = np.linalg.norm(np.asarray(b).ravel()), np.abs(b).max()
    return {"l2": float(np.linalg.norm(d) / nb) if nb > 0 else float(np.linalg.norm(d)),
            "max": float(np.abs(d).max() / mb) if mb > 0 else float(np.abs(d).max())}


def _exact_interior(F, B, P, Q, E, lam, io=None, iters=4):
    """The solution of the FP64 discrete interior operator B(x)I + I(x)B - lam
    by iterative refinement with long-double residuals (the FP64
    diagonalisation as the preconditioner), pinned at interior point io
    like the reference's kx=0 mode."""
    Bl = B.astype(np.longdouble)
    U = np.zeros_like(F, dtype=np.longdouble)
    den = E[:, None] + E[None, :] - lam
    if io is not None:
        den[io, io] = np.inf
    for _ in range(iters):
        R = (F.astype(np.longdouble) - (Bl @ U + U @ Bl.T - lam * U)).astype(np.float64)
        d = P @ ((Q @ R @ Q.T) / den) @ P.T
        if io is not None:
            d = d - d[io, io] * np.outer(P[:, io], P[:, io]) / P[io, io] ** 2
        U = U + d.astype(np.longdouble)
    return U.astype(np.float64)


def parity_vs_oracle(ctx, c, m, xalp, rhs, sets, paths, device):
    """The relative error of every path's result against the oracle (the
    reference's CPU algorithm, same LAPACK calls), per field, at cfg1 and
    cfg0.  The kx=0 pressure is compared in the reference's gauge: the
    pinned point U(iofzero+1, iofzero+1) with iofzero from the host's
    LAPACK order, which the caller passes (ductgpu_set_gauge_point).  Two
    operator sources: the library's own eigen-decomposition (the default
    drop-in) and the host's LAPACK operators imported on a grid-only set-up
    (ductgpu_pseudomat_ex + ductgpu_set_operators).  For the Neumann field,
    whose own-operator error is set by FP64 rounding of the eigenvectors,
    the error of both the GPU and the oracle against an extended-precision
    solution of the same discrete operator is given on a subset of modes."""
    import duct_b200 as D
    from duct_b200 import synth
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    ops = O.Ops(m)
    refs = [O.helm3d(f, ops, bound, lam, xalp, nthreads=threads)[0] for (_, bound, lam), f in zip(c["fields"], rhs)]
    precs = {"fp64": D.PREC_FP64, "mixed": D.PREC_MIXED, "int8": D.PREC_INT8}
    out = {"reference": "oracle helm3d (LAPACK dgeev/dgetrf/dgetri + dgemm), same seeded inputs",
           "gauge": "kx=0 pressure pinned at U(iofzero+1,iofzero+1)=0, iofzero=%d from the host LAPACK order "
                    "(ductgpu_set_gauge_point)" % ops.iofzero,
           "cfg1": {}}

    def solve_all(cx, prec):
        for f, (name, bound, lam), r in zip(sets[0], c["fields"], rhs):
            f["rhs"].upload(r)
        cx.solve_fields_dev(sets[0], prec)
        cx.synchronize()
        return [f["sol"].download() for f in sets[0]]

    ctx.set_gauge_point(ops.iofzero)
    own = {}
    for name in paths:
        got = solve_all(ctx, precs[name])
        own[name] = got
        out["cfg1"]["%s_own_operators" % name] = {fn: _errs(g, r) for (fn, _, _), g, r in zip(c["fields"], got, refs)}
    ctx.set_gauge_point(0)
    # the host's LAPACK operators on a grid-only set-up
    with D.Context(device) as c2:
        c2.pseudomat_ex(m, D.SETUP_NO_EIGEN)
        c2.set_operators("d", ops.ED, ops.PD, ops.PDM1)
        c2.set_operators("n", ops.EN, ops.PN, ops.PNM1, ops.iofzero)
        got = solve_all(c2, D.PREC_FP64)
        out["cfg1"]["fp64_lapack_operators"] = {fn: _errs(g, r) for (fn, _, _), g, r in zip(c["fields"], got, refs)}
    # accuracy of the Neumann field against the extended-precision solution
    ip = [i for i, (_, b, _) in enumerate(c["fields"]) if b == "n"]
    if ip and own:
        i = ip[0]
        lam0 = c["fields"][i][2]
        E, P, Q = np.asarray(ops.EN), np.asarray(ops.PN), np.asarray(ops.PNM1)
        io = ops.iofzero - 1
        sub = [k for k in (0, 1, 2, 8, 32, len(xalp) - 1) if k < len(xalp)]
        err = {name: 0.0 for name in own}
        eo, nrm = 0.0, 0.0
        for k in sub:
            lam = lam0 + xalp[k] ** 2
            F = rhs[i][1:-1, 1:-1, k]
            for part in (np.real, np.imag):
                Fk = np.ascontiguousarray(part(F))
                if not np.any(Fk):
                    continue
                X = _exact_interior(Fk, np.asarray(ops.D2Bn), P, Q, E, lam, io if abs(lam) < 1e-10 else None)
                for name in own:
                    err[name] += np.sum((part(own[name][i][1:-1, 1:-1, k]) - X) ** 2)
                eo += np.sum((part(refs[i][1:-1, 1:-1, k]) - X) ** 2)
                nrm += np.sum(X ** 2)
        pe = {"modes": sub, "oracle_l2": float(np.sqrt(eo / nrm)),
              "solution": "long-double-residual iterative refinement of the FP64 Neumann interior operator"}
        for name in own:
            pe["gpu_%s_own_operators_l2" % name] = float(np.sqrt(err[name] / nrm))
        out["cfg1"]["p_vs_extended_precision"] = pe
    # cfg0: 33^2, 17 modes, Dirichlet, lambda = kx^2 + 4e6
    c0 = synth.config("cfg0")
    m0, nm0 = c0["my"], c0["nmodes"]
    x0 = c0["alp"] * np.arange(nm0)
    ops0 = O.Ops(m0)
    r0 = synth.chebyshev_rhs(m0, m0, nm0, seed=0, ib=0)
    out["cfg0"] = {}
    for (fname, bound, lam) in c0["fields"]:
        ref0 = O.helm3d(r0, ops0, bound, lam, x0, nthreads=threads)[0]
        with D.Context(device) as c3:
            c3.pseudomat(m0)
            for name in paths:
                if name == "int8" and m0 > 129:
                    continue
                g = c3.helm3d(r0.copy(order="F"), bound, lam, x0, precision=precs[name])
                out["cfg0"]["%s_own_operators_%s" % (name, fname)] = _errs(g, ref0)
    return out


def bf16_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)).get("bf16_tflops")
    return 1590.0


def fp64_peak():
    p = os.path.join(ROOT, "profiles", "measured_fp64_peak.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["fp64_tflops"], "measured cuBLAS DGEMM on this pool (profiles/measured_fp64_peak.json)"
    return None, "no measured FP64 peak available"

# laminar square-duct flow rate (max velocity 1): the bulk Reynolds number
# Re = Q / (4 nu) of src/operators.F:2335 fixes nu for a given Re
Q_LAMINAR = 1.9081638750


def dns_cfg4(args, local, with_cpu):
    """Config 4: RK3/CN DNS of the square duct at mgalx = 256 (85 modes), my =
    mz = 193, Lx = 4 pi, Re_b = 4400, dt = 2e-4, 10 % seeded divergence-free
    perturbation, CMASSFLOW, statistics gathered every step; the FP64 solve.
    The 200 steps of the config are timed as CUDA-graph replays of the
    substeps (one graph launch per substep) after 3 warm-up steps; the
    per-kernel-class shares come from 2 more steps launched directly with a
    CUDA event pair around every launch.  The reference's CPU path (the
    oracle's step, every host core) runs one step from the same initial
    state, and the GPU's fields and statistics after that step are compared
    with it (the GPU's own eigen-decompositions, as the drop-in runs)."""
    import duct_b200 as D
    from duct_b200 import synth
    cfg = synth.dns_config("cfg4")
    m, mg, alp, dt = cfg["my"], cfg["mgalx"], cfg["alp"], cfg["dt"]
    fnu = Q_LAMINAR / (4.0 * cfg["re_b"])
    nsteps = cfg["steps"] if args.dns_steps is None else args.dns_steps
    u, v, w, p, _ = synth.dns_initial(mg, m, alp, cfg["amp"], seed=4)
    out = {"config": "cfg4: mgalx=256 (85 modes) x 193 x 193, Lx=4pi, Re_b=4400, dt=2e-4, 10%% perturbation, "
                     "CMASSFLOW, statistics every step, FP64 solves", "steps": nsteps, "warmup": 3}
    with D.Context(local) as ctx:
        ctx.pseudomat(m)
        with D.Dns(ctx, mg, alp, fnu, dt, cmassflow=True, hist_cap=nsteps + 8) as d:
            d.set_fields(u, v, w, p)
            d.steps(3, stats_every=1)
            ctx.synchronize()
            clocks = ClockSampler(local)
            clocks.start()
            ctx.event_record(0)
            d.steps(nsteps, stats_every=1)
            ctx.event_record(1)
            ms = ctx.event_elapsed(0, 1)
            clk = clocks.stop()
            st = d.statistics()
            out.update({"steps_per_s": 1e3 * nsteps / ms, "ms_per_step": ms / nsteps, "clocks": clk,
                        "divmax_last_step": [float(x) for x in st["divmax"]],
                        "step": "3 substeps, each one CUDA-graph launch"})
            d.set_graphs(False)
            ctx.profile(True)
            ctx.profile_reset()
            ctx.event_record(0)
            d.steps(2, stats_every=1)
            ctx.event_record(1)
            ms2 = ctx.event_elapsed(0, 1)
            names = {D.K_LINES: "chebyshev_lines (transyz+derivyz+transyz as the collocation matrices' "
                                 "flip-symmetric half blocks on the FP64 tensor cores, with the daxpy/dscal epilogues)",
                     D.K_ADVECTION: "x_fft_products (fourx, 2/3 rule, mult)",
                     D.K_PASS_FP64: "helm3d_gemm_passes", D.K_NEUMANN: "helm3d_neumann_fill",
                     D.K_WALLS: "helm3d_walls", D.K_OTHER: "impose_mass_flow", D.K_STATS: "statistics"}
            shares = {}
            for k, nm in names.items():
                kms, kn = ctx.profile_read(k)
                shares[nm] = {"ms_per_step": kms / 2, "launches_per_step": kn / 2, "share": kms / ms2}
            lms, ln = ctx.profile_read(D.K_LINES)
            lbytes = ctx.profile_bytes(D.K_LINES)
            lflops = ctx.profile_flops(D.K_LINES)
            ams, an = ctx.profile_read(D.K_ADVECTION)
            abytes = ctx.profile_bytes(D.K_ADVECTION)
            ctx.profile(False)
            peak, peak_src = hbm_peak()
            fpk, fpk_src = fp64_peak()
            out["kernel_classes"] = shares
            ltf = lflops / (lms * 1e-3) / 1e12
            out["roofline"] = {
                "chebyshev_lines": {"bound": "fp64_tensor", "achieved": ltf, "peak": fpk, "unit": "TFLOP/s",
                                    "frac": (ltf / fpk) if fpk else None, "flops_per_step": lflops / 2,
                                    "peak_source": fpk_src,
                                    "note": "DMMA flops executed (padded 16-row tiles included) over the line "
                                            "kernels' event-timed duration",
                                    "hbm": {"achieved": lbytes / (lms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                                            "frac": lbytes / (lms * 1e-3) / 1e9 / peak, "bytes_per_step": lbytes / 2,
                                            "note": "algorithmic bytes (each field read or written once)"}},
                "x_fft_products": {"bound": "hbm", "achieved": abytes / (ams * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                                   "frac": abytes / (ams * 1e-3) / 1e9 / peak},
                "peak_source": peak_src}
            try:
                out["checkpoint"] = dns_checkpoint(ctx, d)
            except (OSError, D.DuctGPUError) as e:     # a box without a writable temp directory
                out["checkpoint"] = {"error": str(e)}
    if with_cpu:
        from oracle import oracle as O
        threads = os.cpu_count() or 1
        O.set_blas_threads(1)
        orc = O.Dns(u, v, w, p, mg, alp, fnu, dt, cmassflow=True, nthreads=threads)
        nref = 2
        t0 = time.perf_counter()
        for _ in range(nref):
            orc.step(stats=True)
        el = time.perf_counter() - t0
        out["cpu_reference"] = {"steps_per_s": nref / el, "cores": threads, "kind": "port",
                                "sample": "%d steps of the oracle's RK3/CN substeps (same initial state)" % nref}
        with D.Context(local) as ctx:
            ctx.pseudomat(m)
            # the kx=0 pressure pinned at the reference's point (LAPACK order)
            ctx.set_gauge_point(orc.ops.iofzero)
            with D.Dns(ctx, mg, alp, fnu, dt, cmassflow=True) as d:
                d.set_fields(u, v, w, p)
                d.steps(nref, stats_every=1)
                got = d.fields()
                st = d.statistics()
        ref = orc.statistics()
        hist = np.array([h["stress4"] + h["energy"] + h["energy2"] for h in orc.history])
        out["parity_after_2_steps"] = {
            "reference": "oracle DNS steps (LAPACK operators), same seeded state; GPU with its own "
                         "eigen-decompositions, kx=0 pressure pinned at the oracle's iofzero; statistics "
                         "accumulated over both steps (the second step's from the state after the first)",
            "fields": {fn: _errs(g, r) for fn, g, r in zip("uvwp", got, (orc.u, orc.v, orc.w, orc.p))},
            "statistics": {k: _errs(st[k], ref[k]) for k in ("mean", "prod", "ppb", "spec")},
            "stress_energy_history": _errs(st["hist"], hist)}
    return out


def _fs_rates(directory, nbytes):
    """Plain write / read rates of the file system under `directory` for a
    file of nbytes (numpy tofile / fromfile, no fsync): the bound the
    checkpoint calls run against."""
    import tempfile
    buf = np.random.default_rng(0).integers(0, 255, nbytes, dtype=np.uint8)
    with tempfile.TemporaryDirectory(dir=directory) as tdir:
        path = os.path.join(tdir, "plain.bin")
        t0 = time.perf_counter()
        buf.tofile(path)
        tw = time.perf_counter() - t0
        t0 = time.perf_counter()
        back = np.fromfile(path, dtype=np.uint8)
        tr = time.perf_counter() - t0
    assert back.size == nbytes
    return {"write_GBps": nbytes / tw / 1e9, "read_GBps": nbytes / tr / 1e9}


def dns_checkpoint(ctx, d):
    """The stepper's state written as the reference's uvwp_NNNN.h5
    (save_4fields_fou_hdf5 + writeheader_hdf5) to a temporary directory and
    read back as a restart (read_4fields_fou_hdf5): wall-clock times of the
    calls (to the page cache, no fsync), the swap kernels' event time, and
    whether the restart restored the fields bit for bit."""
    import tempfile
    import duct_b200 as D
    before = d.fields()
    with tempfile.TemporaryDirectory() as tdir:
        path = D.uvwp_filename(tdir + "/", 1)
        ctx.profile(True)
        ctx.profile_reset()
        t0 = time.perf_counter()
        d.save_hdf5(path, time=0.0)
        t_save = time.perf_counter() - t0
        kms, kn = ctx.profile_read(D.K_OTHER)
        ctx.profile(False)
        nbytes = os.path.getsize(path)
        t0 = time.perf_counter()
        d.load_hdf5(path)
        t_load = time.perf_counter() - t0
    after = d.fields()
    field_bytes = 4 * before[0].nbytes
    fs = _fs_rates(tempfile.gettempdir(), nbytes)
    shm = None
    if os.path.isdir("/dev/shm"):
        st = os.statvfs("/dev/shm")
        if st.f_bavail * st.f_frsize > 3 * nbytes:
            with tempfile.TemporaryDirectory(dir="/dev/shm") as tdir:
                path = D.uvwp_filename(tdir + "/", 1)
                t0 = time.perf_counter()
                d.save_hdf5(path, time=0.0)
                ts = time.perf_counter() - t0
                t0 = time.perf_counter()
                d.load_hdf5(path)
                tl = time.perf_counter() - t0
            shm = {"save_ms": 1e3 * ts, "save_GBps": field_bytes / ts / 1e9, "load_ms": 1e3 * tl,
                   "load_GBps": field_bytes / tl / 1e9, "file_system": _fs_rates("/dev/shm", nbytes)}
    return {"file_bytes": nbytes, "field_bytes": field_bytes, "tmpdir": tempfile.gettempdir(),
            "tmpdir_plain_io": fs, "dev_shm": shm,
            "save_ms": 1e3 * t_save, "save_GBps": field_bytes / t_save / 1e9,
            "load_ms": 1e3 * t_load, "load_GBps": field_bytes / t_load / 1e9,
            "swap_kernels": {"launches": kn, "ms": kms, "GBps": field_bytes / (kms * 1e-3) / 1e9 if kms else None,
                             "note": "HBM -> big-endian -> mapped pinned host chunks (the host link bounds it)"},
            "restart_bit_exact": all(np.array_equal(a, b) for a, b in zip(before, after)),
            "note": "wall clock of ductgpu_dns_save_hdf5 / _load_hdf5 (file in the page cache, no fsync)"}


def uneven_rect_rate(ctx, args):
    """The uneven batch of rectangular ducts (aspect 1-4 at (65,65), (65,129),
    (49,145), (33,129) with 32, 48, 64, 96 modes; u, v, w Dirichlet with
    lambda = kx^2 + 2/(nu dt), nu = 1/4400, dt = 5e-4, and the Neumann
    pressure with lambda = kx^2, kx = k): 16 fields in one batched call,
    replayed from a CUDA graph; FP64 passes on the flip-symmetric half blocks
    (every duct has matching walls per direction; the fields' groups of
    equal half-block sizes on concurrent streams), as one persistent launch,
    and on the full operators for comparison.  Inputs (180 MB) exceed L2."""
    import duct_b200 as D
    from duct_b200 import synth
    ducts = (((65, 65), 1.0, 32), ((65, 129), 2.0, 48), ((49, 145), 3.0, 64), ((33, 129), 4.0, 96))
    h = 2.0 / ((1.0 / 4400.0) * 5.0e-4)
    fields, keep = [], []
    for slot, ((my, mz), aspect, nm) in enumerate(ducts):
        ctx.pseudomat_temp(slot, my, mz, 1.0, aspect)
        ctx.pseudomat_temp(4 + slot, my, mz, 1.0, aspect, ("n", "n"), ("n", "n"))
        xalp = 1.0 * np.arange(nm)
        for fld in range(4):
            neu = fld == 3
            f = synth.chebyshev_rhs(my, mz, nm, seed=10 * slot + fld, ib=0)
            r, o = ctx.device_array(f.shape), ctx.device_array(f.shape)
            r.upload(f)
            keep += [r, o]
            fields.append(dict(rhs=r, sol=o, xalp=xalp, alambda=0.0 if neu else h, ib=0,
                               slot=(4 + slot) if neu else slot))
    def timed(fold):
        ctx.set_rect_fold(fold)
        gid = ctx.graph_create(fields, rect=True)
        for _ in range(max(3, args.warmup)):
            ctx.graph_launch(gid)
        ctx.synchronize()
        steps = max(10, args.steps)
        ctx.event_record(0)
        for _ in range(steps):
            ctx.graph_launch(gid)
        ctx.event_record(1)
        ms = ctx.event_elapsed(0, 1) / steps
        ctx.synchronize()
        ctx.graph_destroy(gid)
        return ms, steps

    ms_full, _ = timed(0)
    ms_queue, _ = timed(2)
    ms, steps = timed(1)
    ctx.set_rect_fold(1)
    for x in keep:
        x.free()
    per_step = 4 * sum(nm for _, _, nm in ducts)
    return {"value": per_step / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "mode_solves_per_step": per_step,
            "fields": len(fields), "steps": steps,
            "config": "4 rectangular ducts (65x65, 65x129, 49x145, 33x129; 32/48/64/96 modes) x (u, v, w, p)",
            "step": "CUDA-graph replay of ductgpu_solve_rect_fields_dev (16 fields): flip-symmetric half blocks, "
                    "fields grouped by half-block sizes (3 groups), each group's four passes on a stream of "
                    "its own (12 GEMM-pass launches, parallel graph branches)",
            "single_launch": {"value": per_step / (ms_queue * 1e-3), "ms_per_step": ms_queue,
                              "step": "the same, the four passes of all 16 fields as ONE persistent launch "
                                      "(tiles in pass order, per-plane counters between the passes)"},
            "full_operators": {"value": per_step / (ms_full * 1e-3), "ms_per_step": ms_full,
                               "step": "the same on the full operators, one launch per GEMM pass"}}


def torch_sm_count():
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count


def traffic_from_profile(kernel):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p)).get(kernel, {}).get("bytes_per_launch")
    return None


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured copy (MEASURED_PEAKS.json)"
    return 6650.0, "fallback 6.65 TB/s"


def transform_rates(ctx, reps=20):
    """Achieved HBM bandwidth of the memory-bound kernels on a config-4 sized
    field (my = mz = 193, 85 modes, 50.7 MB complex128): transyz along y and
    z, derivyz, and the pencil transposes.  Four buffers rotate (203 MB > L2);
    algorithmic bytes = read + write of one field per call."""
    import ctypes as C
    import duct_b200 as D
    L = D.lib()
    m, nm = 193, 85
    shape = (m, m, nm)
    rng = np.random.default_rng(0)
    host = np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    bufs = [ctx.device_array(shape) for _ in range(4)]
    for b in bufs:
        b.upload(host)
    fbytes = host.nbytes
    peak, src = hbm_peak()
    h = ctx.h
    ops = {
        # forward and backward alternate so the values keep their size
        "transyz_y": lambda i: L.ductgpu_transyz_dev(h, C.c_void_p(bufs[i % 4].ptr), m, m, nm, b"y",
                                                     -1 if (i // 4) % 2 == 0 else 1),
        "transyz_z": lambda i: L.ductgpu_transyz_dev(h, C.c_void_p(bufs[i % 4].ptr), m, m, nm, b"z",
                                                     -1 if (i // 4) % 2 == 0 else 1),
        "derivyz_y": lambda i: L.ductgpu_derivyz_dev(h, C.c_void_p(bufs[i % 4].ptr), C.c_void_p(bufs[(i + 2) % 4].ptr),
                                                     m, m, nm, b"y", 1, 1.0, b"n", 1.0),
        "derivyz_z": lambda i: L.ductgpu_derivyz_dev(h, C.c_void_p(bufs[i % 4].ptr), C.c_void_p(bufs[(i + 2) % 4].ptr),
                                                     m, m, nm, b"z", 1, 1.0, b"n", 1.0),
        "cxyz2yzx": lambda i: L.ductgpu_cxyz2yzx_dev(h, C.c_void_p(bufs[i % 4].ptr), C.c_void_p(bufs[(i + 2) % 4].ptr),
                                                     nm, m, m),
    }
    out = {}
    for name, op in ops.items():
        for i in range(3):
            assert op(i) == 0, ctx.last_error()
        ctx.synchronize()
        ctx.event_record(2)
        for i in range(reps):
            op(i)
        ctx.event_record(3)
        ms = ctx.event_elapsed(2, 3) / reps
        gbs = 2.0 * fbytes / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "achieved_gbs": gbs, "frac": gbs / peak}
    for b in bufs:
        b.free()
    return {"field": "193x193x85 complex128 (50.7 MB), 4 rotating buffers", "peak_gbs": peak,
            "peak_source": src, "kernels": out}


def measure_e2e(ctx, c, m, nm, xalp, rhs, prec, args, pg, world):
    """End to end through the drop-in helm3d on pinned host arrays."""
    import ctypes as C
    import duct_b200 as D
    L = D.lib()
    nbytes = rhs[0].nbytes
    hr, hs = [], []
    for f in rhs:
        p = C.c_void_p()
        ctx._check(L.ductgpu_host_alloc(ctx.h, nbytes, C.byref(p)))
        a = np.ctypeslib.as_array((C.c_double * (nbytes // 8)).from_address(p.value))
        a[:] = f.ravel(order="F").view(np.float64)
        hr.append((p, a))
        q = C.c_void_p()
        ctx._check(L.ductgpu_host_alloc(ctx.h, nbytes, C.byref(q)))
        hs.append(q)
    x = np.ascontiguousarray(xalp)

    nf = len(rhs)
    pr = (C.c_void_p * nf)(*[p.value for p, a in hr])
    ps = (C.c_void_p * nf)(*[q.value for q in hs])
    bounds = "".join(b for _, b, _ in c["fields"]).encode()
    lams = np.array([lam for _, _, lam in c["fields"]], dtype=np.float64)

    def step():
        # the four helm3d calls of a substep in one pipelined call
        ctx._check(L.ductgpu_helm3d_batch(ctx.h, nf, C.cast(pr, C.c_void_p), C.cast(ps, C.c_void_p), bounds,
                                          lams.ctypes.data_as(C.c_void_p), m, m, 0, nm - 1,
                                          x.ctypes.data_as(C.c_void_p), prec))

    steps = max(3, args.steps // 5)
    for _ in range(max(3, args.warmup)):
        step()
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    el = max_over_ranks(pg, time.perf_counter() - t0)
    for p, a in hr:
        L.ductgpu_host_free(ctx.h, p)
    for q in hs:
        L.ductgpu_host_free(ctx.h, q)
    per_step = nm * len(rhs)
    return {"value": world * per_step * steps / el, "unit": UNIT,
            "h2d_bytes_per_step": nbytes * len(rhs), "d2h_bytes_per_step": nbytes * len(rhs),
            "steps": steps, "api": "ductgpu_helm3d_batch (u, v, w, p host arrays, pinned; copies overlapped with solves)"}


def main():
    args = parse()
    if args.impl == "reference":
        # rank 0 alone times the CPU reference; other ranks exit without work
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    if args.transforms_only:
        import duct_b200 as D
        with D.Context(0) as ctx:
            print(json.dumps(transform_rates(ctx)), flush=True)
        return
    if args.dns_only:
        print(json.dumps({"cfg4_dns": dns_cfg4(args, 0, not args.no_cpu)}), flush=True)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()

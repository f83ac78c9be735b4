#!/usr/bin/env python
"""Benchmark of the B200 DD-PCG Poisson solver.

One step = one Poisson solve (PCG to 1e-6 relative residual, preconditioner
already initialised) of the workload's domain.  The default workload is the
256^3-cell domain with a Dirichlet sphere and 32^3 subdomains (sub_size 32,
vlevels 4, interior/boundary smoothing 4, sigma_levels 4, sigma_mg 1);
``--config c1`` selects the 64^3-cell, 16^3-subdomain case; ``c5`` the sparse
1024^3-cell sphere union (``c5_half`` the same shape at 512^3); ``c2ml`` the
256^3 domain under two-level DD (the reference's -multilevel yes) at the
two-level demo's defaults (64^3 subdomains split into 32^3 boxes, vlevels 3,
smoothing 1/3, sigma_levels 3), ``tl128`` the same settings at 128^3.

``--impl reference`` times the CPU restatement of the reference dd_pcg path
(the oracle) on the host cores instead.

The output is one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Poisson solves/sec @1e-6 rel. residual"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--config", choices=["c1", "c2", "c3", "p128", "c4", "c5", "c5_half", "c2ml", "tl128"],
                   default="c2",
                   help="c4 = serving: resident uneven domains, solve requests through hdd_server_*")
    p.add_argument("--domains", type=int, default=4, help="c4: resident domains")
    p.add_argument("--requests", type=int, default=32, help="c4: requests per timed run")
    p.add_argument("--slots", type=int, default=4, help="c4: requests in flight")
    p.add_argument("--batch", type=int, default=0, choices=[0, 2, 4],
                   help="c4: requests of one domain solved together in shared launches (0 = off: each "
                        "request on a context of one system; measured faster on this mix)")
    p.add_argument("--fresh-domains", action="store_true",
                   help="c4: every request brings its own new domain (setup counted in its latency)")
    p.add_argument("--one-solve", action="store_true",
                   help="set up, run one solve with per-phase timing and print the phase table "
                        "(the command profiled under ncu; prints no JSON line)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--precision", choices=["reference", "mixed"], default="reference")
    return p.parse_args()


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x, dist, device):
    """The maximum of a per-rank time over all ranks (the whole job's time)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, steps, seconds):
    """Whole-job solves/s: every rank (replica) solves `steps` times."""
    return world * steps / seconds


# The sparse sphere-union workloads are built and handed over as SPGrid pages:
# the generator and the caller hold no dense arrays of their 1024^3 (or 512^3)
# box (the library's setup still expands the pages over the box internally).
PAGED = {"c5": 1, "c5_half": 2}


def workload(cfg):
    from hierarchicaldd_b200 import domains
    if cfg in PAGED:
        return domains.config5_pages(PAGED[cfg])
    return domains.CONFIGS[cfg]()


def set_domain(s, d):
    """Hands domain d to solver s: as SPGrid pages when it is paged, else dense."""
    from hierarchicaldd_b200.domains import PagedDomain
    if isinstance(d, PagedDomain):
        s.Set_Domain_Pages(d.origin, d.flags, d.rhs)
    else:
        s.Set_Domain(d.flags, d.rhs)


PHASES = ["vcycle", "laplace", "pcg_vector", "interface", "sigma_vcycle", "dense_tile_copy",
          "sn_forward", "sn_backward"]


def one_solve(args):
    """Setup and a single timed solve: the command profiled under ncu."""
    from hierarchicaldd_b200 import _lib
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver
    d = workload(args.config)
    m = d.meta
    s = SPGrid_Domain_Decomposition_Solver()
    set_domain(s, d)
    t0 = time.time()
    s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                m["sigma_mg"], tol=1e-6, multilevel=m.get("multilevel", False))
    print(f"{d.name}: setup {time.time() - t0:.1f} s", flush=True)
    lib = _lib.load()
    lib.hdd_set_kernel_timing(s.h, 1)
    r = s.Solve()
    ms = (C.c_double * len(PHASES))()
    cnt = (C.c_longlong * len(PHASES))()
    nbytes = (C.c_double * len(PHASES))()
    lib.hdd_get_kernel_timing(s.h, ms, cnt)
    lib.hdd_get_kernel_bytes(s.h, nbytes)
    print(f"solve: {r['iterations']} iterations, {r['solve_ms']:.2f} ms, true residual {r['true_residual_inf']:.3e}")
    for i, n in enumerate(PHASES):
        print(f"phase {n:16s} {ms[i]:10.3f} ms {cnt[i]:6d} launches {nbytes[i]:.6e} algorithmic bytes")
    print(f"kernel launches {s.Kernel_Launches()}")
    s.close()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_traffic(kernel, workload):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    `kernel` on `workload` from the committed ncu summaries, or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and not line.startswith("#") and parts[0] == kernel and parts[1] == workload:
                    return float(parts[2])
    except OSError:
        pass
    return None


def oracle_iterations(cfg):
    """PCG iterations of the oracle's full solve of a workload at 1e-6 relative
    residual, with where the count comes from: the committed fixture made by
    tests/golden/make_c2_fixture.py (a full FP32 oracle run) for c2, by
    tests/golden/make_two_level_fixture.py for c2ml and tl128, None for
    workloads whose oracle samples are whole solves."""
    if cfg == "c2":
        path = os.path.join(ROOT, "tests", "golden", "c2_oracle.npz")
        if os.path.exists(path):
            return int(np.load(path)["iterations_fp32"]), "tests/golden/c2_oracle.npz (full FP32 oracle solve)"
    if cfg in ("c2ml", "tl128"):
        path = os.path.join(ROOT, "tests", "golden", "two_level_oracle.npz")
        key = f"{cfg}_iterations_fp32"
        if os.path.exists(path) and key in np.load(path).files:
            return int(np.load(path)[key]), "tests/golden/two_level_oracle.npz (full FP32 oracle solve)"
    return None, None


# PCG iterations of the bounded CPU sample in the GPU arm's line: whole solves
# where one takes seconds, else a few iterations scaled by the oracle's count.
SAMPLE_ITERATIONS = {"c1": None, "c2": 2, "p128": 4, "c2ml": 1, "tl128": 4}


def make_oracle(d):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_ffi import Oracle
    m = d.meta
    return Oracle(d.size, d.sub_size, d.flags, vlevels=m["vlevels"], nVcycles=m["nVcycles"],
                  interior_smoothing=m["interior_smoothing"], boundary_smoothing=m["boundary_smoothing"],
                  sigma_levels=m["sigma_levels"], sigma_smoothing=m["sigma_smoothing"], sigma_mg=m["sigma_mg"],
                  multilevel=m.get("multilevel", False))


def precision_mode(args, d):
    """PCG precision: the workload's own (the sparse workload asks for the
    precision form) unless --precision mixed asks for the precision form."""
    return 1 if args.precision == "mixed" or d.meta.get("precision_mode", 0) == 1 else 0


def config_dict(d, args, world=1):
    """The workload description shared by both arms' lines."""
    m = d.meta
    return {"workload": d.name, "size": list(d.size), "sub_size": list(d.sub_size), "vlevels": m["vlevels"],
            "nVcycles": m["nVcycles"], "interior_smoothing": m["interior_smoothing"],
            "boundary_smoothing": m["boundary_smoothing"], "sigma_levels": m["sigma_levels"],
            "sigma_smoothing": m["sigma_smoothing"], "sigma_mg": m["sigma_mg"], "tol": 1e-6,
            "precision": "mixed" if precision_mode(args, d) == 1 else "reference",
            "multilevel": bool(m.get("multilevel", False)),
            "l2": "working set > L2 (no flush)", "parallelism": f"replicas{world}"}


def level0_updates_per_iteration(d):
    """Level-0 stencil evaluations per PCG iteration per Active|Interface cell:
    the Laplacian of q = A s, plus per V-cycle 2 x (boundary + interior +
    boundary) smoothing sweeps (each computes the residual over every active
    cell) and the residual before restriction, for the 2 x nVcycles V-cycles
    of one preconditioner application (4 x nVcycles under two-level DD, whose
    subdomain solves run V-cycles twice each).  Coarse levels are not counted."""
    m = d.meta
    per_vcycle = 2 * (2 * m["boundary_smoothing"] + m["interior_smoothing"]) + 1
    passes = 4 if m.get("multilevel") else 2
    return 1 + passes * m["nVcycles"] * per_vcycle


def cpu_baseline(args, d):
    """The oracle on the host cores, on a bounded sample of the same workload."""
    cores = os.cpu_count() or 1
    t0 = time.time()
    o = make_oracle(d)
    setup_s = time.time() - t0
    iters = SAMPLE_ITERATIONS[args.config]
    if iters is None:
        t0 = time.time()
        _, it, _ = o.solve(d.rhs, tol=1e-6)
        dt = time.time() - t0
        return {"value": 1.0 / dt, "unit": "solves/s", "cores": cores, "kind": "port",
                "sample": (f"one whole oracle solve of {d.name} ({it} PCG iterations, {dt:.2f} s, OpenMP over "
                           f"{cores} threads); oracle setup {setup_s:.1f} s untimed")}
    full, src = oracle_iterations(args.config)
    _, _, _, times = o.solve_timed(d.rhs, tol=0.0, max_it=iters, min_it=iters)
    per_it = float(times[-1]) / iters
    line = {"unit": "solves/s", "cores": cores, "kind": "port", "ms_per_pcg_iteration": per_it * 1e3}
    if full is None:
        line.update(value=None, sample=f"{iters} oracle PCG iterations of {d.name}, {per_it:.2f} s each; "
                                       f"no full-solve count for this workload")
        return line
    line.update(value=1.0 / (per_it * full),
                sample=(f"{iters} PCG iterations of {d.name} on the oracle ({per_it:.2f} s each, OpenMP over "
                        f"{cores} threads) times the oracle's {full}-iteration solve ({src}); "
                        f"oracle setup {setup_s:.1f} s untimed"))
    return line


def run_reference(args, rank):
    """The reference's CPU path (its restatement in oracle/, since the reference
    itself cannot be built here) on this workload, on the host cores.

    One full oracle solve runs to 1e-6 relative residual, so its PCG iteration
    count and its wall time are measured in this run; value = 1 / that solve's
    wall time.  A step is one PCG iteration of that solve: the first `warmup`
    iterations are warm-up, the next `steps` are the timed steps
    (ms_per_step), and the solve then runs on, untimed, to convergence.  For
    the 64^3 workload, whose solves take seconds, a step is a whole solve."""
    if rank != 0:
        return
    if args.config not in ("c1", "c2", "p128"):
        print(json.dumps({"impl": "reference", "unavailable": f"no bounded oracle run is defined for "
                          f"{args.config}: its oracle setup alone takes from tens of minutes to hours"}),
              flush=True)
        return
    d = workload(args.config)
    cores = os.cpu_count() or 1
    t0 = time.time()
    o = make_oracle(d)
    setup_s = time.time() - t0
    print(f"[bench reference] {d.name}: oracle setup {setup_s:.1f} s", file=sys.stderr, flush=True)
    whole_solves = args.config == "c1"
    durations, solves = [], []
    while len(durations) < args.warmup + args.steps:
        t1 = time.time()
        _, it, info, times = o.solve_timed(d.rhs, tol=1e-6, max_it=2000)
        solves.append((time.time() - t1, it, info))
        durations.extend([solves[-1][0]] if whole_solves else list(np.diff(np.concatenate([[0.0], times]))))
    timed = np.array(durations[args.warmup:args.warmup + args.steps])
    solve_s, its, info = solves[0]
    v = 1.0 / solve_s
    step = "one whole oracle solve" if whole_solves else (
        f"one PCG iteration of a full oracle solve: iterations {args.warmup + 1}..{args.warmup + args.steps} of "
        f"the solve are the timed steps, the first {args.warmup} warm-up")
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(timed.mean()) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": config_dict(d, args),
            "step": step, "iterations": int(its), "iterations_measured_in_run": True,
            "solve_s": solve_s, "ms_per_pcg_iteration": solve_s / max(its, 1) * 1e3,
            "true_residual_inf": float(info["true_res_inf"] / info["b_inf"]),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": (f"one full oracle solve of {d.name} ({its} PCG iterations measured in this "
                                        f"run, {solve_s:.1f} s, OpenMP over {cores} threads); oracle setup "
                                        f"{setup_s:.1f} s untimed")},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def percentiles(lat_ms):
    a = np.asarray(lat_ms, np.float64)
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)), "max": float(a.max())}


def run_serving(args):
    """Serving workload: uneven resident domains (cube sides 64..192, random
    Dirichlet spheres), solve requests with 1-3 delta sources, rhs in and
    solution out through host buffers.

    * serving form: mixed precision (FP32 operators, FP64 PCG scalars and
      iterate) with the coarsest interface level solved exactly
      (HDD_COARSE_EXACT), through the hdd_server_* C ABI with ``--slots``
      workers, each a driver that solves its domain's queued requests as
      its contexts free up (``--batch`` 2 or 4: several requests of one
      domain solved together in shared launches);
    * plain drop-in: the reference's settings (reference precision, 200
      coarsest smoothing steps) through hdd_set_rhs_dense / hdd_solve /
      hdd_get_solution_dense, one request at a time;
    * the serving form with one request in flight, for the gain of
      concurrency alone and for the check that every result is bit-identical
      alone and in the mix.
    Saturated: all requests queued at once, solves/s = requests / makespan.
    Open loop: Poisson arrivals at 0.8x the plain path's saturated rate;
    latency = arrival to finish.
    """
    from hierarchicaldd_b200 import _lib, domains
    from hierarchicaldd_b200.server import SolveServer, make_options
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver

    ds = domains.serving_mix(args.domains)
    rng = np.random.Generator(np.random.Philox(44))
    K = args.requests
    picks = [int(i) for i in rng.integers(0, len(ds), K)]
    rhs = [domains.serving_rhs(ds[i], rng) for i in picks]
    gaps = rng.exponential(1.0, K)

    def serving_meta(d):
        m = dict(d.meta)
        m.update(precision_mode=_lib.PRECISION_MIXED, coarse_solve=_lib.COARSE_EXACT)
        return m

    srv = SolveServer(slots=args.slots, batch=args.batch)
    t0 = time.perf_counter()
    ids = [srv.add_domain(d.flags, make_options(d.size, d.sub_size, tol=1e-6, max_iters=1000, **serving_meta(d)))
           for d in ds]
    for dom in ids:
        srv.wait_domain(dom)
    setup_s = time.perf_counter() - t0
    print(f"[bench] serving: {len(ds)} domains resident after {setup_s:.1f} s", file=sys.stderr, flush=True)
    # The plain drop-in: one handle per domain, reference settings.
    plain = []
    for d in ds:
        m = dict(d.meta)
        m.pop("precision_mode", None)
        m.pop("true_residual_every", None)
        h = SPGrid_Domain_Decomposition_Solver()
        h.Set_Domain(d.flags, d.rhs)
        h.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                    m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                    m["sigma_mg"], tol=1e-6, max_iters=1000)
        plain.append(h)
    for i, dom in enumerate(ids):  # warm-up: one solve per domain on each path
        srv.poll(srv.submit(dom, ds[i].rhs), dom, want_x=False)
        plain[i].Set_RHS(ds[i].rhs)
        plain[i].Solve(allow_not_converged=True)

    def digest(r):  # (status, result, solution digest, latency)
        return r[0], r[1], hashlib.sha1(r[2].tobytes()).hexdigest(), r[3]

    def plain_solve(k):
        t = time.perf_counter()
        h = plain[picks[k]]
        h.Set_RHS(rhs[k])
        res = h.Solve(allow_not_converged=True)
        x = h.Solution()
        return 0 if res["converged"] else 3, res, x, (time.perf_counter() - t) * 1e3

    def saturated(in_flight):
        out, t = [], time.perf_counter()
        if in_flight == 0:
            out = [digest(plain_solve(k)) for k in range(K)]
        elif in_flight == 1:
            for k in range(K):
                out.append(digest(srv.poll(srv.submit(ids[picks[k]], rhs[k]), ids[picks[k]])))
        else:
            reqs = [srv.submit(ids[picks[k]], rhs[k]) for k in range(K)]
            out = [digest(srv.poll(r, ids[picks[k]])) for k, r in enumerate(reqs)]
        return time.perf_counter() - t, out

    def open_loop(rate, serving):
        arrivals = np.cumsum(gaps / rate)
        lat, t = [], time.perf_counter()
        if not serving:
            for k in range(K):
                now = time.perf_counter() - t
                if arrivals[k] > now:
                    time.sleep(arrivals[k] - now)
                plain_solve(k)
                lat.append((time.perf_counter() - t - arrivals[k]) * 1e3)
            return lat
        reqs, done = [], {}

        def collect():
            for k in range(K):
                while len(reqs) <= k:
                    time.sleep(1e-4)
                done[k] = srv.poll(reqs[k], ids[picks[k]], want_x=False)
        th = threading.Thread(target=collect)
        th.start()
        for k in range(K):
            now = time.perf_counter() - t
            if arrivals[k] > now:
                time.sleep(arrivals[k] - now)
            reqs.append(srv.submit(ids[picks[k]], rhs[k]))
        th.join()
        return [done[k][3] for k in range(K)]  # submit (= arrival) to finish

    with ClockSampler(0) as clk:
        t_plain, r_plain = saturated(0)
        t_alone, r_alone = saturated(1)
        t_serve, r_serve = saturated(args.slots)
    plain_rate, alone_rate, serve_rate = K / t_plain, K / t_alone, K / t_serve
    rate = 0.8 * plain_rate
    lat_plain = open_loop(rate, False)
    lat_serve = open_loop(rate, True)
    srv_mem = srv.memory()
    same = all(a[0] == b[0] and a[1]["iterations"] == b[1]["iterations"] and a[2] == b[2]
               for a, b in zip(r_alone, r_serve))
    statuses = [r[0] for r in r_serve]
    its = [r[1]["iterations"] for r in r_serve]
    its_plain = [r[1]["iterations"] for r in r_plain]
    tres = max(r[1]["true_residual_inf"] for r in r_serve)
    tres_plain = max(r[1]["true_residual_inf"] for r in r_plain)
    cells = [int(np.prod(ds[i].size)) for i in picks]
    for dom in ids:
        srv.remove_domain(dom)
    srv.close()
    for h in plain:
        h.close()
    line = {
        "metric": "Poisson solves/sec @1e-6 rel. residual (serving) + p50/p99 latency", "value": serve_rate,
        "unit": "solves/s", "n_gpus": 1, "steps": K, "warmup": len(ds), "ms_per_step": 1e3 / serve_rate,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 dots, alpha/beta, iterate)",
        "data": "synthetic",
        "config": {"workload": "c4_serving_sample", "domains": [d.name for d in ds], "requests": K,
                   "slots": args.slots, "batch": args.batch, "precision": "mixed", "coarse_solve": "exact",
                   "tol": 1e-6,
                   "l2": "no flush: resident domains, per-request working sets from 1 MB to 30 MB per vector"},
        "plain_one_in_flight": {"value": plain_rate, "unit": "solves/s",
                                "settings": "reference precision, 200 coarsest smoothing steps (hdd_solve)",
                                "saturated_latency_ms": percentiles([r[3] for r in r_plain]),
                                "open_loop_latency_ms": percentiles(lat_plain),
                                "iterations": {"min": int(min(its_plain)), "max": int(max(its_plain))},
                                "max_true_residual": tres_plain},
        "serving_form_one_in_flight": {"value": alone_rate, "unit": "solves/s",
                                       "speedup_from_concurrency": serve_rate / alone_rate},
        "latency_ms": {"saturated": percentiles([r[3] for r in r_serve]), "open_loop": percentiles(lat_serve),
                       "open_loop_rate": rate},
        "speedup_vs_plain": serve_rate / plain_rate,
        "results_identical_alone_and_in_mix": bool(same),
        "statuses": {str(s_): statuses.count(s_) for s_ in set(statuses)},
        "iterations": {"min": int(min(its)), "max": int(max(its))},
        "max_true_residual": tres,
        "setup_s": setup_s, "device_bytes_reserved": srv_mem[0],
        "e2e": {"value": serve_rate, "unit": "solves/s", "h2d_bytes_per_step": 4 * float(np.mean(cells)),
                "d2h_bytes_per_step": 4 * float(np.mean(cells))},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_serving_fresh(args):
    """Serving with a new domain per request, as the serving workload states it:
    each request is a domain (cube side cycling through 64..192, 1-4 random
    Dirichlet spheres) and a right-hand side, so its setup (interface
    assembly, factorisations, uploads) is part of its latency.

    * plain drop-in: one request at a time with the reference's settings
      (hdd_create, hdd_initialize_preconditioner, hdd_solve, hdd_destroy);
    * serving form (mixed precision, exact coarsest interface solve): the
      same one at a time through the server, then all requests queued at
      once; the server admits domains by HBM footprint, sets up to slots - 1
      of them while others solve, and each domain is removed once its result
      is collected.
    solves/s = requests / makespan; latency = domain added to result ready.
    """
    from hierarchicaldd_b200 import _lib, domains
    from hierarchicaldd_b200.server import SolveServer, make_options
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver

    K = args.requests
    ds = domains.serving_mix(K, seed=45)
    srv = SolveServer(slots=args.slots, batch=args.batch)

    def serving_meta(d):
        m = dict(d.meta)
        m.update(precision_mode=_lib.PRECISION_MIXED, coarse_solve=_lib.COARSE_EXACT)
        return m

    opts = [make_options(d.size, d.sub_size, tol=1e-6, max_iters=1000, **serving_meta(d)) for d in ds]

    def digest(x):
        return hashlib.sha1(x.tobytes()).hexdigest()

    with ClockSampler(0) as clk:
        plain, t = [], time.perf_counter()
        for d in ds:
            ta = time.perf_counter()
            m = d.meta
            h = SPGrid_Domain_Decomposition_Solver()
            h.Set_Domain(d.flags, d.rhs)
            h.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                        m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                        m["sigma_mg"], tol=1e-6, max_iters=1000)
            res = h.Solve(allow_not_converged=True)
            h.Solution()
            h.close()
            plain.append((0 if res["converged"] else 3, res["iterations"], (time.perf_counter() - ta) * 1e3))
        t_plain = time.perf_counter() - t
        alone, t = [], time.perf_counter()
        for k, d in enumerate(ds):
            ta = time.perf_counter()
            dom = srv.add_domain(d.flags, opts[k])
            st, res, x, _ = srv.poll(srv.submit(dom, d.rhs), dom)
            alone.append((st, res["iterations"], digest(x), (time.perf_counter() - ta) * 1e3))
            srv.remove_domain(dom)
        t_alone = time.perf_counter() - t
        serve, t = [], time.perf_counter()
        doms, reqs = [], []
        for k, d in enumerate(ds):
            doms.append(srv.add_domain(d.flags, opts[k]))
            reqs.append(srv.submit(doms[-1], d.rhs))
        for k in range(K):
            # the server's latency runs from the submit, made right after the add
            st, res, x, lat = srv.poll(reqs[k], doms[k])
            serve.append((st, res["iterations"], digest(x), lat))
            srv.remove_domain(doms[k])
        t_serve = time.perf_counter() - t
    srv.close()
    same = all(a[:3] == b[:3] for a, b in zip(alone, serve))
    statuses = [r[0] for r in serve]
    cells = [int(np.prod(d.size)) for d in ds]
    serve_rate, plain_rate, alone_rate = K / t_serve, K / t_plain, K / t_alone
    line = {
        "metric": "Poisson solves/sec @1e-6 rel. residual (serving, a new domain per request) + p50/p99 latency",
        "value": serve_rate, "unit": "solves/s", "n_gpus": 1, "steps": K, "warmup": 0,
        "ms_per_step": 1e3 / serve_rate, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 dots, alpha/beta, iterate)", "data": "synthetic",
        "config": {"workload": "c4_serving_fresh_domains", "requests": K, "slots": args.slots,
                   "sides": sorted({d.size[0] - 1 for d in ds}), "precision": "mixed", "coarse_solve": "exact",
                   "tol": 1e-6, "l2": "no flush: every request is a new domain"},
        "plain_one_in_flight": {"value": plain_rate, "unit": "solves/s",
                                "settings": "reference precision, 200 coarsest smoothing steps",
                                "latency_ms": percentiles([r[2] for r in plain]),
                                "statuses": {str(s_): [r[0] for r in plain].count(s_) for s_ in {r[0] for r in plain}}},
        "serving_form_one_in_flight": {"value": alone_rate, "unit": "solves/s",
                                       "latency_ms": percentiles([r[3] for r in alone]),
                                       "speedup_from_concurrency": serve_rate / alone_rate},
        "latency_ms": percentiles([r[3] for r in serve]),
        "speedup_vs_plain": serve_rate / plain_rate,
        "results_identical_alone_and_in_mix": bool(same),
        "statuses": {str(s_): statuses.count(s_) for s_ in set(statuses)},
        "e2e": {"value": serve_rate, "unit": "solves/s", "h2d_bytes_per_step": 8 * float(np.mean(cells)),
                "d2h_bytes_per_step": 4 * float(np.mean(cells))},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.config == "c4":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving path: "
                                  "its solver handles one domain per process"}), flush=True)
            return
        run_reference(args, rank)
        return
    if args.one_solve:
        one_solve(args)
        return
    if args.config == "c4":
        if args.fresh_domains:
            run_serving_fresh(args)
        else:
            run_serving(args)
        return
    if world > 1 and "OMP_NUM_THREADS" not in os.environ:
        # N replicas share the host for their (OpenMP) setup: split the cores.
        os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or 1) // world))
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from hierarchicaldd_b200 import _lib
    from hierarchicaldd_b200.domains import ACTIVE, PagedDomain
    from hierarchicaldd_b200.solver import SPGrid_Domain_Decomposition_Solver

    d = workload(args.config)
    m = d.meta
    s = SPGrid_Domain_Decomposition_Solver(device=local_rank)
    set_domain(s, d)
    t0 = time.time()
    s.Initialize_Preconditioner(m["vlevels"], d.size, d.sub_size, m["sigma_levels"], m["nVcycles"],
                                m["interior_smoothing"], m["boundary_smoothing"], m["sigma_smoothing"],
                                m["sigma_mg"], tol=1e-6, precision_mode=precision_mode(args, d),
                                true_residual_every=int(m.get("true_residual_every", 20)),
                                multilevel=m.get("multilevel", False))
    setup_s = time.time() - t0
    try:
        setup_phases = s.Setup_Timing()
    except Exception as e:  # a diagnostic only
        setup_phases = {"error": str(e)}
    print(f"[bench] {d.name}: setup {setup_s:.1f} s {setup_phases}", file=sys.stderr, flush=True)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for i in range(args.warmup):
        r0 = s.Solve()
        print(f"[bench] warmup {i}: {r0['solve_ms']:.2f} ms, {r0['iterations']} iterations", file=sys.stderr, flush=True)
    launches0 = s.Kernel_Launches()
    barrier()
    res = []
    with ClockSampler(local_rank) as clk:
        t_wall = time.time()
        for _ in range(args.steps):
            res.append(s.Solve())
        barrier()
        t_wall = time.time() - t_wall
    launches = s.Kernel_Launches() - launches0
    dev_ms = np.array([r["solve_ms"] for r in res])
    total_ms = max_over_ranks(float(dev_ms.sum()), dist, "cuda")
    value = job_throughput(world, args.steps, total_ms / 1000.0)

    # End to end through the C ABI with pinned host buffers: H2D of b, solve,
    # D2H of x (dense arrays of the box, or the SPGrid pages of a paged domain).
    paged = isinstance(d, PagedDomain)
    cells = int(d.rhs.size) if paged else int(np.prod(d.size))
    pin_b = torch.empty(cells, dtype=torch.float32, pin_memory=True)
    pin_x = torch.empty(cells, dtype=torch.float32, pin_memory=True)
    pin_b.numpy()[:] = d.rhs.ravel()
    lib = _lib.load()
    fp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_float))
    if paged:
        origin = np.ascontiguousarray(d.origin, np.int32)
        op = origin.ctypes.data_as(C.POINTER(C.c_int))
        set_rhs = lambda: lib.hdd_set_rhs_pages(s.h, origin.shape[0], op, fp(pin_b))
        get_x = lambda: lib.hdd_get_solution_pages(s.h, origin.shape[0], op, fp(pin_x))
    else:
        set_rhs = lambda: lib.hdd_set_rhs_dense(s.h, fp(pin_b))
        get_x = lambda: lib.hdd_get_solution_dense(s.h, fp(pin_x))
    barrier()
    t_e2e = time.perf_counter()
    for _ in range(args.steps):
        st = set_rhs()
        assert st == 0, st
        s.Solve()
        st = get_x()
        assert st == 0, st
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t_e2e     # host copies are part of this step, so host time
    e2e_val = job_throughput(world, args.steps, max_over_ranks(t_e2e, dist, "cuda"))

    # Per-phase device timing (separate, instrumented solve): CUDA events on
    # the solver's stream around each phase's launches, with the phase's
    # algorithmic bytes accounted by the library.
    ms = (C.c_double * len(PHASES))()
    cnt = (C.c_longlong * len(PHASES))()
    nbytes = (C.c_double * len(PHASES))()
    lib.hdd_set_kernel_timing(s.h, 1)
    prof = s.Solve()
    lib.hdd_get_kernel_timing(s.h, ms, cnt)
    lib.hdd_get_kernel_bytes(s.h, nbytes)
    lib.hdd_set_kernel_timing(s.h, 0)
    phases = PHASES
    phase_ms = {n: float(ms[i]) for i, n in enumerate(phases)}
    phase_n = {n: int(cnt[i]) for i, n in enumerate(phases)}

    # Roofline (HBM-bound kernels) of every timed kernel; the dominant one by
    # device time is the headline.
    hbm, peak_kind = peaks()
    vbox = d.sub_size[0] // 2 if m.get("multilevel") else d.sub_size[0]  # V-cycle box and tile edge
    kernels = {0: "vcycle_cluster_kernel" if vbox == 32 else "vcycle_kernel",
               1: "laplace_dot_march_kernel" if vbox in (8, 16, 32) else "laplace_dot_kernel",
               6: "sn_forward_kernel", 7: "sn_backward_kernel"}
    per_kernel = {}
    for i, kname in kernels.items():
        if cnt[i] == 0 or ms[i] <= 0:
            continue
        gbs = nbytes[i] / (ms[i] * 1e-3) / 1e9
        per_kernel[kname] = {"ms": float(ms[i]), "launches": int(cnt[i]),
                             "bytes_per_launch": float(nbytes[i] / cnt[i]), "achieved_gbs": gbs,
                             "frac": gbs / hbm}
    top = max(kernels, key=lambda i: ms[i])
    top_name = kernels[top]
    achieved = per_kernel.get(top_name, {}).get("achieved_gbs")
    traffic = measured_traffic(top_name, d.name)

    its = [r["iterations"] for r in res]
    lat = np.sort(dev_ms)
    # Active|Interface cells after the divider = the caller's Active cells.
    n_solve = int(np.count_nonzero(d.flags & ACTIVE))
    it0 = its[0] if its else 0
    updates = n_solve * level0_updates_per_iteration(d) * it0
    o_its, o_src = oracle_iterations(args.config)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_dict(d, args, world),
        "iterations": it0, "oracle_iterations": o_its, "oracle_iterations_source": o_src,
        "ms_per_pcg_iteration": total_ms / args.steps / max(it0, 1),
        "cell_updates_per_s": world * updates / (total_ms / args.steps * 1e-3),
        "cell_updates_definition": (f"level-0 stencil evaluations: {n_solve} Active|Interface cells x "
                                    f"{level0_updates_per_iteration(d)} per PCG iteration (1 Laplacian + "
                                    f"2 x nVcycles x (2 x (2 boundary + interior) sweeps + 1 residual)) x "
                                    f"{it0} iterations per solve; coarse levels not counted"),
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "true_residual_inf": res[-1]["true_residual_inf"] if res else None,
        "setup_s": setup_s, "setup_phases_s": setup_phases,
        "setup_host_threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
        "e2e": {"value": e2e_val, "unit": "solves/s", "h2d_bytes_per_step": 4 * cells, "d2h_bytes_per_step": 4 * cells},
        "gpu_launches": int(launches),
        "phase_ms_per_solve": phase_ms, "phase_launches_per_solve": phase_n,
        "roofline": {"kernel": top_name, "bound": "hbm", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                     "peak_kind": peak_kind,
                     "bytes_per_launch": per_kernel.get(top_name, {}).get("bytes_per_launch")},
        "kernels": per_kernel,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.config in SAMPLE_ITERATIONS:
        try:
            line["cpu_baseline"] = cpu_baseline(args, d)
        except Exception as e:  # reported, not fatal
            line["cpu_baseline"] = {"error": str(e)}
    s.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

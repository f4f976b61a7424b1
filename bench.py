#!/usr/bin/env python
"""Benchmark: MG-PCG solves/s (and p50/p99 latency) to 1e-8 relative residual,
mixed precision vs FP64, for the multiresolution cantilever.

One step = SetupGMG(densities) + SolveMG (zero start, ||f-Ku||/||f|| <= 1e-8)
+ Grad (sensitivities and transposed filter), i.e. one "solve plus Grad" of
the reference's per-iteration hot path, on one GPU per rank.  Ranks are
independent replicas (the path does not shard here); the printed value is
the whole-job rate, timed with CUDA events and maximised over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tosp|reference]

`--impl reference` times the reference's default algorithm on the host cores
(the C/OpenMP restatement of the assembled GlobalStiffMatrix / SetupGMG /
SolveMG / Grad path in oracle/): one complete solve, split over the timed steps.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "topopt-slp-3d_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "MG-PCG solves/s and p50/p99 latency at 1e-8 rel. residual, mixed vs FP64 GPU"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh), "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def host_cores():
    """Host threads this process may use (the CPU arms use all of them)."""
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def bench_config(args, spec, pb, n, ngrids, world):
    """The workload keys shared by the GPU line and the reference line."""
    return {"workload": args.workload, "mesh": list(spec["dims"]), "mr_n": n, "ndof": 3 * pb.nnodes,
            "nfree": int(pb.freedofs.size), "density_elements": int(pb.nelem * n ** 3), "ngrids": ngrids,
            "cycle": "V", "omega": spec["omega"], "smooth": "1+1 Jacobi", "tol": 1e-8,
            "l2": "inputs larger than L2 (densities 113 MB, vectors 44 MB each)" if n == 2 and pb.nelem > 10 ** 6
                  else "inputs of this size (between steps the setup rewrites every level)",
            "parallelism": f"replicas x{world}"}


def cpu_solver(args, spec):
    """The assembled-path oracle port for the workload, and the workload built
    with its host filter (no GPU involved)."""
    from oracle.cpu_assembled import CpuAssembled
    from tosp import problems
    from tosp.workloads import build_workload
    n = spec["n"]
    ngrids = args.ngrids or spec["ngrids"]
    pb0 = problems.cantilever(*spec["dims"])
    ca = CpuAssembled(pb0, n, ngrids, spec["omega"], rmin=spec["rmin"], nthreads=host_cores())
    pb, n, xfil, spec = build_workload(args.workload, filter_fn=ca.filter)
    return ca, pb, n, xfil, spec, ngrids


def _full(pb, u_free):
    out = np.zeros(3 * pb.nnodes)
    out[pb.freedofs] = u_free
    return out


def cpu_whole_solve(ca, pb, xfil):
    """One complete solve on the host: SetupGMG + SolveMG from zero to 1e-8 +
    Grad.  Returns the seconds of each part and the results."""
    f = pb.f_full()
    t0 = time.perf_counter()
    ca.setup(xfil)
    t1 = time.perf_counter()
    u, it, nr = ca.solve(np.zeros(f.size), f, 1e-8, 1000)
    t2 = time.perf_counter()
    g, _ = ca.grad(u)
    t3 = time.perf_counter()
    return {"setup_s": t1 - t0, "solve_s": t2 - t1, "grad_s": t3 - t2, "total_s": t3 - t0, "it": it, "relres": nr,
            "u": u, "g": g}


def run_reference(args, world, rank):
    """The reference's default assembled path (genK = true: GlobalStiffMatrix,
    SetupGMG, SolveMG, Grad) restated in C/OpenMP under oracle/, on all host
    threads.  The K timed steps together run ONE complete solve (setup, PCG
    to 1e-8, Grad), split by PCG iteration, so the value is a measured
    whole-solve rate; the W warm-up steps run a setup and W iterations."""
    if rank != 0:
        return 0
    from tosp.workloads import WORKLOADS
    spec = WORKLOADS[args.workload]
    ca, pb, n, xfil, spec, ngrids = cpu_solver(args, spec)
    cores = host_cores()
    f = pb.f_full()
    # warm-up (untimed): a setup, then one PCG iteration per warm-up step
    ca.setup(xfil)
    gen = ca.solve_iter(np.zeros(f.size), f, 1e-8, 1000)
    for _ in range(args.warmup):
        next(gen, None)
    its_planned = spec.get("pcg_iterations_fp64") or 100
    per, parts = [], {"setup_s": 0.0, "solve_s": 0.0, "grad_s": 0.0}
    gen, done = None, False
    for k in range(args.steps):
        t0 = time.perf_counter()
        if k == 0:
            ca.setup(xfil)
            gen = ca.solve_iter(np.zeros(f.size), f, 1e-8, 1000)
            parts["setup_s"] = time.perf_counter() - t0
        ts = time.perf_counter()
        last = k == args.steps - 1
        target = its_planned * (k + 1) / args.steps
        while not done and (last or ca.it - 1 < target):
            done = next(gen, None) is None
        parts["solve_s"] += time.perf_counter() - ts
        if last:
            tg = time.perf_counter()
            ca.grad(ca.x)
            parts["grad_s"] = time.perf_counter() - tg
        per.append(time.perf_counter() - t0)
    total = float(sum(per))
    value = 1.0 / total
    sample = (f"one complete {args.workload} solve (SetupGMG + SolveMG from zero to 1e-8 in {ca.it - 1} PCG "
              f"iterations + Grad with the transposed filter) of the assembled path restated in C/OpenMP, "
              f"{total:.1f} s on {cores} host threads, split over the {args.steps} timed steps by PCG iteration")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * total / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": bench_config(args, spec, pb, n, ngrids, world),
            "cg": "reference beta (I/SolveMG.m:43-46)",
            "solve": {"pcg_iterations": int(ca.it), "relres": float(ca.nr),
                      **{k: round(v, 3) for k, v in parts.items()}},
            "cpu_baseline": {"value": round(value, 6), "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


class _Timed:
    """Wraps a solve path and accumulates wall time per entry point (each
    call is synchronous)."""

    def __init__(self, inner):
        self.inner = inner
        self.t = {"filter": 0.0, "setup": 0.0, "solve": 0.0, "grad": 0.0}

    def _run(self, key, fn, *a, **k):
        t0 = time.perf_counter()
        out = fn(*a, **k)
        self.t[key] += time.perf_counter() - t0
        return out

    def ApplyFilter(self, x, trans=False):
        return self._run("filter", self.inner.ApplyFilter, x, trans=trans)

    def SetupGMG(self, x):
        return self._run("setup", self.inner.SetupGMG, x)

    def SolveMG(self, x, f):
        return self._run("solve", self.inner.SolveMG, x, f)

    def Grad(self, u):
        return self._run("grad", self.inner.Grad, u)


def run_slp(args):
    """Full SLP loop (host LP) on the GPU solve path: config 0 (FP64) or
    config 3 (mixed precision, MR factor 3, GradProj at the end)."""
    import torch
    import tosp
    from tosp import problems as P
    from tosp import slp
    torch.cuda.set_device(0)
    if args.slp == "config0":
        pb = P.cantilever(48, 24, 24)
        n, prec, ngr, rmin, volfrac, iters, lp, omega, cycle = 1, tosp.PREC_FP64, 3, 1.5, 0.3, 20, "knapsack", 0.6, 0
        prj = slp.PrjParams(op=False)
    else:
        pb = P.bridge(160, 80, 40)
        # cycle and omega unspecified for this loop: the reference defaults
        # (W-cycle, omega 0.5; I/TopOpt3D.m:172-174)
        n, prec, ngr, rmin, volfrac, iters, lp, omega, cycle = 3, tosp.PREC_MIXED, 4, 2.5 / 3, 0.2, 100, "knapsack", 0.5, 1
        prj = slp.PrjParams(op=True)
    iters = args.slp_iters or iters
    lp = args.lp or lp
    mg = tosp.default_mg(ngrids=ngr, cycle=cycle, omega=omega, smoothiter1=1, smoothiter2=1, tolMG=1e-8,
                         maxiterMG=2000, flexible=1 if prec == tosp.PREC_MIXED else 0,
                         cg_product=args.cg_product if prec == tosp.PREC_MIXED else 0)
    if prec == tosp.PREC_MIXED:
        # high-contrast designs defeat the FP32 V-cycle: stalled mixed solves
        # are finished in FP64, which then serves the rest of the loop
        solver = tosp.FallbackSolver(pb, mg, mr_n=n, p=3.0, emin=1e-9, opfilter=1, rmin=rmin, maxstall=100)
    else:
        solver = tosp.Solver(pb, mg, precision=prec, mr_n=n, p=3.0, emin=1e-9, opfilter=1, rmin=rmin)
    timed = _Timed(solver)
    x0 = np.full(pb.nelem * n ** 3, volfrac)
    per_it = []
    last = [time.perf_counter()]

    def on_iter(h):
        now = time.perf_counter()
        per_it.append(now - last[0])
        last[0] = now
    t0 = time.perf_counter()
    res = slp.str_slp(timed, pb, volfrac, x0, slp.SlpParams(maxiter=iters, lp=lp), prj=prj, on_iter=on_iter)
    wall = time.perf_counter() - t0
    steps = len(res.history)
    line = {"metric": f"SLP loop ({args.slp}): seconds per SLP iteration", "value": round(wall / max(steps, 1), 4),
            "unit": "s/iteration", "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
            "dtype": "f64" if prec == tosp.PREC_FP64 else "f64 outer CG / f32+bf16 V-cycle",
            "config": {"workload": args.slp, "mesh": [pb.nelx, pb.nely, pb.nelz], "mr_n": n, "volfrac": volfrac,
                       "rmin": rmin, "lp": lp, "ngrids": ngr, "cycle": "VW"[cycle], "omega": omega,
                       "cg_product": int(mg.cg_product)},
            "slp": {"accepted": res.iters, "rejected": res.rejected, "opstop": res.opstop, "F_final": res.F,
                    "F_first": res.history[0]["F"] if res.history else None,
                    "pcg_iterations_total": int(sum(res.pcgit)), "pcg_iterations": [int(i) for i in res.pcgit],
                    "unconverged_solves": int(sum(1 for st in res.pcgstatus if st != 0)), "wall_s": round(wall, 3)},
            "time_s": {k: round(v, 3) for k, v in timed.t.items()},
            "time_per_iteration_s": {k: round(v / max(steps, 1), 4) for k, v in timed.t.items()}}
    if prec == tosp.PREC_MIXED:
        line["slp"]["fp64_fallbacks"] = solver.fallbacks
    if prj.op:
        line["slp"]["volume_rounded"] = float(res.xstar.mean())
        line["slp"]["rounded_fraction_0_1"] = float(np.mean((res.xstar == 0) | (res.xstar == 1)))
    if args.slp == "config3":
        # the final design solved again on the GPU path and, independently,
        # from zero on the host (the reference's assembled path restated in
        # C/OpenMP, FP64, the same W-cycle) to a tighter tolerance: compliances
        # compared, and the GPU displacement's residual with the host operator
        from oracle.cpu_assembled import CpuAssembled
        xf_final = solver.ApplyFilter(res.x)
        solver.SetupGMG(xf_final)
        u_final, it_final, rr_final, rc_final = solver.SolveMG(res.u, pb.f)
        res.u = u_final
        ca = CpuAssembled(pb, n, ngr, omega, rmin=rmin, nthreads=host_cores(), cycle=cycle)
        t1 = time.perf_counter()
        ca.setup(xf_final)
        u_cpu, it_cpu, rr_cpu = ca.solve(np.zeros(3 * pb.nnodes), pb.f_full(), 1e-10, 20000)
        t_cpu = time.perf_counter() - t1
        uf = np.zeros(3 * pb.nnodes)
        uf[pb.freedofs] = u_final
        r = pb.f_full() - ca.apply(0, uf)
        F_gpu, F_cpu = float(pb.f @ u_final), float(pb.f_full() @ u_cpu)
        line["cpu_check"] = {"relres_cpu_operator": float(np.linalg.norm(r[pb.freedofs]) / np.linalg.norm(pb.f)),
                             "compliance_gpu": F_gpu, "compliance_cpu": F_cpu,
                             "compliance_rel_diff": abs(F_gpu - F_cpu) / abs(F_cpu),
                             "cpu_solve": {"it": int(it_cpu), "relres": float(rr_cpu), "s": round(t_cpu, 1),
                                           "cores": host_cores()},
                             "final_solve_it": int(it_final), "final_solve_relres": float(rr_final),
                             "final_solve_status": int(rc_final)}
    if args.check_cpu and args.slp == "config0":
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_solver import OracleSolver
        orc = OracleSolver(pb, n=n, ngrids=ngr, cycle=cycle, omega=omega, rmin=rmin)
        t1 = time.perf_counter()
        ro = slp.str_slp(orc, pb, volfrac, x0, slp.SlpParams(maxiter=iters, lp=lp), prj=prj)
        tcpu = time.perf_counter() - t1
        line["cpu_baseline"] = {"value": round(tcpu / max(len(ro.history), 1), 4), "unit": "s/iteration",
                                "cores": os.cpu_count(), "kind": "port",
                                "sample": f"the same {iters}-iteration SLP loop on the NumPy/SciPy oracle "
                                          "(assembled K, SetupGMG, SolveMG, Grad)"}
        line["parity"] = {"F_rel_diff": abs(ro.F - res.F) / abs(ro.F),
                          "design_max_abs_diff": float(np.abs(ro.x - res.x).max()),
                          "same_accept_reject": [h["it"] for h in ro.history] == [h["it"] for h in res.history]}
    print(json.dumps(line))
    return 0


def run_serving(args):
    """Serving stream: 512 seeded requests (mesh nx x nx/2 x nx/2, nx in
    {32, 64, 96, 128}, MR factor 1 or 2, cantilever/bridge/torsion, GRF
    densities), each a mixed-precision MG-PCG solve to 1e-8 plus Grad,
    arriving as a Poisson process; admitted by slots and HBM budget."""
    import torch
    import tosp
    from tosp import workloads as W
    torch.cuda.set_device(0)
    reqs = W.serving_requests(args.serving_count, seed=7)
    pool = W.FieldPool(seed=7)
    probs, items = {}, []
    for nx, n, bc, idx, eta in reqs:
        key = (nx, bc)
        if key not in probs:
            probs[key] = W.serving_problem(nx, bc)
        items.append((probs[key], n, pool.field(nx, n, idx, eta), W.serving_levels(nx)))

    def submit(srv, item):
        pb, n, x, ng = item
        # cycle and omega unspecified for the stream: the reference defaults
        mg = tosp.default_mg(ngrids=ng, cycle=1, omega=W.REF_OMEGA, tolMG=1e-8, maxiterMG=1000, flexible=1,
                             maxstall=60, small_cycle_max=args.small_levels, cg_product=args.cg_product)
        return srv.submit(pb, x, mg=mg, precision=tosp.PREC_MIXED, mr_n=n, p=3.0, emin=1e-9, opfilter=1,
                          rmin=1.0 if n > 1 else 1.5)

    out = []
    srv = tosp.Server(max_slots=args.slots, hbm_budget_bytes=int(args.budget_gb * (1 << 30)))
    seen = {}
    for it in items:                                   # warm-up: handles per shape, one request each
        k = (id(it[0]), it[1])
        if k not in seen:
            pb, n, x, ng = it
            mg = tosp.default_mg(ngrids=ng, cycle=1, omega=W.REF_OMEGA, tolMG=1e-8, maxiterMG=1000, flexible=1,
                                 maxstall=60, small_cycle_max=args.small_levels, cg_product=args.cg_product)
            if args.prepare > 0:
                srv.prepare(pb, count=args.prepare, mg=mg, precision=tosp.PREC_MIXED, mr_n=n,
                            rmin=1.0 if n > 1 else 1.5)
            seen[k] = submit(srv, it)
    for rid in seen.values():
        srv.wait(rid)
        srv.result(rid)
    clocks = Clocks(0)
    clocks.start()
    for lam in [float(r) for r in args.rates.split(",")]:
        arrivals = np.cumsum(np.random.default_rng(7).exponential(1.0 / lam, len(items)))
        ids = []
        t0 = time.perf_counter()
        for item, ta in zip(items, arrivals):
            dt = t0 + ta - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids.append(submit(srv, item))
        stats = []
        for rid in ids:
            srv.wait(rid)
            stats.append(srv.result(rid)[2])
        t1 = time.perf_counter()
        for k, st in enumerate(stats):
            if st["relres"] > 1e-8 or st["status"] != 0:
                nx, n, bc, idx, eta = reqs[k]
                print(json.dumps({"unconverged": [nx, n, bc, idx, round(eta, 4)], "it": st["it"],
                                  "relres": st["relres"], "status": st["status"]}), file=sys.stderr)
        lat = np.array([st["ms_latency"] for st in stats])
        out.append({"rate_per_s": lam, "solves_per_s": round(len(ids) / (t1 - t0), 3),
                    "p50_ms": round(float(np.percentile(lat, 50)), 2), "p99_ms": round(float(np.percentile(lat, 99)), 2),
                    "mean_run_ms": round(float(np.mean([st["ms_run"] for st in stats])), 2),
                    "max_it": int(max(st["it"] for st in stats)),
                    "fp64_fallbacks": int(sum(1 for st in stats if st["precision"] == 0)),
                    "all_converged": bool(all(st["relres"] <= 1e-8 for st in stats))})
        print(json.dumps(out[-1]), file=sys.stderr)
    clk = clocks.stop()
    counters = srv.counters()
    srv.close()
    best = max(out, key=lambda r: r["solves_per_s"])
    line = {"metric": "serving stream: solves/s and p50/p99 latency (mixed MG-PCG to 1e-8 + Grad)",
            "value": best["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
            "data": "synthetic", "dtype": "f64 outer CG / f32+bf16 V-cycle",
            "config": {"workload": "serving stream seed 7", "requests": len(items), "slots": args.slots,
                       "hbm_budget_gb": args.budget_gb, "small_levels": args.small_levels,
                       "cg_product": args.cg_product,
                       "mesh_nx": list(W.SERVING_NX), "mr_n": [1, 2],
                       "cycle": "W", "omega": W.REF_OMEGA,
                       "bc": list(W.SERVING_BC)},
            "rates": out, "clocks": clk, "runner": counters}
    print(json.dumps(line))
    return 0


def run_sweep(args):
    """Multigrid settings per precision on the benchmark workload: V/W cycle,
    Jacobi sweeps, omega and grid count, each arm timed over a few solves
    (setup + solve + Grad, device-resident inputs).  One JSON line with every
    setting and each precision's fastest."""
    import ctypes as C
    import itertools
    import torch
    import tosp
    from tosp.workloads import WORKLOADS, build_workload
    torch.cuda.set_device(0)
    spec = WORKLOADS[args.workload]
    pb, n, xfil, spec = build_workload(args.workload, filter_fn=lambda x: x)
    dev = torch.device("cuda", 0)
    xfil_d = torch.tensor(xfil, dtype=torch.float64, device=dev)
    f_d = torch.tensor(pb.f, dtype=torch.float64, device=dev)
    u_d = torch.zeros(pb.freedofs.size, dtype=torch.float64, device=dev)
    ufull_d = torch.zeros(3 * pb.nnodes, dtype=torch.float64, device=dev)
    g_d = torch.zeros(xfil.size, dtype=torch.float64, device=dev)
    fidx_d = torch.tensor(pb.freedofs, dtype=torch.int64, device=dev)
    lib = tosp._lib
    rows = []
    grids = [int(v) for v in args.sweep_grids.split(",")]
    # arms: (name, precision, cg_product, replace_drop)
    arms = [("mixed_cg64", tosp.PREC_MIXED, 0, 0.1), ("fp64", tosp.PREC_FP64, 0, 0.1)]
    arms += [("mixed_cg32", tosp.PREC_MIXED, 1, float(d)) for d in args.sweep_drops.split(",")]
    for (arm, prec, cgp, drop), cycle, (nu1, nu2), omega, ng in itertools.product(
            arms, (0, 1), ((1, 1), (1, 2), (2, 2), (3, 3)), (0.5, 0.6), grids):
        mg = tosp.default_mg(ngrids=ng, cycle=cycle, omega=omega, smoothiter1=nu1, smoothiter2=nu2, tolMG=1e-8,
                             maxiterMG=1000, flexible=1, cg_product=cgp, replace_drop=drop)
        tag = {"prec": arm, "cycle": "VW"[cycle], "sweeps": [nu1, nu2], "omega": omega}
        if cgp:
            tag["replace_drop"] = drop
        try:
            s = tosp.Solver(pb, mg, precision=prec, mr_n=n, p=3.0, emin=1e-9, opfilter=1, rmin=spec["rmin"])
        except tosp.TospError as e:
            rows.append(dict(tag, ngrids=ng, error=str(e)[:120]))
            continue

        def step():
            s.SetupGMG(xfil_d)
            u_d.zero_()
            it, rr = C.c_int32(), C.c_double()
            rc = lib.tosp_solve_mg(s.h, u_d.data_ptr(), f_d.data_ptr(), u_d.numel(), C.byref(it), C.byref(rr))
            ufull_d.zero_()
            ufull_d[fidx_d] = u_d
            lib.tosp_grad(s.h, ufull_d.data_ptr(), ufull_d.numel(), g_d.data_ptr(), None, g_d.numel())
            return rc, it.value, rr.value
        rc, it, rr = step()
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.sweep_steps):
            rc, it, rr = step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.sweep_steps
        rows.append(dict(tag, ngrids=s.info()["ngrids"], status=rc, it=it, relres=rr, ms=round(ms, 3),
                         solves_per_s=round(1000.0 / ms, 3) if rc == 0 else None,
                         replacements=s.stats()["replacements"]))
        print(json.dumps(rows[-1]), file=sys.stderr)
        s.close()
    ok = [r for r in rows if r.get("solves_per_s")]
    best = {p: max((r for r in ok if r["prec"] == p), key=lambda r: r["solves_per_s"])
            for p in ("mixed_cg64", "mixed_cg32", "fp64")}
    print(json.dumps({"metric": "multigrid settings sweep (solves/s, setup + solve to 1e-8 + Grad)",
                      "workload": args.workload, "rows": rows, "best": best,
                      "best_over_best_fp64": {p: round(best[p]["solves_per_s"] / best["fp64"]["solves_per_s"], 3)
                                              for p in ("mixed_cg64", "mixed_cg32")}}))
    return 0


def profile_filter(args):
    import torch
    import tosp
    from tosp.workloads import WORKLOADS
    spec = WORKLOADS[args.workload]
    pb = tosp.problems.cantilever(*spec["dims"])
    n = spec["n"]
    s = tosp.Solver(pb, tosp.default_mg(ngrids=args.ngrids or spec["ngrids"]), precision=tosp.PREC_MIXED, mr_n=n,
                    p=3.0, emin=1e-9, opfilter=1, rmin=spec["rmin"])   # launches the weights pass
    nd = pb.nelem * n ** 3
    x = torch.rand(nd, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    y = torch.empty_like(x)
    for trans in (0, 1):
        rc = tosp._lib.tosp_apply_filter(s.h, x.data_ptr(), y.data_ptr(), nd, trans)
        if rc != 0:
            raise tosp.TospError(rc, tosp._lib.tosp_last_error(s.h).decode())
    torch.cuda.synchronize()
    s.close()
    print("profile-filter done")
    return 0


def profile_kernels(args):
    import torch
    import tosp
    from tosp.workloads import WORKLOADS, build_workload
    spec = WORKLOADS[args.workload]
    pb, n, xfil, spec = build_workload(args.workload, filter_fn=lambda x: x)
    mg = tosp.default_mg(ngrids=args.ngrids or spec["ngrids"], cycle=0, omega=spec["omega"], tolMG=1e-8,
                         maxiterMG=1000, flexible=1, cg_product=args.cg_product)
    s = tosp.Solver(pb, mg, precision=tosp.PREC_MIXED, mr_n=n, p=3.0, emin=1e-9, opfilter=1, rmin=spec["rmin"])
    s.SetupGMG(xfil)
    r = np.random.default_rng(0).standard_normal(pb.freedofs.size)
    s.KelemProd(r)       # one FP64 product (the outer CG's operator)
    s.MGCycle(r)         # one V-cycle: two launches of the V-cycle's finest operator
    if args.cg_product:
        s.KelemProdCG32(r)   # one launch of the CG's tensor-core product
    if args.profile_solve:
        u, it, rr, rc = s.SolveMG(np.zeros(pb.f.size), pb.f)   # one full mixed solve
        print("solve iterations", it)
    torch.cuda.synchronize()
    s.close()
    print("profile run done")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tosp", choices=["tosp", "reference"])
    ap.add_argument("--workload", default="cantilever192x96x96_mr2")
    ap.add_argument("--fp64-steps", type=int, default=0, help="timed steps of the FP64 arm (0: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-w-cycle", action="store_true", help="skip the secondary W-cycle measurement")
    ap.add_argument("--ngrids", type=int, default=0, help="override the workload's grid count")
    ap.add_argument("--flexible", type=int, default=1, help="flexible (Polak-Ribiere) CG beta in both arms")
    ap.add_argument("--cg-product", type=int, default=1, choices=[0, 1],
                    help="mg.cg_product of the headline mixed arm (the other value is timed beside it): 0 FP64 "
                         "product every CG iteration, 1 tensor-core product with FP64 residual replacement")
    ap.add_argument("--slp", default="", choices=["", "config0", "config3"],
                    help="full SLP loop: config0 = 48x24x24 cantilever, FP64, 20 iterations; config3 = 160x80x40 "
                         "bridge (reference axes), MR 3, mixed precision, 100 iterations + GradProj")
    ap.add_argument("--slp-iters", type=int, default=0)
    ap.add_argument("--check-cpu", action="store_true", help="config0: run the same SLP loop on the oracle")
    ap.add_argument("--lp", default="", choices=["", "highs", "knapsack"], help="LP solver of the SLP loop")
    ap.add_argument("--serving", action="store_true",
                    help="serving stream (seed 7): Poisson arrivals at --rates, p50/p99 latency and solves/s")
    ap.add_argument("--sweep", action="store_true",
                    help="multigrid settings per precision (cycle, sweeps, omega, grids) on the workload")
    ap.add_argument("--sweep-grids", default="4,5")
    ap.add_argument("--sweep-drops", default="0.1", help="sweep: replace_drop values of the cg_product 1 arm")
    ap.add_argument("--sweep-steps", type=int, default=3)
    ap.add_argument("--rates", default="10,20,50,100,200,500")
    ap.add_argument("--serving-count", type=int, default=512)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--prepare", type=int, default=2, help="serving: idle handles created per shape before the stream")
    ap.add_argument("--small-levels", type=int, default=0,
                    help="serving: mg.small_cycle_max of the requests (0: off; k > 0: the levels with at most k "
                         "nodes run as the persistent cycle, one launch per visit for a whole shape batch)")
    ap.add_argument("--budget-gb", type=float, default=64.0)
    ap.add_argument("--profile-solve", action="store_true",
                    help="with --profile-kernels: also one full mixed-precision solve (launch lists)")
    ap.add_argument("--profile-filter", action="store_true",
                    help="one handle on the workload's density mesh: the filter weights, then one forward and one "
                         "transposed ApplyFilter on device vectors (a short run for ncu captures of the filter)")
    ap.add_argument("--profile-kernels", action="store_true",
                    help="one mixed-precision handle: setup, one FP64 product and one V-cycle, then exit "
                         "(a short run for ncu captures of the operator kernels)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.profile_kernels:
        return profile_kernels(args)
    if args.profile_filter:
        return profile_filter(args)
    if args.serving:
        return run_serving(args)
    if args.sweep:
        return run_sweep(args)
    if args.slp:
        return run_slp(args)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    import tosp
    from tosp.workloads import build_workload

    from tosp import replicas

    def barrier():
        replicas.barrier()

    def max_over_ranks(v):
        return replicas.max_over_ranks(v, device="cuda")

    # ---- workload -------------------------------------------------------------
    holder = {}

    def gpu_filter(x):
        return holder["s64"].ApplyFilter(x)

    from tosp.workloads import WORKLOADS
    spec0 = WORKLOADS[args.workload]
    nelx, nely, nelz = spec0["dims"]
    pb0 = tosp.problems.cantilever(nelx, nely, nelz)
    ngrids = args.ngrids or spec0["ngrids"]
    mg = tosp.default_mg(ngrids=ngrids, cycle=0, omega=spec0["omega"], smoothiter1=1, smoothiter2=1, tolMG=1e-8,
                         maxiterMG=1000, flexible=args.flexible)
    n = spec0["n"]
    kw = dict(mr_n=n, p=3.0, emin=1e-9, opfilter=1, rmin=spec0["rmin"])
    holder["s64"] = tosp.Solver(pb0, mg, precision=tosp.PREC_FP64, **kw)
    pb, n, xfil, spec = build_workload(args.workload, filter_fn=gpu_filter)
    s64 = holder["s64"]
    mg_cg = {}
    for cgp in (0, 1):
        mg_cg[cgp] = tosp.MgParams.from_buffer_copy(mg)
        mg_cg[cgp].cg_product = cgp
    arm_name = {0: "mixed_cg64", 1: "mixed_cg32"}
    smx = tosp.Solver(pb, mg_cg[args.cg_product], precision=tosp.PREC_MIXED, **kw)
    smx_alt = tosp.Solver(pb, mg_cg[1 - args.cg_product], precision=tosp.PREC_MIXED, **kw)
    dev = torch.device("cuda", local)
    xfil_d = torch.tensor(xfil, dtype=torch.float64, device=dev)
    f_d = torch.tensor(pb.f, dtype=torch.float64, device=dev)
    u_d = torch.zeros(pb.freedofs.size, dtype=torch.float64, device=dev)
    ufull_d = torch.zeros(3 * pb.nnodes, dtype=torch.float64, device=dev)
    g_d = torch.zeros(xfil.size, dtype=torch.float64, device=dev)
    fidx_d = torch.tensor(pb.freedofs, dtype=torch.int64, device=dev)
    lib = tosp._lib
    import ctypes as C

    def step_dev(s):
        s.SetupGMG(xfil_d)
        u_d.zero_()
        it, rr = C.c_int32(), C.c_double()
        rc = lib.tosp_solve_mg(s.h, u_d.data_ptr(), f_d.data_ptr(), u_d.numel(), C.byref(it), C.byref(rr))
        if rc != 0:
            raise tosp.TospError(rc, lib.tosp_last_error(s.h).decode())
        ufull_d.index_copy_(0, fidx_d, u_d)    # U(freedofs) = u; fixed entries stay zero
        rc = lib.tosp_grad(s.h, ufull_d.data_ptr(), ufull_d.numel(), g_d.data_ptr(), None, g_d.numel())
        if rc != 0:
            raise tosp.TospError(rc, lib.tosp_last_error(s.h).decode())
        return it.value, rr.value

    def timed(s, steps, warmup):
        for _ in range(warmup):
            step_dev(s)
        torch.cuda.synchronize()
        barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        its = []
        l0 = tosp.kernel_launches()
        ev[0].record()
        for k in range(steps):
            its.append(step_dev(s))
            ev[k + 1].record()
        torch.cuda.synchronize()
        launches = tosp.kernel_launches() - l0
        barrier()
        per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
        return per, its, launches

    clocks = Clocks(local)
    clocks.start()
    per_mx, its_mx, launches = timed(smx, args.steps, args.warmup)
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(per_mx))
    fp64_steps = args.fp64_steps or args.steps
    per_64, its_64, _ = timed(s64, fp64_steps, args.warmup)
    total64 = max_over_ranks(sum(per_64))
    # the other mixed arm (cg_product), same steps
    per_alt, its_alt, _ = timed(smx_alt, args.steps, args.warmup)
    total_alt = max_over_ranks(sum(per_alt))
    # solutions of every arm (outside the timed regions) for the true residuals
    # and the errors against FP64
    sol = {}
    replacements = {}
    for key, s in ((arm_name[args.cg_product], smx), (arm_name[1 - args.cg_product], smx_alt), ("fp64", s64)):
        step_dev(s)
        g_full = g_d.cpu().numpy().copy()
        sol[key] = (u_d.cpu().numpy().copy(), g_full)
        replacements[key] = s.stats()["replacements"]
    stats_mx = smx.stats()

    # ---- end to end through the C ABI with pinned host buffers ------------------
    xfil_h = torch.tensor(xfil, dtype=torch.float64).pin_memory()
    f_h = torch.tensor(pb.f, dtype=torch.float64).pin_memory()
    u_h = torch.zeros(pb.freedofs.size, dtype=torch.float64).pin_memory()
    uf_h = torch.zeros(3 * pb.nnodes, dtype=torch.float64).pin_memory()
    g_h = torch.zeros(xfil.size, dtype=torch.float64).pin_memory()
    fidx_h = torch.tensor(pb.freedofs, dtype=torch.int64)

    def step_host(s):
        lib.tosp_setup_gmg(s.h, xfil_h.data_ptr(), xfil_h.numel())
        u_h.zero_()
        it, rr = C.c_int32(), C.c_double()
        lib.tosp_solve_mg(s.h, u_h.data_ptr(), f_h.data_ptr(), u_h.numel(), C.byref(it), C.byref(rr))
        # U(freedofs) = u; the fixed entries of uf_h stay zero (never written)
        uf_h.index_copy_(0, fidx_h, u_h)
        lib.tosp_grad(s.h, uf_h.data_ptr(), uf_h.numel(), g_h.data_ptr(), None, g_h.numel())
        return it.value

    e2e_steps = max(3, args.steps)
    step_host(smx)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        step_host(smx)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    h2d = 8 * (xfil.size + 2 * pb.freedofs.size + 3 * pb.nnodes)
    d2h = 8 * (pb.freedofs.size + xfil.size)
    # parity guard: the host path gives the same gradient as the device path
    assert torch.allclose(g_h, g_d.cpu(), rtol=1e-6, atol=1e-12 * float(g_h.abs().max()))

    # true relative residuals ||f - K u|| / ||f|| of both arms' solutions, with
    # one FP64 product each (not the CG's recurrence residual)
    relres_true = {}
    nf = float(np.linalg.norm(pb.f))
    for key, (u_sol, _) in sol.items():
        relres_true[key] = float(np.linalg.norm(pb.f - s64.KelemProd(u_sol)) / nf)

    # ---- kernel roofline (finest-level operators) ---------------------------------
    peaks, peak_kind = load_peaks()
    s_cg32 = smx if args.cg_product == 1 else smx_alt
    ms_op32 = smx.time_operator(tosp.PREC_MIXED, reps=10)
    ms_op64 = smx.time_operator(tosp.PREC_FP64, reps=10)
    ms_opcg = s_cg32.time_operator(2, reps=10)
    ndof, nsub, nel = 3 * pb.nnodes, xfil.size, pb.nelem
    bytes32 = 4 * ndof + 4 * ndof + 2 * nsub + ndof      # x, y fp32, SIMP bf16, free mask
    bytescg = 4 * ndof + 4 * ndof + 4 * nsub + ndof      # x, y fp32, SIMP fp32, free mask
    bytes64 = 8 * ndof + 8 * ndof + 8 * nsub + ndof
    flops = nel * n ** 3 * 1200                           # 576 FMA + 24 scalings per sub-block
    it_mx = its_mx[-1][0]
    applies32 = 2 * (it_mx - 1)                           # residual + post-smooth per V-cycle
    if args.cg_product == 1:
        appliescg = it_mx - 1                             # the CG's product, every iteration
        applies64 = stats_mx["replacements"]              # residual replacements
    else:
        appliescg = 0
        applies64 = it_mx - 1                             # the CG's product, every iteration
    traffic = {}
    tp = os.path.join(ROOT, "profiles", "operator_traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(args.workload, {})
    ach32 = bytes32 / (ms_op32 * 1e-3) / 1e9
    achcg = bytescg / (ms_opcg * 1e-3) / 1e9
    ach64 = bytes64 / (ms_op64 * 1e-3) / 1e9
    ach64_tf = flops / (ms_op64 * 1e-3) / 1e12
    fma_exec = nel * (2148 if n == 2 else 300 * (n ** 3 + 2))      # FMAs the FP64 kernel executes per launch
    share32 = applies32 * ms_op32 / (total_ms / args.steps)
    sharecg = appliescg * ms_opcg / (total_ms / args.steps)
    share64 = applies64 * ms_op64 / (total_ms / args.steps)
    rf64 = {"bound": "hbm", "achieved": round(ach64, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": round(ach64 / peaks["hbm_gbs"], 4), "traffic": traffic.get("fp64_operator_bytes_per_launch"),
            "kernel": "k_fine_apply64<2> (outer-CG FP64 operator)", "algorithmic_bytes_per_launch": bytes64,
            "ms_per_launch": round(ms_op64, 4), "peak_source": peak_kind,
            "fp64_pipe": {"executed_fma_per_launch": fma_exec,
                          "achieved_tflops": round(2 * fma_exec / (ms_op64 * 1e-3) / 1e12, 2),
                          "nominal_peak_tflops": 37.0}}
    rf32 = {"bound": "hbm", "achieved": round(ach32, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": round(ach32 / peaks["hbm_gbs"], 4), "traffic": traffic.get("fp32_operator_bytes_per_launch"),
            "kernel": f"k_fine_apply_tc<{n}> (V-cycle operator, tcgen05 sub-cell block products)"
                      if (n * pb.nely) % 2 == 0 else "k_fine_apply<float,bf16> (V-cycle operator)",
            "algorithmic_bytes_per_launch": bytes32, "ms_per_launch": round(ms_op32, 4), "peak_source": peak_kind}
    rfcg = {"bound": "hbm", "achieved": round(achcg, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": round(achcg / peaks["hbm_gbs"], 4), "traffic": traffic.get("cg32_operator_bytes_per_launch"),
            "kernel": f"k_fine_apply_tc<{n},float> (CG product of cg_product 1, FP32 factors)",
            "algorithmic_bytes_per_launch": bytescg, "ms_per_launch": round(ms_opcg, 4), "peak_source": peak_kind}
    # the dominant kernel of the timed step carries the contract's roofline
    ranked = sorted([(share64, rf64), (share32, rf32), (sharecg, rfcg)], key=lambda t: -t[0])
    roofline, roofline_other = ranked[0][1], [r for _, r in ranked[1:]]
    kernels = {
        "fine_op_fp32": {"ms": round(ms_op32, 4), "GBps": round(ach32, 1), "per_solve": applies32,
                         "share_of_step": round(share32, 3)},
        "fine_op_cg32": {"ms": round(ms_opcg, 4), "GBps": round(achcg, 1), "per_solve": appliescg,
                         "share_of_step": round(sharecg, 3)},
        "fine_op_fp64": {"ms": round(ms_op64, 4), "TFLOPs_fp64_dense_formula": round(ach64_tf, 2),
                         "GBps": round(ach64, 1), "per_solve": applies64, "share_of_step": round(share64, 3)},
    }

    value = world * args.steps / (total_ms * 1e-3)
    lat = np.array(per_mx)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 outer CG / f32+bf16 V-cycle",
        "data": "synthetic",
        "config": bench_config(args, spec0, pb, n, ngrids, world),
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3), "p99": round(float(np.percentile(lat, 99)), 3)},
        "mixed_arm": arm_name[args.cg_product],
        "pcg_iterations": {arm_name[args.cg_product]: it_mx, arm_name[1 - args.cg_product]: its_alt[-1][0],
                           "fp64": its_64[-1][0]},
        "relres": {arm_name[args.cg_product]: its_mx[-1][1], arm_name[1 - args.cg_product]: its_alt[-1][1],
                   "fp64": its_64[-1][1]},
        "relres_true": relres_true,
        "residual_replacements": replacements,
        "cg": "flexible beta r'(s - s_old)/rho_old in every arm" if args.flexible else "reference beta",
        "fp64": {"value": round(world * fp64_steps / (total64 * 1e-3), 4), "unit": "solves/s",
                 "ms_per_step": round(total64 / fp64_steps, 3), "steps": fp64_steps},
        arm_name[1 - args.cg_product]: {
            "value": round(world * args.steps / (total_alt * 1e-3), 4), "unit": "solves/s",
            "ms_per_step": round(total_alt / args.steps, 3), "steps": args.steps,
            "over_fp64": round((args.steps / total_alt) / (fp64_steps / total64), 3)},
        "mixed_over_fp64": round((args.steps / total_ms) / (fp64_steps / total64), 3),
        "setup_ms": round(stats_mx["ms_setup"], 3),
        "e2e": {"value": round(world * e2e_steps / e2e_s, 4), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "roofline_other_operator": roofline_other,
        "kernels": kernels,
        "clocks": clk,
    }
    if not args.no_w_cycle:
        # the reference's default cycle (W, I/TopOpt3D.m:172-174) on the same
        # workload, both arms, as a secondary figure
        mgw = tosp.MgParams.from_buffer_copy(mg_cg[args.cg_product])
        mgw.cycle = 1
        mgw64 = tosp.MgParams.from_buffer_copy(mgw)
        mgw64.cg_product = 0
        smw = tosp.Solver(pb, mgw, precision=tosp.PREC_MIXED, **kw)
        s6w = tosp.Solver(pb, mgw64, precision=tosp.PREC_FP64, **kw)
        per_w, its_w, _ = timed(smw, 3, 3)
        per_w64, its_w64, _ = timed(s6w, 3, 3)
        tw, tw64 = max_over_ranks(sum(per_w)), max_over_ranks(sum(per_w64))
        line["w_cycle"] = {
            "mixed": {"value": round(world * 3 / (tw * 1e-3), 4), "ms_per_step": round(tw / 3, 3),
                      "pcg_iterations": its_w[-1][0], "relres": its_w[-1][1]},
            "fp64": {"value": round(world * 3 / (tw64 * 1e-3), 4), "ms_per_step": round(tw64 / 3, 3),
                     "pcg_iterations": its_w64[-1][0], "relres": its_w64[-1][1]},
            "mixed_over_fp64": round(tw64 / tw, 3), "unit": "solves/s"}
        smw.close()
        s6w.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # one complete solve of the same workload on the host cores (the
        # reference's assembled path restated in C/OpenMP), which is also the
        # FP64 oracle the GPU arms' errors are stated against
        ca, _, _, _, _, _ = cpu_solver(args, spec0)
        cs = cpu_whole_solve(ca, pb, xfil)
        cores = host_cores()
        line["cpu_baseline"] = {
            "value": round(1.0 / cs["total_s"], 6), "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": (f"one complete solve of the same workload, measured: SetupGMG {cs['setup_s']:.1f} s + "
                       f"SolveMG {cs['solve_s']:.1f} s ({cs['it'] - 1} PCG iterations to {cs['relres']:.2e}) + Grad "
                       f"{cs['grad_s']:.1f} s, the reference's assembled path restated in C/OpenMP on {cores} "
                       f"host threads")}
        uo, go = cs["u"][pb.freedofs], cs["g"]
        Fo = float(pb.f @ uo)
        line["error_vs_fp64_oracle"] = {
            key: {"u_rel_max": float(np.abs(u_sol - uo).max() / np.abs(uo).max()),
                  "F_rel": float(abs(pb.f @ u_sol - Fo) / abs(Fo)),
                  "dFdrho_rel_max": float(np.abs(g_sol - go).max() / np.abs(go).max())}
            for key, (u_sol, g_sol) in sol.items()}
        line["error_vs_fp64_oracle"]["oracle"] = "the CPU solve above (assembled K, FP64, reference beta)"
        line["relres_true_cpu_operator"] = {
            key: float(np.linalg.norm((pb.f_full() - ca.apply(0, _full(pb, u_sol)))[pb.freedofs]) / nf)
            for key, (u_sol, _) in sol.items()}
    if rank == 0:
        print(json.dumps(line))
    smx.close()
    smx_alt.close()
    s64.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

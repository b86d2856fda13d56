"""Benchmark: ms per Stokes solve to relative residual 1e-8 on one B200.

Workload (default): layered257 — 257^3 nodes (67.3 M unknowns), 6 levels
(257-131-68-36-20-12), layered lithosphere with viscosity 1e4 at the bottom
to 1 at the top (45 constant layers), a dense slab block (viscosity 1e3,
density +1), a weak zone (viscosity 1e-2), free-slip box, 2x2x2 markers per
cell (134 M markers), seed 5.  Inputs are seeded synthetic data of those
shapes (no public dataset exists).

One step = one complete Stokes solve (coarse viscosities, cell factors,
coarsest LU and inverse, FP64 outer GCR iterations whose preconditioner is
one FP32 V-cycle) from a zero initial guess
on node fields resident in HBM, to ||b - Ax|| / ||b|| <= 1e-8 in FP64.  The
line also reports the plain FP64 solve (FP64 GCR, FP64 V-cycle), the
relative L2 error of each field against the FP64 GPU solve and against the
oracle port's converged solution, the end-to-end host-array call, one RK4
marker advection step, one heat-equation step, and the oracle port on the
host cores (cpu_baseline).

    python bench.py [--gpus N --steps K --warmup W] [--config 1|2|3|4|5] [--impl reference]

Under torchrun (N > 1) every rank solves its own replica (the solve does not
shard); the timed region is bracketed by a barrier and the max over ranks is
reported.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms per Stokes solve to rel.residual 1e-8 (mixed vs FP64, 1 B200); HBM GB/s"
WORKLOADS = {
    1: "sphere33: 33^3 nodes, 3 levels, centred sphere viscosity 1e3 radius 0.2, 4x4x4 markers/cell, seed 1",
    2: ("spheres65: 65^3 nodes, 4 levels, 8 spheres viscosity 1e-3..1e3 (contrast 1e6), "
        "2x2x2 markers/cell, free-slip box, seed 2"),
    3: ("spheres129: 129^3 nodes, 5 levels, 20 spheres viscosity 1e-2..1e4 (contrast 1e6), "
        "2x2x2 markers/cell, free-slip box, seed 3"),
    4: ("batch64: 64 independent models, nodes per axis uniform in {33,49,65,81,97}, 1-10 spheres viscosity "
        "1e-2..1e2, 2x2x2 markers/cell, free-slip boxes, seed 4; solved concurrently (one stream and CUDA graphs "
        "per instance) vs one after another"),
    5: ("layered257: 257^3 nodes, 6 levels, 45 layers viscosity 1e4..1 with depth, slab 1e3 (density +1), "
        "weak zone 1e-2, 2x2x2 markers/cell, free-slip box, seed 5"),
}
CONFIG_IDX = 5
WORKLOAD = WORKLOADS[CONFIG_IDX]
# Algorithmic bytes of the dominant kernel, counted per node as the scope
# table counts them: one FP32 sweep of the cell-block smoother (both colours)
# reads the 4 unknowns, 4 right-hand sides and 4 viscosity fields once and
# writes the 4 unknowns once, 64 B per node; one colour pass is half a sweep.
# (The stored-factor smoother also reads 22 factors per cell of the colour,
# 44 B per node and pass, which the measured DRAM traffic shows but the
# algorithmic count does not include.)
SWEEP_BYTES_PER_NODE = 64
KERNEL_OF_SMOOTHER = {0: "k_vanka<float>", 1: "k_vanka_stored<float>", 2: "k_vanka_full<float>",
                      3: "k_vanka_fast<float>"}


def pass_bytes(nodes):
    """Algorithmic bytes of one level-0 colour pass (half a sweep)."""
    return SWEEP_BYTES_PER_NODE * nodes // 2


# Marker advection: per marker read x, y, z (12 B) and the type (1 B), write
# x, y, z (12 B); per node read the FP64 velocities (24 B) and write and
# re-read their float copies (12 + 12 B) once (the 8-node gathers of the
# four Runge-Kutta stages hit L2).
MOVEMARK_BYTES_PER_MARKER = 25
MOVEMARK_BYTES_PER_NODE = 48


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=CONFIG_IDX)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--solve-only", action="store_true",
                    help="warm-up + timed resident solves + smoother timing only (profiling runs)")
    ap.add_argument("--heat-only", action="store_true",
                    help="only the heat-equation step on the workload's grid, with seeded velocities and "
                         "stresses instead of a solve (profiling runs)")
    ap.add_argument("--restart", type=int, default=16, help="GCR restart length")
    ap.add_argument("--smoother", type=int, default=1,
                    help="smoother when --tune-iters 0 (profiling runs; the default run autotunes)")
    ap.add_argument("--sweep-growth", type=int, default=2, help="sweep growth per level when --tune-iters 0")
    ap.add_argument("--max-iter", type=int, default=200, help="outer iteration cap (profiling runs)")
    ap.add_argument("--tune-iters", type=int, default=12,
                    help="outer iterations per autotuner trial (run once, before the timed region); 0 = no tuning")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(nodes):
    """DRAM bytes of one level-0 FP32 stored-factor smoother pass from the
    committed ncu summary (captured at 129^3; the pass streams every node
    once, so its traffic scales with the node count), or None."""
    p = os.path.join(ROOT, "profiles", "ncu_vanka_stored_f32_level0.txt")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_node:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) * nodes if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(gpus):
    rank, world = 0, 1
    if gpus > 1 or "WORLD_SIZE" in os.environ:
        import datetime
        import torch
        import torch.distributed as dist
        rank = int(os.environ.get("RANK", 0))
        world = int(os.environ.get("WORLD_SIZE", 1))
        local = int(os.environ.get("LOCAL_RANK", rank))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return rank, world, local, dist
    return rank, world, 0, None


def cpu_solve_ms(model, threads: int, steps: int = 1):
    """The oracle port (same algorithm, FP64, OpenMP) on the host cores."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    if not O.available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all"], check=True, stdout=subprocess.DEVNULL)
    times, its = [], []
    f = O.ronurecalc(model)
    for _ in range(steps):
        s = O.OracleSolver(model, npre=[4] * (model.multinum + 1), npost=[4] * (model.multinum + 1))
        t0 = time.perf_counter()
        s.set_fields(f)
        h = s.solve(tol=1e-8, max_cycles=200, restart=16)
        times.append((time.perf_counter() - t0) * 1e3)
        its.append(len(h) - 1)
        s.close()
    return times, its


def reference_own_solver(model, cycles: int = 6):
    """Bounded run of the reference's own vpiterate() path (oracle/_ref):
    first iteration (assembly + direct coarsest solve) and further V-cycles,
    reporting ms per cycle and the true residual reached."""
    from oracle import refdrv
    if not refdrv.available():
        return None
    r = refdrv.RefModel(model, npre=[4] * (model.multinum + 1), npost=[4] * (model.multinum + 1))
    t0 = time.perf_counter()
    r.ronurecalc()
    t1 = time.perf_counter()
    r.first_iteration()
    t2 = time.perf_counter()
    res = [r.residual()[0]]
    for _ in range(cycles):
        r.vcycle(False)
        res.append(r.residual()[0])
    t3 = time.perf_counter()
    return {"threads": r.num_threads(), "ronurecalc_ms": (t1 - t0) * 1e3, "first_iteration_ms": (t2 - t1) * 1e3,
            "ms_per_vcycle": (t3 - t2) * 1e3 / cycles, "true_rel_residual": res}


def run_reference(args):
    """The reference arm on the host cores: the oracle port (the reference's
    discretisation with the solver this build runs, C + OpenMP on every host
    core; the reference's own vpiterate() does not reach 1e-8 on these
    models, see reference_own_solver).  Small workloads: K full solves.
    Workloads above 8 M nodes: a full solve takes many minutes on the host,
    so the set-up is timed once and each step is one outer iteration (one
    warm-up, at most two timed); the value is set-up + iterations to 1e-8
    (from the oracle's own converged run, stored with the fixture) x the mean
    ms per iteration."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    from pardiso2_b200 import model as M
    m = M.config_model(args.config)
    threads = os.cpu_count() or 1
    big = m.nodenum > 8_000_000
    line = {"impl": "reference", "metric": METRIC, "unit": "ms", "n_gpus": args.gpus, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args.config, m, args.gpus)}
    if not big:
        n = args.warmup + args.steps
        times, its = cpu_solve_ms(m, threads, steps=max(1, n))
        timed = times[args.warmup:] or times
        v = statistics.mean(timed)
        line.update({"value": v, "steps": len(timed), "warmup": args.warmup, "ms_per_step": v,
                     "iterations": its[-1]})
        sample = "full solve of the workload to 1e-8 per step (oracle port: same discretisation and algorithm " \
                 "in C + OpenMP)"
    else:
        import ctypes as C
        os.environ["OMP_NUM_THREADS"] = str(threads)
        from oracle import oracle as O
        if not O.available():
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all"], check=True,
                           stdout=subprocess.DEVNULL)
        fx = fixture(args.config)
        nl = m.multinum + 1
        C.c_int.in_dll(O.lib(), "p2o_smoother").value = int(fx["oracle_smoother"]) if fx is not None else 2
        sweeps = [int(x) for x in fx["oracle_sweeps"]] if fx is not None else [4] * nl
        f = O.ronurecalc(m)
        so = O.OracleSolver(m, npre=sweeps, npost=sweeps)
        t0 = time.perf_counter()
        so.set_fields(f)
        setup_ms = (time.perf_counter() - t0) * 1e3
        warm, steps = min(args.warmup, 1), max(1, min(args.steps, 2))
        its_ms = []
        for k in range(warm + steps):
            t0 = time.perf_counter()
            so.solve(tol=0.0, max_cycles=1, restart=16)
            if k >= warm:
                its_ms.append((time.perf_counter() - t0) * 1e3)
        so.close()
        n_it = oracle_iters_to(fx["hist"], 1e-8) if fx is not None else None
        per_it = statistics.mean(its_ms)
        v = setup_ms + per_it * n_it if n_it else float("nan")
        line.update({"value": v, "steps": steps, "warmup": warm, "ms_per_step": per_it,
                     "setup_ms": setup_ms, "ms_per_iteration": per_it, "iterations_to_1e-8": n_it})
        sample = ("oracle port set-up once + one outer iteration per step (%d warm-up, %d timed); value = set-up "
                  "+ %s iterations to 1e-8 (the oracle's own converged run) x mean ms per iteration"
                  % (warm, steps, n_it))
    line["cpu_baseline"] = {"value": line["value"], "unit": "ms", "cores": threads, "kind": "port", "sample": sample}
    line["e2e"] = {"value": line["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    if not big:
        try:
            line["reference_own_solver"] = reference_own_solver(m)
        except Exception as e:  # the reference's own MG is bounded here, never required
            line["reference_own_solver"] = {"error": str(e)}
    else:
        nn = m.levels.total_nodes if hasattr(m.levels, "total_nodes") else m.nodenum
        line["reference_own_solver"] = {
            "not_run": "its row store (57 coefficients x 12 B per node of every level, %.1f GB) and per-thread "
                       "accumulation buffers (about 1.8 GB per thread) exceed the bounded run; it stalls far above "
                       "1e-8 on the smaller workloads" % (57 * 12 * nn / 1e9)}
    print(json.dumps(line), flush=True)


def shard_instances(sizes, world):
    """Greedy balance of instances (by node count, largest first) over ranks:
    returns the instance indices of every rank."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def heat_leg(prob, m, args, with_cpu: bool, synthetic: bool = False):
    """One thermal step (titerate) on the workload's grid through the public
    API: fixed z planes and insulating walls on every level, seeded thermal
    fields (thermal_fields), the resident solution's velocities (adiabatic
    heating) and its stresses / strain rates (shear heating), the workload's
    markers with types 0/1 (diffused) and 70 (reset to the node
    temperature).  All levels of the grid, 3 smoothing sweeps down and up,
    10 on the coarsest; a step of about 2.5 diffusion times of a cell (2000 s
    on the 65^3 unit box, scaled with the squared spacing on other grids) in
    sub-steps of at most 25 K, errors below 2e-3 K (above the float
    temperatures' error floor, about 1.2e-3 K at 129^3)."""
    import numpy as np
    from pardiso2_b200 import capi
    from pardiso2_b200 import model as M
    n = m.nodenum
    bc = M.with_thermal_bc(m)
    prob.ctx.heat_set_bc(bc, n)
    th = M.thermal_fields(m, seed=31, heat=(2e4, 8e4))
    if synthetic:
        rng = np.random.Generator(np.random.PCG64(32))
        vel = [(rng.random(n) * 0.02 - 0.01).astype(np.float32) for _ in range(3)]
        se = [(rng.random(n) * 2 - 1).astype(np.float32) for _ in range(12)]
    else:
        sol = prob.ctx.solution(n)
        vel = [np.ascontiguousarray(sol[k], np.float32) for k in ("vx", "vy", "vz")]
        st = {k: np.zeros(n, np.float32) for k in capi.Context.STRESS_KEYS}
        prob.ctx.stress_strain(st)
        se = [st[k] for k in capi.Context.STRESS_KEYS]
    nt = m.multinum
    pre = [3] * nt + [0]
    post = [0] + [3] * (nt - 1) + [10]
    hp = capi.heat_params(multinumt=nt, multicyct=1, pre=pre, post=post, heatmin=2e-3, max_cycles=200)
    q = np.arange(m.markx.size)
    mt = np.where(q % 9 == 4, 70, m.markt).astype(np.int8)
    markk = np.where(q % 3 == 0, 0.0, 900.0).astype(np.float32)
    markers = (m.markx, m.marky, m.markz, mt)
    dt = 2000.0 * (64.0 / (m.shape[0] - 1)) ** 2
    for _ in range(max(1, args.warmup)):
        prob.ctx.titerate(hp, dt, th, vel=vel, se=se, markers=markers, markk=markk)
    runs = [prob.ctx.titerate(hp, dt, th, vel=vel, se=se, markers=markers, markk=markk)[2] for _ in range(args.steps)]
    info = runs[-1]
    out = {"ms": statistics.mean(r.ms_total for r in runs), "nodes": n, "markers": int(q.size), "levels": nt + 1,
           "dt_s": dt,
           "substeps": info.substeps, "error_checks": info.cycles, "heatsum": info.heatsum, "heatmin": hp.heatmin,
           "converged": bool(info.converged), "launches": int(info.kernels),
           "timing": "CUDA events around the call, host<->device copies of the fields and markers included"}
    if with_cpu:
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__))))
        from oracle import oracle as O
        hpd = dict(timestep=dt, maxtkstep=hp.maxtkstep, heatmin=hp.heatmin, t0koef=1.0, t1koef=1.0, heatdif=1.0,
                   tdeep=hp.tdeep, zdeep=hp.zdeep, gx=m.params.gx, gy=m.params.gy, gz=m.params.gz, multicyct=1,
                   frictyn=1, adiabyn=1, max_cycles=200, pre=pre, post=post)
        t0 = time.perf_counter()
        _, _, oi = O.titerate(m.gx, m.gy, m.gz, nt, bc.bondt, bc.bondv1, bc.bondn1, hpd, th, vel=vel, se=se,
                              markers=markers, markk=markk)
        out["cpu_baseline"] = {"value": (time.perf_counter() - t0) * 1e3, "unit": "ms", "cores": 1, "kind": "port",
                               "sample": "the same step with the oracle port (lexicographic Gauss-Seidel, %d error "
                                         "checks)" % oi["cycles"]}
    return out


def run_batch(args, rank, world, local, dist):
    """The batched workload: this rank's share of the 64 instances, solved
    one after another and then all at once (p2_stokes_solve_batch)."""
    import numpy as np
    import torch
    import pardiso2_b200 as P
    from pardiso2_b200 import capi
    from pardiso2_b200 import model as M

    specs = M.batch_specs(64, 4)
    mine = shard_instances([n ** 3 for n, _, _ in specs], world)[rank]
    models, probs, tunes = [], [], []
    for i in mine:
        m = M.batch_model(*specs[i])
        p = P.StokesProblem(m, device=local, precision=0, tol=1e-8, restart=args.restart)
        p.ctx.upload_markers(m.markx, m.marky, m.markz, m.markt, m.rocks.n0, m.rocks.n1, m.rocks.ro)
        p.ctx.ronurecalc_resident()
        tunes.append(p.autotune(min(args.tune_iters, 8)).as_dict() if args.tune_iters > 0 else None)
        models.append(m)
        probs.append(p)
    ctxs = [p.ctx for p in probs]
    dofs = sum(m.real_dofs() for m in models)
    for _ in range(args.warmup):
        capi.solve_batch(ctxs)
    # one after another (each solve timed on its own stream)
    seq = []
    for _ in range(args.steps):
        seq.append(sum(c.solve_resident(check=False).ms_total for c in ctxs))
    # all at once
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    batch, lat, launches, ok = [], [], 0, True
    for _ in range(args.steps):
        infos, ms = capi.solve_batch(ctxs)
        batch.append(ms)
        lat.extend(x.ms_total for x in infos)
        launches += sum(x.kernels for x in infos)
        ok = ok and all(x.status == 0 for x in infos)
    torch.cuda.synchronize()
    clocks = clk.stop()
    if dist:
        dist.barrier()
    batch_ms, seq_ms = statistics.mean(batch), statistics.mean(seq)
    if dist:
        t = torch.tensor([batch_ms, seq_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        batch_ms, seq_ms = float(t[0].item()), float(t[1].item())
        d = torch.tensor([float(dofs)], dtype=torch.float64, device="cuda")
        dist.all_reduce(d)
        dofs_all = float(d.item())
    else:
        dofs_all = float(dofs)
    # end to end: node fields from pinned host memory, the batch, solutions back
    keys = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
    host = []
    for m, p in zip(models, probs):
        f = p.ctx.get_nodes(m.nodenum)
        pin = {k: torch.empty(m.nodenum, dtype=torch.float32, pin_memory=True).numpy() for k in keys}
        for k in keys:
            pin[k][:] = f[k]
        sol = {k: torch.empty(m.nodenum, dtype=torch.float64, pin_memory=True).numpy() for k in ("vx", "vy", "vz", "pr")}
        host.append((pin, sol))
    e2e = []
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for p, (pin, _) in zip(probs, host):
            p.ctx.set_nodes(pin)
        capi.solve_batch(ctxs)
        for p, (_, sol) in zip(probs, host):
            p.ctx._check(p.ctx.L.p2_get_solution(p.ctx.h, *[capi._ptr(sol[k]) for k in ("vx", "vy", "vz", "pr")]),
                         "p2_get_solution")
        if it >= args.warmup:
            e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = statistics.mean(e2e)
    if dist:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    nodes = sum(m.nodenum for m in models)
    # dominant kernel: level-0 colour pass of the smoother on the largest instance
    big = max(range(len(models)), key=lambda i: models[i].nodenum)
    sm_big = tunes[big]["smoother"] if tunes[big] else 1
    pass_ms = capi.DebugHooks(ctxs[big]).time_smoother(0, 40)
    bytes_per_launch = pass_bytes(models[big].nodenum)
    achieved = bytes_per_launch / (pass_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    line = {
        "metric": METRIC, "value": batch_ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": batch_ms, "higher_is_better": False, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32 V-cycle / f64 outer", "data": "synthetic",
        "config": {"workload": WORKLOADS[4], "instances": len(specs), "instances_per_rank": len(mine),
                   "unknowns": int(dofs_all), "l2": "working set of all instances (GBs) larger than L2",
                   "parallelism": ("instances sharded over %d ranks, " % world if world > 1 else "")
                   + "concurrent streams, host worker pool"},
        "converged": ok, "sequential_ms": seq_ms, "speedup_batch_vs_sequential": seq_ms / batch_ms,
        "unknowns_per_s": dofs_all / (batch_ms * 1e-3),
        "unknowns_per_s_sequential": dofs_all / (seq_ms * 1e-3),
        "instance_latency_ms": {"mean": statistics.mean(lat), "max": max(lat), "min": min(lat)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profile_traffic(models[big].nodenum) if sm_big == 1 else None,
                     "kernel": KERNEL_OF_SMOOTHER[sm_big]
                     + " level-0 colour pass, largest instance (%d^3)" % models[big].shape[0], "bytes_per_launch": bytes_per_launch, "ms_per_launch": pass_ms,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, burst)",
                     "timing": "each launch timed alone by CUDA events after a 256 MB L2 flush, mean of 40"},
        "clocks": clocks,
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 24 * nodes, "d2h_bytes_per_step": 32 * nodes},
        "autotune": {"smoother_full": sum(1 for t in tunes if t and t["smoother"] == 1),
                     "sweep_growth_2": sum(1 for t in tunes if t and t["sweep_growth"] == 2)},
    }
    for p in probs:
        p.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def config_dict(cfg, m, gpus):
    """The workload description both arms print (identical dicts)."""
    return {"workload": WORKLOADS.get(cfg, str(cfg)), "unknowns": m.real_dofs(), "levels": m.multinum + 1,
            "markers": int(m.markx.size),
            "l2": "flushed (256 MB write) before every step; the working set (GBs) exceeds L2",
            "parallelism": "replicas" if gpus > 1 else "1 GPU"}


def rel_l2(a, b):
    d = np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    nb = np.linalg.norm(np.asarray(b, np.float64))
    return float(d / nb) if nb > 0 else float(d)


FIXTURES = {3: "spheres129_solution.npz", 5: "layered257_solution.npz"}
SOL_KEYS = ("vx", "vy", "vz", "pr")


def fixture(cfg):
    path = os.path.join(ROOT, "tests", "golden", FIXTURES.get(cfg, "-"))
    return np.load(path) if os.path.exists(path) else None


def velocity_rel_l2(sol, ref):
    """Relative L2 error of the velocity as one vector field (vx, vy, vz)."""
    d = sum(float(np.linalg.norm(np.asarray(sol[k], np.float64) - np.asarray(ref[k], np.float64))) ** 2
            for k in SOL_KEYS[:3])
    r = sum(float(np.linalg.norm(np.asarray(ref[k], np.float64))) ** 2 for k in SOL_KEYS[:3])
    return float((d / r) ** 0.5) if r > 0 else float(d ** 0.5)


def errors_vs_fixture(sol, m, fx):
    """Relative L2 error per field and of the velocity vector on the
    fixture's sub-lattice (every stride-th node per axis), and of the
    full-field norms, against the oracle port's solution converged to 1e-10."""
    nx, ny, nz = m.shape
    st = int(fx["stride"])
    out = {}
    sub = {}
    for k in SOL_KEYS:
        sub[k] = np.asarray(sol[k], np.float64).reshape(nz, nx, ny)[::st, ::st, ::st].reshape(-1)
        out[k] = rel_l2(sub[k], fx["sub_" + k])
        out[k + "_norm"] = float(abs(np.linalg.norm(sol[k]) - float(fx["norm_" + k])) / float(fx["norm_" + k]))
    out["velocity"] = velocity_rel_l2(sub, {k: fx["sub_" + k] for k in SOL_KEYS})
    return out


def oracle_iters_to(hist, tol):
    h = np.asarray(hist)
    idx = np.nonzero(h <= tol)[0]
    return int(idx[0]) if idx.size else None


def cpu_sample(m, cfg, threads, iters=1):
    """Bounded run of the oracle port (kind "port": the same discretisation
    and algorithm in C + OpenMP) on the host cores: set-up (cell factors,
    coarsest LU) and `iters` outer iterations, timed; the solve estimate is
    set-up + (iterations to 1e-8) x (ms per iteration), the iteration count
    taken from the oracle's own converged run stored with the fixture.
    Returns (estimate_ms, detail dict)."""
    import ctypes as C
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    if not O.available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all"], check=True, stdout=subprocess.DEVNULL)
    fx = fixture(cfg)
    f = O.ronurecalc(m)
    nl = m.multinum + 1
    C.c_int.in_dll(O.lib(), "p2o_smoother").value = int(fx["oracle_smoother"]) if fx is not None else 2
    sweeps = [int(v) for v in fx["oracle_sweeps"]] if fx is not None else [4] * nl
    s = O.OracleSolver(m, npre=sweeps, npost=sweeps)
    t0 = time.perf_counter()
    s.set_fields(f)
    setup_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    h = s.solve(tol=0.0, max_cycles=iters, restart=16)
    it_ms = (time.perf_counter() - t0) * 1e3 / iters
    s.close()
    n_it = oracle_iters_to(fx["hist"], 1e-8) if fx is not None else None
    est = setup_ms + it_ms * n_it if n_it else None
    return est, {"setup_ms": setup_ms, "ms_per_iteration": it_ms, "iterations_timed": iters,
                 "iterations_to_1e-8": n_it, "residual_after": float(h[-1])}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local, dist = dist_setup(args.gpus)
    if args.config == 4:
        import torch
        torch.cuda.set_device(local)
        run_batch(args, rank, world, local, dist)
        return
    import torch
    import pardiso2_b200 as P
    from pardiso2_b200 import capi
    from pardiso2_b200 import model as M

    torch.cuda.set_device(local)
    m = M.config_model(args.config)
    n = m.nodenum
    big = n > 8_000_000
    prob = P.StokesProblem(m, device=local, precision=0, tol=1e-8, restart=args.restart, max_iter=args.max_iter,
                           smoother=args.smoother, sweep_growth=args.sweep_growth)
    if args.heat_only:
        heat = heat_leg(prob, m, args, False, synthetic=True)
        prob.close()
        if rank == 0:
            print(json.dumps({"metric": "ms per heat-equation step (titerate)", "value": heat["ms"], "unit": "ms",
                              "heat_only": True, "config": args.config, "heat": heat}), flush=True)
        return
    ronu_ms = [prob.ctx.upload_markers(m.markx, m.marky, m.markz, m.markt, m.rocks.n0, m.rocks.n1, m.rocks.ro)
               or prob.ctx.ronurecalc_resident() for _ in range(3)]
    # smoother and sweep schedule for this model, chosen once (outside the timed region)
    if args.tune_iters > 0:
        tune = prob.autotune(args.tune_iters)
    else:
        from pardiso2_b200.capi import TuneInfo
        tune = TuneInfo(smoother=args.smoother, sweep_growth=args.sweep_growth, est_ms=float("nan"),
                        rate=float("nan"), candidates=0, trial_iters=0, sweep_max=64, restart=args.restart,
                        sweeps0=4)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def one(p):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        info = p.ctx.solve_resident(check=False)
        return info

    for _ in range(args.warmup):
        one(prob)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    infos = [one(prob) for _ in range(args.steps)]
    torch.cuda.synchronize()
    clocks = clk.stop()
    if dist:
        dist.barrier()
    dev_ms = sum(i.ms_total for i in infos)
    launches = sum(i.kernels for i in infos)
    if dist:
        t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
    ms_per_step = dev_ms / args.steps
    value = dev_ms / (args.steps * world)   # ms per solve for the whole job

    # the dominant kernel: level-0 FP32 colour pass of the cell-block smoother
    H = capi.DebugHooks(prob.ctx)
    pass_ms = H.time_smoother(0, 40)
    bytes_per_launch = pass_bytes(n)
    achieved = bytes_per_launch / (pass_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic(n) if tune.smoother == 1 else None
    if args.solve_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "ms", "solve_only": True,
                              "config": args.config, "autotune": tune.as_dict(),
                              "iterations": infos[-1].iterations,
                              "gpu_launches": launches, "smoother_ms_per_pass": pass_ms,
                              "smoother_GBps": achieved}), flush=True)
        prob.close()
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    sol = prob.ctx.solution(n)

    # the plain FP64 solve (FP64 GCR, FP64 V-cycle) for comparison; fewer
    # steps on the large grids (each is about a second there)
    # the FP64 solve gets its own autotuned schedule (the same candidates),
    # so each precision runs its best configuration
    p64 = P.StokesProblem(m, device=local, precision=1, tol=1e-8, restart=args.restart, smoother=args.smoother,
                          sweep_growth=args.sweep_growth)
    p64.ctx.upload_markers(m.markx, m.marky, m.markz, m.markt, m.rocks.n0, m.rocks.n1, m.rocks.ro)
    p64.ctx.ronurecalc_resident()
    tune64 = p64.autotune(args.tune_iters) if args.tune_iters > 0 else tune
    k64 = min(args.steps, 3) if big else args.steps
    for _ in range(max(1, min(args.warmup, 1 if big else args.warmup))):
        one(p64)
    i64 = [one(p64) for _ in range(k64)]
    fp64_ms = sum(i.ms_total for i in i64) / k64
    sol64 = p64.ctx.solution(n)
    p64.close()
    err_vs_fp64 = {k: rel_l2(sol[k], sol64[k]) for k in SOL_KEYS}
    err_vs_fp64["velocity"] = velocity_rel_l2(sol, sol64)
    del sol64
    # against the oracle: its converged solution (fixture) on the large grids,
    # a live oracle solve to 1e-11 on the small ones
    err_vs_oracle = None
    fx = fixture(args.config)
    if fx is not None:
        err_vs_oracle = dict(errors_vs_fixture(sol, m, fx), reference="oracle port solution to 1e-10 (fixture "
                             "tests/golden/%s), sub-lattice every %d-th node per axis" % (FIXTURES[args.config],
                                                                                        int(fx["stride"])))
    elif rank == 0 and args.config <= 2 and not args.no_cpu_baseline:
        from oracle import oracle as O
        os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
        so = O.OracleSolver(m, npre=[4] * (m.multinum + 1), npost=[4] * (m.multinum + 1))
        so.set_fields(O.ronurecalc(m))
        so.solve(tol=1e-11, max_cycles=400, restart=16)
        ref = so.solution()
        so.close()
        err_vs_oracle = {k: rel_l2(sol[k], ref[k]) for k in SOL_KEYS}
        err_vs_oracle["velocity"] = velocity_rel_l2(sol, ref)
        err_vs_oracle["reference"] = "oracle port solved live to 1e-11, full fields"

    # one marker advection step (movemark, RK4) of the resident markers through
    # the resident solution of the last timed solve; CFL 0.5 on the finest cell
    vmax = max(float(np.abs(sol[k]).max()) for k in ("vx", "vy", "vz"))
    hmin = min(float(np.diff(g).min()) for g in (m.gx, m.gy, m.gz))
    dt_move = 0.5 * hmin / vmax
    del sol
    for _ in range(args.warmup):
        prob.ctx.movemark_resident(dt_move)
    move_ms = statistics.mean(prob.ctx.movemark_resident(dt_move) for _ in range(args.steps))
    nmark = int(m.markx.size)
    move_bytes = MOVEMARK_BYTES_PER_MARKER * nmark + MOVEMARK_BYTES_PER_NODE * n

    # end to end through the public C ABI with pinned host buffers
    keys = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
    host_nodes = prob.ctx.get_nodes(n)
    pinned = {k: torch.empty(n, dtype=torch.float32, pin_memory=True).numpy() for k in keys}
    for k in keys:
        pinned[k][:] = host_nodes[k]
    del host_nodes
    vx = torch.zeros(n, dtype=torch.float32, pin_memory=True).numpy()
    vy = torch.zeros(n, dtype=torch.float32, pin_memory=True).numpy()
    vz = torch.zeros(n, dtype=torch.float32, pin_memory=True).numpy()
    pr = torch.zeros(n, dtype=torch.float64, pin_memory=True).numpy()
    e2e = []
    ke2e = min(args.steps, 5) if big else args.steps
    for it in range(min(args.warmup, 2) + ke2e):
        vx[:] = 0; vy[:] = 0; vz[:] = 0; pr[:] = 0
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        prob.ctx.set_nodes(pinned)
        info = prob.ctx.stokes_solve(vx, vy, vz, pr)
        t1 = time.perf_counter()
        if it >= min(args.warmup, 2):
            e2e.append((t1 - t0) * 1e3)
    e2e_ms = statistics.mean(e2e)
    if dist:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item()) / world
    last = infos[-1]
    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 V-cycle / f64 outer GCR", "data": "synthetic",
        "config": config_dict(args.config, m, world),
        "solver": {"smoother": ("full" if tune.smoother else "diagonal") + " cell-block Vanka, autotuned",
                   "sweeps": "%d pre + %d post on level 0; 4 x %d^l on level l >= 1, at most %d"
                             % (tune.sweeps0, tune.sweeps0, tune.sweep_growth, tune.sweep_max),
                   "mixed": "FP64 GCR(%d) (true residual and update in FP64), FP32 V-cycle" % tune.restart,
                   "fp64": "FP64 GCR(%d), FP64 V-cycle, %s cell block, %d + %d sweeps on level 0, 4 x %d^l on level "
                           "l >= 1 at most %d (autotuned on its own)"
                           % (tune64.restart, "full" if tune64.smoother else "diagonal", tune64.sweeps0,
                              tune64.sweeps0, tune64.sweep_growth, tune64.sweep_max)},
        "converged": all(i.status == 0 for i in infos), "iterations": last.iterations,
        "rel_residual": last.rel_residual,
        "fp64_ms_per_solve": fp64_ms, "fp64_steps": k64, "iterations_fp64": i64[-1].iterations,
        "speedup_mixed_vs_fp64": fp64_ms / ms_per_step,
        "err_vs_fp64": err_vs_fp64, "err_vs_oracle": err_vs_oracle,
        "setup_ms": last.ms_setup, "vcycles_ms": last.ms_vcycles,
        "ronurecalc_ms": statistics.mean(ronu_ms[1:]),
        "unknowns_per_s": m.real_dofs() * world / (ms_per_step * 1e-3),
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": KERNEL_OF_SMOOTHER[tune.smoother] + " level-0 colour pass",
                     "bytes_per_launch": bytes_per_launch, "bytes_per_node": SWEEP_BYTES_PER_NODE // 2,
                     "ms_per_launch": pass_ms,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, burst)",
                     "timing": "each launch timed alone by CUDA events after a 256 MB L2 flush, mean of 40"},
        "clocks": clocks,
        "e2e": {"value": e2e_ms, "unit": "ms", "steps": ke2e,
                # node fields (6 float) and the initial guess (3 float + double pressure) up,
                # the solution (3 float + double pressure) down
                "h2d_bytes_per_step": 24 * n + 20 * n, "d2h_bytes_per_step": 20 * n},
    }
    line["movemark"] = {"ms": move_ms, "markers": nmark, "markmod": "RK4", "dt": dt_move,
                        "achieved_GBps": move_bytes / (move_ms * 1e-3) / 1e9, "bytes_per_step": move_bytes,
                        "launches": 2}
    line["heat"] = heat_leg(prob, m, args, rank == 0 and world == 1 and not args.no_cpu_baseline and args.config <= 2)
    line["autotune"] = tune.as_dict()
    line["autotune_fp64"] = tune64.as_dict()
    prob.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        if args.config <= 2:
            times, its = cpu_solve_ms(m, threads, steps=1)
            line["cpu_baseline"] = {"value": times[0], "unit": "ms", "cores": threads, "kind": "port",
                                    "sample": "one full solve of the workload to 1e-8 (oracle port, %d iterations)"
                                              % its[0]}
        else:
            est, det = cpu_sample(m, args.config, threads, iters=1)
            if est is not None:
                line["cpu_baseline"] = dict({"value": est, "unit": "ms", "cores": threads, "kind": "port",
                                             "sample": "oracle port set-up + 1 timed outer iteration of the "
                                                       "workload; value = set-up + iterations to 1e-8 (from the "
                                                       "oracle's own converged run) x ms per iteration"}, **det)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

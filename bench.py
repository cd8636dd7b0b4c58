#!/usr/bin/env python
"""Benchmark of the HigFlow per-time-step hot path on B200.

One JSON line on rank 0.  A step is one full HigFlow time step (viscoelastic cell
stage, explicit intermediate velocity, Poisson projection) of every case of the
workload.  The default workload is the batched configuration: 256 independent
2D Giesekus lid-driven cavities (side N log-uniform in [32, 256], seed 0) in one
batch program, mixed precision; the same batch is also timed in plain FP64 and
the mixed-vs-plain field error is reported.  With N GPUs every rank runs its own
batch of the same population drawn with seed = rank (independent instances; no
collective on the data path) and ``value`` is the cell-steps of all ranks over
the slowest rank's device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c4|c4_64|c1|cav2d_1024|cav3d_128]
  python bench.py --impl reference ...   # the reference's own CPU step
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "cell-steps/s and served solves/s + p99, mixed vs plain FP64 GPU at rel err 1e-6"
UNIT = "cell-steps/s"
L2_FLUSH_BYTES = 256 << 20

WORKLOADS = {
    "c4": dict(
        name="batched 2D Giesekus lid-driven cavities: 256 instances, side N log-uniform in [32,256] "
             "(seed 0), Wi uniform [0.1,2.0], alpha uniform [0,0.5], beta 0.1, Re 1, log-conformation "
             "kernel from identity, explicit Euler at 0.2x the explicit bound, CUBISTA, AMG-CG Poisson; "
             "programs recorded by HigTree (bit-exact stencils); one batch, one CUDA graph launch per step",
        batch="c4", precision="mixed", dim=2,
    ),
    "c4_64": dict(
        name="the first 64 cavities of the batched Giesekus population (seed 0), otherwise as c4; a smaller "
             "case of the same kernels for profiling",
        batch="c4", count=64, precision="mixed", dim=2,
    ),
    "c1": dict(
        name="2D Newtonian lid-driven cavity 64x64 (uniform quadtree, unit square), Re=100, lid u=1, "
             "explicit Euler dt=1e-4, CUBISTA, incremental projection, Poisson CG to 1e-10 relative residual, "
             "zero initial fields; program recorded by HigTree",
        dim=2, n=64, Re=100.0, dt=1e-4, precision="fp64",
    ),
    "c3_48": dict(
        name="3D Newtonian lid-driven cavity 48^3 (uniform octree, unit cube), Re=400, lid u=1, explicit "
             "Euler dt=1e-4, CUBISTA, incremental projection, AMG-CG Poisson, zero initial fields; program "
             "recorded by HigTree (the configured 128^3 needs about 3 hours of host stencil recording and "
             "24 GB of stencils, so this line runs the largest cube recorded in about a minute)",
        dim=3, n=48, Re=400.0, dt=1e-4, precision="mixed",
    ),
}


def shard(draws, rank, world):
    """This rank's instances of one population: greedy longest-processing-time
    partition by cost N^2 x steps (each instance to the least-loaded rank, the
    largest first); every instance lands on exactly one rank."""
    from higflow_b200 import workloads
    return [draws[i] for i in workloads.partition([d.cells * d.steps for d in draws], world)[rank]]


def load_program(wl, rank=0, world=1):
    from higflow_b200 import host, workloads
    if wl.get("batch") == "c4":
        draws = workloads.batched_giesekus()[:wl.get("count", 256)]
        return workloads.batch(shard(draws, rank, world))
    return host.record(host.cavity(wl["dim"], wl["n"], Re=wl["Re"], dt=wl["dt"]))


# ---------------------------------------------------------------------------
def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# compulsory bytes per launch of each phase, from the program being executed:
# every array the kernel must read or write, each element counted once.
def _row_bytes(prog, codes_list):
    """Header bytes (template, base, rhs) of the distinct general rows these slot
    codes use, plus their templates' entries, each counted once."""
    parts = [(-c[c < 0].astype(np.int64) - 1) for c in codes_list]
    r = np.unique(np.concatenate(parts)) if parts else np.zeros(0, np.int64)
    if r.size == 0:
        return 0
    tm = np.unique(prog.row_tmpl[r])
    nnz = int((prog.tmpl_ptr[tm + 1] - prog.tmpl_ptr[tm]).sum())
    return r.size * 16 + tm.size * 8 + nnz * 12


def cg_iter_bytes(sinfo, mixed):
    """Algorithmic bytes of one preconditioned CG iteration over every instance
    of the batch, each array a pass reads or writes counted once per pass, with
    the finest operator counted in the reference's CSR layout (4 B per row, 4 + w
    per non-zero) as the algorithmic-bytes convention does; the engine's row
    templates read 4 B per row instead, so its DRAM traffic is lower.  Passes:
    direction + q = A p and update on the FP64 finest operator, then the
    V-cycle (hf_pcg.cuh) in FP32 (mixed) or FP64, or the Jacobi z."""
    lv = sinfo["levels"]
    n0, nnz0 = lv[0][0], lv[0][1]
    b = n0 * (4 + 8 * 4) + nnz0 * 12          # dir: ptr, col+val, z, p_old -> p, q
    b += n0 * 8 * 6                            # update: p, q, r, x -> x, r
    if sinfo["method"] != "amg-cg":
        return b + n0 * 8 * 3                  # z = D^-1 r: r, dinv -> z
    s = 4 if mixed else 8
    nl = len(lv) - 1                           # concatenated levels; the last entry is the dense solves
    for l in range(nl - 1):
        n, na, npp, nr = lv[l]
        nn = lv[l + 1][0]
        b += n * 4 + na * (4 + s) + n * (s + (8 if l == 0 else s)) + n * s * 2      # down
        b += nn * 4 + nr * (4 + s) + n * s + nn * s                                 # restrict
        b += n * 4 + npp * (4 + s) + nn * s + n * s * 2                             # prolong
        if l > 0:
            b += n * 4 + na * (4 + s) + n * s * 4                                   # post
    crows, cdense = lv[-1][0], lv[-1][1]
    b += cdense * s + crows * s * 2                                                 # dense solves
    b += n0 * (8 + 4 + 2 * s + 8) + nnz0 * (4 + s)                                  # finest post -> z
    return b


def phase_bytes(prog, sinfo=None):
    D = prog.dim
    nf = sum(prog.nfacet[:D])
    nc = prog.ncell
    ve = prog.viscoelastic
    b = {}
    vel = sum(s.size for s in prog.vel_slots) * 4 + nf * (4 + 2 + 4)        # slots, flags, delta, instance
    vel += nf * 8 * 3 + nc * 8 * 2                                          # u (read), u* (write), FU; p, F
    if ve:
        vel += nc * 8 * D * D                                              # S
    vel += _row_bytes(prog, [s.ravel() for s in prog.vel_slots])
    b["velocity"] = vel
    if ve:
        cs = prog.cell_slots
        # slots, flags, delta, instance; u faces; Du, S, K read; Du, S, Knew written
        b["ve_cell"] = cs.size * 4 + nc * (4 + 2 + 4) + nf * 8 + nc * 8 * D * D * 6 + _row_bytes(prog, [cs.ravel()])
    b["final"] = sum(s[1:3].size for s in prog.vel_slots) * 4 + nf * (8 * 2 + 2 + 4) + nc * 8 * 3
    return b


# ---------------------------------------------------------------------------
def _barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _max_over_ranks(x, world, device):
    """max of x over the ranks (one scalar all-reduce; the only collective)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    on_gpu = dist.get_backend() == "nccl"
    t = torch.tensor([x], device=f"cuda:{device}" if on_gpu else "cpu", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed_steps(case, steps, device, world, flush, stream, profile=True):
    """K steps, each bracketed by CUDA events on the case stream (L2 flushed
    before each, outside the events); returns device ms summed over steps."""
    import torch
    if profile:
        case.profile(True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    _barrier(world)
    torch.cuda.synchronize(device)
    t_wall = time.perf_counter()
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            evs[k][0].record(stream)
        case.step(1, sync=False)       # one graph launch, queued behind the start event
        with torch.cuda.stream(stream):
            evs[k][1].record(stream)
        case.synchronize()             # outside the events: reads the phase events, checks the solve
    case.synchronize()
    torch.cuda.synchronize(device)
    t_wall = time.perf_counter() - t_wall
    _barrier(world)
    return sum(a.elapsed_time(b) for a, b in evs), t_wall


def fields_of(case, prog):
    from higflow_b200 import program as hp
    out = {f"u{d}": case.get(hp.FIELD_U, d) for d in range(prog.dim)}
    out["p"] = case.get(hp.FIELD_P)
    if prog.viscoelastic:
        for k in range(prog.dim ** 2):
            out[f"K{k}"] = case.get(hp.FIELD_KERNEL, k)
    return out


def run_b200(args, rank, world, device):
    import torch
    from higflow_b200 import engine
    from higflow_b200 import program as hp

    wl = WORKLOADS[args.workload]
    t0 = time.perf_counter()
    prog = load_program(wl, rank, world)
    t_program = time.perf_counter() - t0
    mixed = wl["precision"] == "mixed"
    prec = hp.PREC_MIXED if mixed else hp.PREC_FP64
    t0 = time.perf_counter()
    case = engine.Case(prog, engine.options(rtol=1e-10, atol=1e-300, device=device, precision=prec,
                                            eager=args.eager))
    t_create = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(case.stream(), device=device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")

    for _ in range(args.warmup):
        case.step(1)
    case.synchronize()
    st0 = case.stats()
    it0 = case.instance_iters()
    with ClockSampler(device) as clk:
        dev_ms, t_wall = timed_steps(case, args.steps, device, world, flush, stream)
    st = case.stats()
    dit = case.instance_iters() - it0
    launches = st.kernel_launches - st0.kernel_launches
    iters = st.total_iters - st0.total_iters
    phases = case.phase_times()
    case.profile(False)
    t_s = _max_over_ranks(dev_ms / 1e3, world, device)
    cells = prog.ncell
    value = cells * args.steps * world / t_s

    # roofline of the dominant phase (device time inside the timed region).
    # Per phase: compulsory bytes of all its launches in the timed steps; the
    # Poisson iterations weight each instance's rows by its own iteration count.
    sinfo = case.solver_info()
    pb = {p: v * phases[p][1] for p, v in phase_bytes(prog, sinfo).items() if p in phases}
    if sinfo["method"] in ("amg-cg", "jacobi-cg"):
        sizes = np.diff(prog.cell_off) if prog.ninst > 1 else np.array([prog.ncell])
        equiv_iters = float((dit * sizes).sum()) / float(sizes.sum())
        pb["poisson_iter"] = cg_iter_bytes(sinfo, mixed) * equiv_iters
    cand = [p for p in phases if phases[p][1] > 0 and p in pb]
    dom = max(cand, key=lambda p: phases[p][0])
    dom_ms, dom_launch = phases[dom]
    per_launch_s = dom_ms / 1e3 / dom_launch
    achieved = pb[dom] / (dom_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()
    traffic = None
    tfile = os.path.join(REPO, "profiles", f"traffic_{args.workload}.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get(dom)
        except Exception:
            traffic = None

    # mixed vs plain: the same batch from the same state, both forms, K steps
    extra = {}
    if mixed and not args.no_extras:
        state = {k: v.copy() for k, v in fields_of(case, prog).items()}
        m_case = case
        plain = engine.Case(prog, engine.options(rtol=1e-10, atol=1e-300, device=device, precision=hp.PREC_FP64))
        for key, arr in state.items():
            fid, comp = (hp.FIELD_U, int(key[1])) if key[0] == "u" else \
                (hp.FIELD_P, 0) if key == "p" else (hp.FIELD_KERNEL, int(key[1:]))
            plain.set(fid, comp, arr)
        # S and dp carry state too: copy them
        for k in range(prog.dim ** 2 if prog.viscoelastic else 0):
            plain.set(hp.FIELD_S, k, m_case.get(hp.FIELD_S, k))
        plain.set(hp.FIELD_DP, 0, m_case.get(hp.FIELD_DP, 0))
        pstream = torch.cuda.ExternalStream(plain.stream(), device=device)
        p_ms, _ = timed_steps(plain, args.steps, device, world, flush, pstream, profile=False)
        p_t = _max_over_ranks(p_ms / 1e3, world, device)
        plain_value = cells * args.steps * world / p_t
        m_case.step(args.steps)
        m_case.synchronize()
        a, b = fields_of(m_case, prog), fields_of(plain, prog)
        errs = {k: float(np.linalg.norm(a[k] - b[k]) / max(np.linalg.norm(b[k]), 1e-300)) for k in a}
        extra = {"plain_fp64": {"value": plain_value, "ms_per_step": p_ms / args.steps},
                 "mixed_over_plain": value / plain_value,
                 "mixed_vs_plain_rel_l2": max(errs.values()),
                 "mixed_vs_plain_rel_l2_by_field": errs}
        plain.close()

    # end to end through the C ABI with pinned host buffers, copies every step
    ninst = case.instances()
    e2e = None if args.no_extras else end_to_end(case, prog, args, world, device)
    case.close()
    if wl.get("batch") == "c4" and wl.get("count", 256) == 256 and not args.no_extras and not args.no_serve:
        extra["served"] = served(args, device)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if not mixed else "f32+f64",
        "data": "synthetic",
        "config": {"workload": wl["name"], "instances": ninst, "cells": cells,
                   "facets": sum(prog.nfacet[:prog.dim]),
                   "precision": "mixed (FP32 AMG V-cycle preconditioner; FP64 CG recurrences, finest operator, "
                                "gathers, eigen, time update)" if mixed else "plain FP64",
                   "poisson": f"{sinfo['method']}, rtol 1e-10 on ||b - A x|| per instance",
                   "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write, outside the step events)",
                   "parallelism": f"replicas x{world}",
                   "program": "recorded by the HigFlow host (HigTree's own stencils, ids and weights)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "bytes_per_launch": pb[dom] / dom_launch, "launch_us": per_launch_s * 1e6,
                     "peak_source": peak_kind},
        "phase_roofline": {p: {"GB/s": pb[p] / (phases[p][0] / 1e3) / 1e9, "launches": phases[p][1]}
                           for p in cand},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "poisson_iters_per_step": iters / args.steps,
        "phases_ms_per_step": {p: v[0] / args.steps for p, v in phases.items()},
        "setup_s": {"program": t_program, "create": t_create},
        "wall_s": t_wall,
        "clocks": clk.summary(),
    }
    line.update(extra)
    return line


def served(args, device):
    """The served stream on one device: the first 64 requests of the seeded
    stream (Poisson arrivals at 50/s, 2D cavities N in logU[64, 512]; 40 %
    Newtonian, 40 % Oldroyd-B, 20 % Giesekus), step counts scaled by 1/50,
    submitted at their arrival times to an hf_server (150 GB budget).  Programs
    are built before the clock starts (a request carries its program).
    Time to solution = submission to completion, queueing included."""
    from higflow_b200 import engine
    from higflow_b200 import program as hp
    from higflow_b200 import workloads
    reqs = workloads.served_requests()
    progs = [(workloads.program(c), c) for _, c in reqs]
    srv = engine.Server(budget_gb=150.0, max_active=64, chunk_steps=16, setup_threads=8, device=device)
    opts = engine.options(rtol=1e-10, atol=1e-300, device=device, precision=hp.PREC_MIXED)
    ids = []
    t0 = time.perf_counter()
    for (t_arr, _), (prog, c) in zip(reqs, progs):
        lag = t_arr - (time.perf_counter() - t0)
        if lag > 0:
            time.sleep(lag)
        ids.append(srv.submit(prog, opts, c.steps))
    tts, queue = [], []
    failed, failures = 0, {}
    for rid in ids:
        status, q, t = srv.wait(rid)
        if status != 0:
            failed += 1
            msg = engine._server_lib().hf_server_last_error().decode(errors="replace")
            failures.setdefault(str(status), msg)
        tts.append(t)
        queue.append(q)
        srv.release(rid)
    makespan = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    cells = sum(p.ncell * c.steps for p, c in progs)
    return {
        "requests": len(ids), "failed": int(failed), "failures": failures, "solves_per_s": len(ids) / makespan,
        "p50_s": float(np.percentile(tts, 50)), "p99_s": float(np.percentile(tts, 99)),
        "queue_p50_s": float(np.percentile(queue, 50)), "queue_p99_s": float(np.percentile(queue, 99)),
        "cell_steps_per_s": cells / makespan, "makespan_s": makespan, "arrival_window_s": reqs[-1][0],
        "cell_steps": int(st.cell_steps),
        "workload": "first 64 requests of the served stream (seed 0): Poisson arrivals 50/s, 2D lid-driven "
                    "cavities N log-uniform [64,512], 40% Newtonian Re 100, 40% Oldroyd-B Wi U[0.1,1.5], 20% "
                    "Giesekus (cavity geometry), steps U{500..5000} scaled by 1/50; mixed precision; HBM budget "
                    "150 GB; up to 64 cases stepping at once, 16 steps per dispatch",
    }


def end_to_end(case, prog, args, world, device):
    """The metric through the C ABI with pinned host buffers: every step copies
    the state fields host -> device, steps, and copies them back."""
    import ctypes as C
    import torch
    from higflow_b200 import engine
    from higflow_b200 import program as hp
    cells = prog.ncell
    pinned = {}
    names = [(hp.FIELD_U, d) for d in range(prog.dim)] + [(hp.FIELD_P, 0)]
    if prog.viscoelastic:
        names += [(hp.FIELD_KERNEL, k) for k in range(prog.dim ** 2)]
    for fid, comp in names:
        n = prog.field_size(fid, comp)
        pinned[(fid, comp)] = torch.empty(n, dtype=torch.float64, pin_memory=True)
        pinned[(fid, comp)].numpy()[:] = case.get(fid, comp)
    h2d = sum(v.numel() * 8 for v in pinned.values())
    L = engine.lib()
    _barrier(world)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for k in range(args.steps):
        for (fid, comp), buf in pinned.items():
            engine._check(L.hf_case_set_field(case.h, fid, comp, C.cast(buf.data_ptr(), C.POINTER(C.c_double)),
                                              buf.numel()))
        case.step(1)
        for (fid, comp), buf in pinned.items():
            engine._check(L.hf_case_get_field(case.h, fid, comp, C.cast(buf.data_ptr(), C.POINTER(C.c_double)),
                                              buf.numel()))
    t_e2e = _max_over_ranks(time.perf_counter() - t0, world, device)
    e2e = {"value": cells * args.steps * world / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d}
    return e2e


# ---------------------------------------------------------------------------
# the reference's own CPU step (oracle build of the reference)
def _ref_worker(args):
    """Run one reference case for `budget` seconds (at least 2 steps); returns
    (cells, steps, seconds)."""
    dim, n, par, budget, warm = args
    os.environ.setdefault("HF_ORACLE_RTOL", "1e-10")
    from oracle import refpy
    spec = refpy.cavity(dim, n, **par)
    c = refpy.RefCase(spec)
    c.step(warm)
    steps, el = 0, 0.0
    while el < budget or steps < 2:
        el += c.step(1)
        steps += 1
    cells = c.ncell
    c.close()
    return cells, steps, el


def reference_rate(wl, budget_s, warmup, procs=None):
    """cell-steps/s of the reference's higflow_solver_step[_viscoelastic] on the
    workload's cases, one single-threaded process per case and core."""
    from higflow_b200 import program as hp
    from higflow_b200 import workloads
    if wl.get("batch") == "c4":
        draws = workloads.batched_giesekus()
        nproc = procs or min(os.cpu_count() or 1, 16)
        jobs = [(2, d.n, dict(Re=d.Re, dt=d.dt, flowtype=hp.VISCOELASTIC, ve_model=hp.GIESEKUS, De=d.De,
                              alpha=d.alpha, beta=d.beta, kernel=hp.KERNEL_LOG), budget_s, warmup)
                for d in draws[:nproc]]
        desc = (f"the first {nproc} cases of the batch (N = {[d.n for d in draws[:nproc]]}), one process each, "
                f"~{budget_s:.0f} s of reference steps per process after {warmup} warm-up steps")
    else:
        nproc = 1
        jobs = [(wl["dim"], wl["n"], dict(Re=wl["Re"], dt=wl["dt"]), budget_s, warmup)]
        desc = f"~{budget_s:.0f} s of reference steps of the same case after {warmup} warm-up steps, one process"
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(jobs)) as pool:
        res = pool.map(_ref_worker, jobs)
    rate = sum(c * s / e for c, s, e in res)
    return rate, len(jobs), desc


def cpu_baseline(wl, budget_s=15.0):
    try:
        from oracle import refpy
        if not refpy.available(wl["dim"]):
            return None
        rate, cores, desc = reference_rate(wl, budget_s, 1)
        return {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": desc + "; reference HigFlow built from its sources (oracle build, single-rank shims)"}
    except Exception as e:  # pragma: no cover
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}


def run_reference(args):
    wl = WORKLOADS[args.workload]
    from oracle import refpy
    if not refpy.available(wl["dim"]):
        print(json.dumps({"impl": "reference", "unavailable": "oracle build of the reference not present"}))
        return
    budget = max(5.0, min(60.0, 0.5 * args.steps))
    rate, cores, desc = reference_rate(wl, budget, args.warmup)
    cb = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["name"]},
        "cpu_baseline": cb, "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c4", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU reference sample")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream run")
    ap.add_argument("--eager", action="store_true",
                    help="launch kernels one by one instead of one CUDA graph per step (kernel profilers)")
    ap.add_argument("--no-extras", action="store_true",
                    help="warm-up and timed steps only (no plain-FP64 comparison, no end-to-end pass); for profiling")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    line = run_b200(args, rank, world, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(WORKLOADS[args.workload])
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

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
    "c4_16": dict(
        name="the first 16 cavities of the batched Giesekus population (seed 0), otherwise as c4; the small case "
             "the kernel profiles are taken on",
        batch="c4", count=16, precision="mixed", dim=2,
    ),
    "c4_16_plain": dict(
        name="the first 16 cavities of the batched Giesekus population (seed 0), otherwise as c4, plain FP64; the "
             "small case the plain form's kernel profiles are taken on",
        batch="c4", count=16, precision="fp64", dim=2,
    ),
    "c1": dict(
        name="2D Newtonian lid-driven cavity 64x64 (uniform quadtree, unit square), Re=100, lid u=1, "
             "explicit Euler dt=1e-4, CUBISTA, incremental projection, Poisson CG to 1e-10 relative residual, "
             "zero initial fields; program recorded by HigTree",
        dim=2, n=64, Re=100.0, dt=1e-4, precision="fp64",
    ),
    "c2": dict(
        name="2D Oldroyd-B 4:1 planar contraction (two trees [-16,0]x[-4,4] and [0,16]x[-1,1] at 32 cells per "
             "unit length, second level on squares of side 1/4 at the contraction corners; 164,128 cells), "
             "Re=0.01, Wi=1.0, beta=1/9, log-conformation from the identity, parabolic inflow of mean 1, dt=5e-5, "
             "semi-implicit Euler velocity (explicit Euler diverges at this dt: dt > Re h^2/4), BiCGStab Poisson "
             "(the refined rows are not symmetric); plain FP64; program recorded by HigTree",
        contraction=32, dim=2, precision="fp64",
    ),
    "c3_32": dict(
        name="3D Newtonian lid-driven cavity 32^3 (uniform octree, unit cube), Re=400, lid u=1, explicit "
             "Euler dt=1e-4, CUBISTA, incremental projection, AMG-CG Poisson, zero initial fields; program "
             "recorded by HigTree in one process (about 3 minutes: 3D rows reach 120 entries, about 950 per cell; "
             "the configured 128^3 would take about 3 hours of recording and 24 GB of stencils)",
        dim=3, n=32, Re=400.0, dt=1e-4, precision="mixed",
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
        # each rank records its own shard, with its share of the host's cores
        return workloads.batch(shard(draws, rank, world), procs=max(1, (os.cpu_count() or 1) // world))
    if wl.get("contraction"):
        return host.record(workloads.contraction_c2(wl["contraction"]))
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
# algorithmic bytes per step of each phase (higflow_b200/roofline.py: the
# reference's kernels' field arrays plus the stencil bytes of their distinct
# queries; the Poisson iterations at the measured count)
def phase_bytes(prog, mixed, iters_per_step, sweeps_per_step):
    from higflow_b200 import roofline
    sb = roofline.step_bytes(prog, mixed)
    nc = prog.ncell
    spmv64 = 4 * (nc + 1) + prog.p_col.size * 12 + 2 * 8 * nc
    w = 4 if mixed else 8
    out = {"velocity": sb["velocity"]["F"] + sb["velocity"]["S"],
           # the velocity stage's rows alone (k_vrows): their stencil bytes
           "velocity_rows": 4 * sb["velocity"]["rows"] + sb["velocity"]["row_entries"] * (4 + w),
           "poisson_init": sb["divergence"]["F"] + sb["divergence"]["S"] + spmv64,
           "poisson_iter": iters_per_step * roofline.poisson_iter_bytes(prog, 4 if mixed else 8)
           + sweeps_per_step * spmv64,
           "final": sb["final"]["F"] + sb["final"]["S"]}
    if "ve_cell" in sb:
        out["ve_cell"] = sb["ve_cell"]["F"] + sb["ve_cell"]["S"]
        # k_ve_cell alone: the stage without the polymeric tensor (k_ve_stress
        # reads the new K and writes S: 8 D^2 x 3 bytes per cell)
        out["ve_cell_main"] = out["ve_cell"] - 8 * prog.dim ** 2 * nc * 3
    return out, sb


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


def _set_state(case, state, prog):
    """Copy a state (fields_of + S + dp) into a case."""
    from higflow_b200 import program as hp
    for key, arr in state.items():
        if key.startswith("u"):
            case.set(hp.FIELD_U, int(key[1:]), arr)
        elif key == "p":
            case.set(hp.FIELD_P, 0, arr)
        elif key == "dp":
            case.set(hp.FIELD_DP, 0, arr)
        elif key.startswith("K"):
            case.set(hp.FIELD_KERNEL, int(key[1:]), arr)
        elif key.startswith("S"):
            case.set(hp.FIELD_S, int(key[1:]), arr)


def full_state(case, prog):
    from higflow_b200 import program as hp
    st = fields_of(case, prog)
    st["dp"] = case.get(hp.FIELD_DP, 0)
    if prog.viscoelastic:
        for k in range(prog.dim ** 2):
            st[f"S{k}"] = case.get(hp.FIELD_S, k)
    return st


def rel_errors(a, b):
    return {k: float(np.linalg.norm(a[k] - b[k]) / max(np.linalg.norm(b[k]), 1e-300)) for k in b}


# the loosest Poisson tolerances tried by the equal-error protocol, loosest first
PROTOCOL_RTOLS = (1e-5, 1e-6, 1e-7, 1e-8, 1e-9, 1e-10)
PROTOCOL_TARGET = 1e-6


def protocol_subset(draws, count=16):
    """Instances at the population's side quantiles (the subset the equal-error
    protocol runs for the configuration's full step count)."""
    order = sorted(range(len(draws)), key=lambda i: (draws[i].n, i))
    pick = sorted({order[int(round(q * (len(order) - 1)))] for q in np.linspace(0.0, 1.0, count)})
    return [draws[i] for i in pick]


def equal_error_protocol(draws, steps, device):
    """Both forms at the loosest Poisson tolerance whose fields stay within
    PROTOCOL_TARGET relative L2 (per field: u, p, K) of the FP64 oracle after
    the configuration's steps, on a size-stratified subset of the population.
    The oracle is the plain FP64 form at rtol 1e-12 (itself pinned to the
    reference at 1e-10 by the GPU parity tests)."""
    from higflow_b200 import engine, workloads
    from higflow_b200 import program as hp
    sub = protocol_subset(draws)
    prog = workloads.batch(sub)

    def run(prec, rtol):
        case = engine.Case(prog, engine.options(rtol=rtol, atol=1e-300, device=device, precision=prec))
        t0 = time.perf_counter()
        case.step(steps)
        el = time.perf_counter() - t0
        out = fields_of(case, prog)
        it = case.stats().total_iters
        case.close()
        return out, el, it

    oracle, _, _ = run(hp.PREC_FP64, 1e-12)
    result = {"subset": [d.n for d in sub], "steps": steps, "target": PROTOCOL_TARGET,
              "oracle": "plain FP64 on the GPU at Poisson rtol 1e-12", "tried": {}}
    for name, prec in (("plain", hp.PREC_FP64), ("mixed", hp.PREC_MIXED)):
        chosen = None
        tried = []
        for rtol in PROTOCOL_RTOLS:
            f, el, it = run(prec, rtol)
            err = rel_errors(f, oracle)
            ok = max(err.values()) <= PROTOCOL_TARGET
            tried.append({"rtol": rtol, "max_rel_l2": max(err.values()), "ok": ok, "seconds": el,
                          "iters_per_instance_step": it / steps / len(sub)})
            if ok:
                chosen = {"rtol": rtol, "rel_l2_by_field": err}
                break
        result["tried"][name] = tried
        result[name] = chosen
    return result


def plain_one_case_at_a_time(draws, rtol, device, steps=10, count=16):
    """The plain FP64 path as a HigFlow case runs it through the drop-in: one
    case per engine case, stepped alone (one CUDA graph launch per step).
    ``count`` instances at the population's side quantiles are timed (CUDA
    events around ``steps`` steps after warm-up); the population's time per
    step is the sum over its instances of the sample's time per step
    interpolated in N^2 (log-log).  Returns cell-steps/s of the whole
    population and the sample."""
    import torch
    from higflow_b200 import engine, workloads
    from higflow_b200 import program as hp
    sub = protocol_subset(draws, count)
    progs = workloads.programs(sub)
    ms = []
    for prog in progs:
        case = engine.Case(prog, engine.options(rtol=rtol, atol=1e-300, device=device, precision=hp.PREC_FP64))
        stream = torch.cuda.ExternalStream(case.stream(), device=device)
        case.step(3)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
        case.step(steps, sync=False)
        with torch.cuda.stream(stream):
            b.record(stream)
        case.synchronize()
        torch.cuda.synchronize(device)
        ms.append(a.elapsed_time(b) / steps)
        case.close()
    x = np.log([d.cells for d in sub])
    y = np.log(ms)
    order = np.argsort(x)
    per = np.exp(np.interp(np.log([d.cells for d in draws]), x[order], y[order]))
    total_ms = float(per.sum())
    cells = sum(d.cells for d in draws)
    return {"value": cells / (total_ms / 1e3), "ms_per_population_step": total_ms,
            "sample": {"N": [d.n for d in sub], "ms_per_step": ms}, "rtol": rtol,
            "method": f"{len(sub)} instances at the population's side quantiles stepped alone ({steps} steps each "
                      "after 3 warm-up, CUDA events), the population's step time the sum of the sample's per-step "
                      "times interpolated in cells (log-log) over its 256 instances"}


def time_form(prog, prec, rtol, state, args, world, device, flush, profile=True):
    """Create a case in one precision form, load the state, warm up, time
    args.steps steps; returns (case, device ms, wall s, stats deltas)."""
    import torch
    from higflow_b200 import engine
    case = engine.Case(prog, engine.options(rtol=rtol, atol=1e-300, device=device, precision=prec,
                                            eager=args.eager))
    if state is not None:
        _set_state(case, state, prog)
    stream = torch.cuda.ExternalStream(case.stream(), device=device)
    for _ in range(args.warmup):
        case.step(1)
    case.synchronize()
    case.start_state = full_state(case, prog)   # the timed region's first state (the e2e pass restarts from it)
    st0 = case.stats()
    it0 = case.instance_iters()
    with ClockSampler(device) as clk:
        dev_ms, t_wall = timed_steps(case, args.steps, device, world, flush, stream, profile=profile)
    st = case.stats()
    return case, dev_ms, t_wall, st0, st, case.instance_iters() - it0, clk.summary()


def whole_configuration(prog, rtol, steps, world, device):
    """Time to solution of the whole configuration, both forms: every
    instance's full step count from rest (fields at rest, conformation at the
    identity), device time with CUDA events around all the steps, the max over
    ranks.  The headline value times steps from rest at the start of the run,
    where the Poisson solves take the most iterations; this is the run's
    average."""
    import torch
    from higflow_b200 import engine
    from higflow_b200 import program as hp
    out = {"steps": steps}
    sizes = np.diff(prog.cell_off) if prog.ninst > 1 else np.array([prog.ncell])
    for form, prec in (("mixed", hp.PREC_MIXED), ("plain", hp.PREC_FP64)):
        case = engine.Case(prog, engine.options(rtol=rtol[form], atol=1e-300, device=device, precision=prec))
        stream = torch.cuda.ExternalStream(case.stream(), device=device)
        case.step(1)            # graph capture and launch-shape tuning (the first of the steps)
        case.synchronize()
        it0 = case.instance_iters()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _barrier(world)
        a.record(stream)
        case.step(steps - 1, sync=False)
        b.record(stream)
        b.synchronize()
        case.synchronize()
        ms = a.elapsed_time(b)
        dit = case.instance_iters() - it0
        case.close()
        t = _max_over_ranks(ms / 1e3, world, device)
        out[form] = {"seconds": t, "cell_steps_per_s": prog.ncell * (steps - 1) * world / t, "rtol": rtol[form],
                     "poisson_iters_per_instance_step": float((dit * sizes).sum()) / float(sizes.sum()) / (steps - 1)}
    out["mixed_over_plain"] = out["mixed"]["cell_steps_per_s"] / out["plain"]["cell_steps_per_s"]
    out["method"] = (f"steps 2..{steps} of the configuration from rest timed on the device as one region (the first "
                     "step captures the graph and tunes launch shapes), each form at its equal-error tolerance")
    return out


def host_info():
    cpu = ""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    cpu = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu": cpu}


def run_b200(args, rank, world, device):
    import torch
    from higflow_b200 import engine, roofline, workloads
    from higflow_b200 import program as hp

    wl = WORKLOADS[args.workload]
    t0 = time.perf_counter()
    prog = load_program(wl, rank, world)
    t_program = time.perf_counter() - t0
    mixed = wl["precision"] == "mixed"
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")
    cells = prog.ncell

    # the equal-error protocol: each form's loosest Poisson tolerance at the
    # configuration's own step count (batched workloads)
    protocol = None
    rtol = {"plain": 1e-10, "mixed": 1e-10}
    if wl.get("batch") == "c4" and not args.no_extras and not args.no_protocol:
        draws = workloads.batched_giesekus()[:wl.get("count", 256)]
        protocol = equal_error_protocol(draws, draws[0].steps, device)
        for k in ("plain", "mixed"):
            if protocol.get(k):
                rtol[k] = protocol[k]["rtol"]

    form = "mixed" if mixed else "plain"
    prec = hp.PREC_MIXED if mixed else hp.PREC_FP64
    t0 = time.perf_counter()
    case, dev_ms, t_wall, st0, st, dit, clocks = time_form(prog, prec, rtol[form], None, args, world, device, flush)
    t_create = time.perf_counter() - t0
    launches = st.kernel_launches - st0.kernel_launches
    iters = st.total_iters - st0.total_iters
    phases = case.phase_times()
    shapes = dict(zip(("k_vrows", "k_velocity", "k_ve_cell"), case.launch_shapes()))
    case.profile(False)
    t_s = _max_over_ranks(dev_ms / 1e3, world, device)
    value = cells * args.steps * world / t_s
    ms_step = dev_ms / args.steps

    # rooflines: per phase (algorithmic bytes per step / phase time per step)
    # and the whole step; Poisson iterations weighted by instance size
    sizes = np.diff(prog.cell_off) if prog.ninst > 1 else np.array([prog.ncell])
    it_step = float((dit * sizes).sum()) / float(sizes.sum()) / args.steps
    sweeps = float(st.last_outer) if mixed else 0.0
    pb, sb = phase_bytes(prog, mixed, it_step, sweeps)
    peak, peak_kind = _peaks()
    phase_rl = {}
    for p, (ms, nl) in phases.items():
        if p in pb and ms > 0:
            phase_rl[p] = {"bytes_per_step": pb[p], "ms_per_step": ms / args.steps, "launches_per_step": nl / args.steps,
                           "GB/s": pb[p] / (ms / args.steps / 1e3) / 1e9,
                           "frac": pb[p] / (ms / args.steps / 1e3) / 1e9 / peak}
    # the roofline kernel: the longest of the step's single kernels (k_vrows,
    # k_velocity = the velocity phase without its rows) and the viscoelastic
    # cell stage (k_ve_cell with its row pairs and k_ve_stress); the Poisson
    # loop (a dozen kernels per iteration) and every phase are beside it
    cands = {}
    if "velocity_rows" in phase_rl:
        cands["velocity_rows"] = ("k_vrows (the velocity stage's stencil rows)", phase_rl["velocity_rows"])
        if "velocity" in phase_rl:
            v, r = phase_rl["velocity"], phase_rl["velocity_rows"]
            ms, by = v["ms_per_step"] - r["ms_per_step"], v["bytes_per_step"] - r["bytes_per_step"]
            if ms > 0:
                cands["velocity_kernel"] = ("k_velocity (the facet kernel)", {
                    "bytes_per_step": by, "ms_per_step": ms, "launches_per_step": 1.0,
                    "GB/s": by / (ms / 1e3) / 1e9, "frac": by / (ms / 1e3) / 1e9 / peak})
    if "ve_cell_main" in phase_rl:
        cands["ve_cell_main"] = ("k_ve_cell (the viscoelastic cell stage's main kernel)", phase_rl["ve_cell_main"])
    elif "ve_cell" in phase_rl:
        cands["ve_cell"] = ("viscoelastic cell stage (k_ve_cell with its row pairs, k_ve_stress)", phase_rl["ve_cell"])
    if not cands:
        cands = {p: (f"{p} phase", v) for p, v in phase_rl.items()}
    dom = max(cands, key=lambda p: cands[p][1]["ms_per_step"])
    dom_name, d = cands[dom]
    traffic = None
    tfile = os.path.join(REPO, "profiles", f"traffic_{args.workload}{'' if mixed else '_plain'}.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get(dom)
        except Exception:
            traffic = None
    ws = roofline.whole_step(prog, mixed, it_step, sweeps)
    whole = {"bytes_per_step": ws["bytes"], "bytes_per_cell_step": ws["bytes"] / cells,
             "GB/s": ws["bytes"] / (ms_step / 1e3) / 1e9, "frac": ws["bytes"] / (ms_step / 1e3) / 1e9 / peak,
             "by_kernel": ws["parts"], "poisson_iter_bytes": ws["poisson"],
             "queries": {k: {q: v[q] for q in ("queries", "centre_hits", "rows", "row_entries")} for k, v in sb.items()}}

    extra = {}
    e2e = None
    state = full_state(case, prog)
    if not args.no_extras:
        e2e = end_to_end(case, prog, args, world, device, case.start_state)
    case.close()
    if mixed and not args.no_extras:
        # the plain FP64 form on the same batch and state, at its own
        # equal-error tolerance
        pcase, p_ms, _, pst0, pst, pdit, pclk = time_form(prog, hp.PREC_FP64, rtol["plain"], state, args, world,
                                                          device, flush, profile=True)
        p_phases = pcase.phase_times()
        pcase.profile(False)
        pcase.close()
        p_t = _max_over_ranks(p_ms / 1e3, world, device)
        plain_value = cells * args.steps * world / p_t
        p_it = float((pdit * sizes).sum()) / float(sizes.sum()) / args.steps
        pws = roofline.whole_step(prog, False, p_it, 0.0)
        extra = {"plain_fp64": {"value": plain_value, "ms_per_step": p_ms / args.steps, "rtol": rtol["plain"],
                                "poisson_iters_per_step": p_it,
                                "phases_ms_per_step": {p: v[0] / args.steps for p, v in p_phases.items()},
                                "whole_step": {"bytes_per_step": pws["bytes"],
                                               "GB/s": pws["bytes"] / (p_ms / args.steps / 1e3) / 1e9,
                                               "frac": pws["bytes"] / (p_ms / args.steps / 1e3) / 1e9 / peak},
                                "clocks": pclk},
                 "mixed_over_plain": value / plain_value}
    if mixed and wl.get("batch") == "c4" and not args.no_extras:
        extra["whole_configuration"] = whole_configuration(prog, rtol, workloads.batched_giesekus()[0].steps, world,
                                                           device)
    if mixed and wl.get("batch") == "c4" and wl.get("count", 256) == 256 and not args.no_extras and world == 1:
        draws = workloads.batched_giesekus()
        one = plain_one_case_at_a_time(draws, rtol["plain"], device)
        one["mixed_batched_over_it"] = value / one["value"]
        extra["plain_fp64_one_case_at_a_time"] = one
    if protocol is not None:
        extra["equal_error_protocol"] = protocol
        if protocol.get("mixed"):
            extra["rel_l2_vs_oracle_by_field"] = {"mixed": protocol["mixed"]["rel_l2_by_field"],
                                                  "plain": (protocol.get("plain") or {}).get("rel_l2_by_field")}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "strong" if wl.get("batch") else "weak", "vs_baseline": None,
        "dtype": "f64" if not mixed else "f32+f64",
        "data": "synthetic",
        "config": {"workload": wl["name"], "instances": prog.ninst or 1, "cells": cells,
                   "facets": sum(prog.nfacet[:prog.dim]),
                   "precision": ("mixed: FP32 stencil weights in the velocity rows (FP64 values and sums; rows "
                                 "sharing one FP32 pattern read it once), FP32 CUBISTA, FP32 AMG-CG sweeps inside "
                                 "FP64 iterative refinement; FP64 eigensystem, kernel transform and time updates")
                                if mixed else "plain FP64",
                   "poisson": f"AMG-CG, rtol {rtol[form]:g} on ||b - A x|| per instance" +
                              (" (loosest meeting 1e-6 relative L2 against the FP64 oracle after the configuration's "
                               "steps)" if protocol else ""),
                   "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write, outside the step events)",
                   "parallelism": f"instances partitioned by cost over {world} GPU(s)" if wl.get("batch") else
                                  f"replicas x{world}",
                   "program": "recorded by the HigFlow host (HigTree's own stencils, ids and weights)"},
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": d["GB/s"], "peak": peak, "unit": "GB/s",
                     "frac": d["frac"], "traffic": traffic,
                     "bytes_per_launch": d["bytes_per_step"] / max(d["launches_per_step"], 1e-9),
                     "launch_us": d["ms_per_step"] * 1e3 / max(d["launches_per_step"], 1e-9),
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind},
        "whole_step_roofline": whole,
        "phase_roofline": phase_rl,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "poisson_iters_per_step": iters / args.steps,
        "poisson_iters_per_instance_step": it_step,
        "refinement_sweeps_last_step": st.last_outer,
        "phases_ms_per_step": {p: v[0] / args.steps for p, v in phases.items()},
        "tuned_block_sizes": shapes,
        "setup_s": {"program": t_program, "create_and_time": t_create},
        "wall_s": t_wall,
        "clocks": clocks,
        "host": host_info(),
    }
    line.update(extra)
    # the served stream and the one-case-at-a-time comparison are one-device
    # measurements: they run at N = 1 only
    if (wl.get("batch") == "c4" and wl.get("count", 256) == 256 and not args.no_extras and not args.no_serve
            and world == 1):
        try:
            line["served"] = served(args, device, rtol["mixed"])
            line["served"]["over_batched"] = line["served"]["cell_steps_per_s"] / value
        except Exception as e:  # the headline stands; the served run reports its failure
            line["served"] = {"error": f"{type(e).__name__}: {e}"}
    return line


def served(args, device, rtol):
    """The served stream on one device: the first args.serve_requests requests
    of the seeded stream (Poisson arrivals at 50/s; 40 % Newtonian cavities,
    40 % Oldroyd-B cavities, 20 % Giesekus channels; N log-uniform in
    [64, 512]; full step counts U{500..5000}), submitted at their arrival times
    to a continuous-batching server (higflow_b200/serve.py: cohorts of waiting
    requests stepped as one batch, each request frozen at its own step count,
    several cohorts at once, 150 GB HBM budget), mixed precision at the
    equal-error tolerance.  Programs are recorded before the clock starts (a
    request carries its program).  Time to solution = submission to
    completion, queueing included."""
    from higflow_b200 import engine, serve, workloads
    from higflow_b200 import program as hp
    reqs = workloads.served_requests(count=args.serve_requests)
    t0 = time.perf_counter()
    progs = workloads.programs([c for _, c in reqs])
    t_record = time.perf_counter() - t0
    opts = engine.options(rtol=rtol, atol=1e-300, device=device, precision=hp.PREC_MIXED)
    srv = serve.BatchServer(device=device, budget_gb=150.0, max_cohorts=8, chunk=32, opts=opts)
    ids = []
    t0 = time.perf_counter()
    for (t_arr, _), prog, (_, c) in zip(reqs, progs, reqs):
        lag = t_arr - (time.perf_counter() - t0)
        if lag > 0:
            time.sleep(lag)
        ids.append(srv.submit(prog, c.steps))
    tts, queue, failed, why, ok = [], [], 0, {}, []
    for rid, (_, c) in zip(ids, reqs):
        status, q, t = srv.wait(rid)
        ok.append(status == 0)
        if status != 0:
            failed += 1
            kind = "newtonian cavity" if c.model < 0 else f"{'oldroyd-b' if c.model == hp.OLDROYD_B else 'giesekus'} " \
                f"{c.geometry}"
            why.setdefault(kind, []).append({"n": c.n, "steps": c.steps, "Wi": round(c.De, 3), "status": int(status),
                                             "error": srv.error(rid)[:160]})
        tts.append(t)
        queue.append(q)
        srv.release(rid)
    makespan = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    cells = sum(p.ncell * c.steps for p, (_, c), good in zip(progs, reqs, ok) if good)
    kinds = {"newtonian cavity": sum(c.model < 0 for _, c in reqs),
             "oldroyd-b cavity": sum(c.model == hp.OLDROYD_B for _, c in reqs),
             "giesekus channel": sum(c.geometry == "channel" for _, c in reqs)}
    return {
        "requests": len(ids), "failed": int(failed), "failures": why, "solves_per_s": sum(ok) / makespan,
        "p50_s": float(np.percentile(tts, 50)), "p99_s": float(np.percentile(tts, 99)),
        "queue_p50_s": float(np.percentile(queue, 50)), "queue_p99_s": float(np.percentile(queue, 99)),
        "cell_steps_per_s": cells / makespan, "makespan_s": makespan, "arrival_window_s": reqs[-1][0],
        "cell_steps": int(cells), "cohorts": st["cohorts"], "kinds": kinds, "record_s": t_record,
        "poisson_rtol": rtol,
        "workload": f"first {len(ids)} requests of the served stream (seed 0): Poisson arrivals 50/s, 2D, N "
                    "log-uniform [64,512], 40% Newtonian cavities Re 100, 40% Oldroyd-B cavities Wi U[0.1,1.5], "
                    "20% Giesekus channels (8x2, 2N x N/2 cells), full step counts U{500..5000}; recorded programs; "
                    "mixed precision; continuous batching (cohorts, per-request step limits), HBM budget 150 GB",
    }


def end_to_end(case, prog, args, world, device, start=None):
    """The metric through the C ABI with pinned host buffers, two ways.

    value: the drop-in's call pattern (higflow_b200/binding/hf_attach.c: the
    fields stay on the device between the host's output points, as HigFlow's
    main loop reads them only to print or save).  Every step copies each
    instance's time step host -> device (hf_case_set_timestep uploads the
    instances' parameters, as the host sets ns->par.dt; not for the
    semi-implicit forms, whose dt is fixed), steps, and reads the step's
    result back (hf_case_stats:
    the Poisson iterations and residual that hf_step hands to the solver
    parameters); the host's output point (hf_sync_to_host: u, p and the
    kernel tensor, device -> host) comes once per timed region, i.e. every
    args.steps steps.

    full_state_every_step: every step copies the state fields host -> device,
    steps, and copies them back (a host that edits the fields between steps).

    Both passes start from `start`, the first state of the device-timed region
    (the same steps are timed; loading a state restarts the pressure's
    initial-guess history, which costs the first steps some iterations)."""
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
        pinned[(fid, comp)] = torch.empty(prog.field_size(fid, comp), dtype=torch.float64, pin_memory=True)
    fields = sum(v.numel() * 8 for v in pinned.values())
    ninst = case.instances()
    dts = torch.empty(ninst, dtype=torch.float64, pin_memory=True)
    dts.numpy()[:] = [p["dt"] for p in prog.inst_par] if prog.inst_par else [prog.par["dt"]]
    L = engine.lib()
    st = hp.HFStats()

    def put(fid, comp, buf):
        engine._check(L.hf_case_set_field(case.h, fid, comp, C.cast(buf.data_ptr(), C.POINTER(C.c_double)),
                                          buf.numel()))

    def get(fid, comp, buf):
        engine._check(L.hf_case_get_field(case.h, fid, comp, C.cast(buf.data_ptr(), C.POINTER(C.c_double)),
                                          buf.numel()))

    # the drop-in's pattern
    if start is not None:
        _set_state(case, start, prog)
    _barrier(world)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for k in range(args.steps):
        engine._check(L.hf_case_set_timestep(case.h, C.cast(dts.data_ptr(), C.POINTER(C.c_double)), ninst))
        engine._check(L.hf_case_step(case.h, 1))
        engine._check(L.hf_case_stats(case.h, C.byref(st)))
    for (fid, comp), buf in pinned.items():
        get(fid, comp, buf)
    t_plugin = _max_over_ranks(time.perf_counter() - t0, world, device)
    # the whole state both ways every step, from the same first state
    if start is not None:
        _set_state(case, start, prog)
    for (fid, comp), buf in pinned.items():
        buf.numpy()[:] = case.get(fid, comp)
    _barrier(world)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for k in range(args.steps):
        for (fid, comp), buf in pinned.items():
            put(fid, comp, buf)
        case.step(1)
        for (fid, comp), buf in pinned.items():
            get(fid, comp, buf)
    t_full = _max_over_ranks(time.perf_counter() - t0, world, device)
    stats_bytes = C.sizeof(hp.HFStats) + 80 * ninst   # the stats struct and the instance scalars it reads
    sie = int(prog.par.get("tempdiscrtype", 0)) in (hp.SEMI_IMPLICIT_EULER, hp.SEMI_IMPLICIT_CN, hp.SEMI_IMPLICIT_BDF2)
    return {"value": cells * args.steps * world / t_plugin, "unit": UNIT,
            "h2d_bytes_per_step": 0 if sie else C.sizeof(hp.HFParams) * ninst,
            "d2h_bytes_per_step": stats_bytes + fields // args.steps,
            "pattern": f"drop-in: per step the time steps in, one step, the step's solver result out; u, p and the "
                       f"kernel tensor out once per {args.steps} steps (the host's output point)",
            "full_state_every_step": {"value": cells * args.steps * world / t_full, "unit": UNIT,
                                      "h2d_bytes_per_step": fields, "d2h_bytes_per_step": fields}}


# ---------------------------------------------------------------------------
# the reference's own CPU step (oracle build of the reference)
def _ref_worker(args):
    """Run one reference case for `budget` seconds (at least 2 steps); returns
    (cells, steps, seconds)."""
    spec, budget, warm = args
    os.environ.setdefault("HF_ORACLE_RTOL", "1e-10")
    from oracle import refpy
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
    workload's cases, one single-threaded process per case and core (the
    reference is serial per MPI rank and MPI is absent here).  Batched
    workloads: min(cores, instances) processes at once, each on an instance
    at one of the population's side quantiles (a cost-representative sample);
    the rate is the sum over the processes."""
    from higflow_b200 import host, workloads
    if wl.get("batch") == "c4":
        draws = workloads.batched_giesekus()[:wl.get("count", 256)]
        nproc = procs or min(os.cpu_count() or 1, len(draws))
        sample = protocol_subset(draws, nproc)
        jobs = [(workloads.spec(d), budget_s, warmup) for d in sample]
        desc = (f"{len(jobs)} instances of the batch at its side quantiles (N = {[d.n for d in sample]}), one "
                f"process each, all at once, ~{budget_s:.0f} s of reference steps per process after {warmup} "
                f"warm-up steps")
    elif wl.get("contraction"):
        jobs = [(workloads.contraction_c2(wl["contraction"]), budget_s, warmup)]
        desc = f"~{budget_s:.0f} s of reference steps of the same case after {warmup} warm-up steps, one process"
    else:
        jobs = [(host.cavity(wl["dim"], wl["n"], Re=wl["Re"], dt=wl["dt"]), budget_s, warmup)]
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
        return {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "host": host_info(),
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
    cb = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc, "host": host_info()}
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
    ap.add_argument("--serve-requests", type=int, default=48, help="requests of the served stream to run")
    ap.add_argument("--eager", action="store_true",
                    help="launch kernels one by one instead of one CUDA graph per step (kernel profilers)")
    ap.add_argument("--no-protocol", action="store_true",
                    help="skip the equal-error tolerance protocol (both forms at Poisson rtol 1e-10)")
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

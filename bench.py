#!/usr/bin/env python
"""Benchmark of the HigFlow per-time-step hot path on B200.

One JSON line on rank 0.  A step is one full HigFlow time step (explicit
intermediate velocity, [viscoelastic cell stage,] Poisson projection) of the
workload's mesh on one GPU; with N GPUs every rank runs its own replica
(replicas only: a single case does not shard) and ``value`` is the cell-steps of
all ranks over the slowest rank's time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c1]
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
    "c1": dict(
        name="2D Newtonian lid-driven cavity 64x64 (uniform quadtree, unit square), Re=100, lid u=1, "
             "explicit Euler dt=1e-4, CUBISTA, incremental projection, Poisson CG to 1e-10 relative residual, "
             "zero initial fields",
        program="c1_cavity2d_64.prog.npz", dim=2, n=64, Re=100.0, dt=1e-4,
    ),
    "cav2d_1024": dict(
        name="2D Newtonian lid-driven cavity 1024x1024 (uniform quadtree, unit square), Re=100, lid u=1, "
             "explicit Euler dt=1e-5, CUBISTA, incremental projection, Poisson CG to 1e-10 relative residual, "
             "zero initial fields; program tiled from the recorded 18x18 seed",
        tiled=True, dim=2, n=1024, Re=100.0, dt=1e-5,
    ),
}


def load_program(wl):
    from higflow_b200 import program as hp
    from higflow_b200 import tiling
    if wl.get("tiled"):
        prog = tiling.cavity(wl["dim"], wl["n"])
    else:
        prog = hp.Program.load(os.path.join(REPO, "higflow_b200", "seeds", wl["program"]))
    prog.par["Re"], prog.par["dt"] = wl["Re"], wl["dt"]
    return prog


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
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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
    rows = set()
    for codes in codes_list:
        g = codes[codes < 0]
        rows.update((-g.astype(np.int64) - 1).tolist())
    if not rows:
        return 0
    r = np.fromiter(rows, dtype=np.int64)
    tm = np.unique(prog.row_tmpl[r])
    nnz = int((prog.tmpl_ptr[tm + 1] - prog.tmpl_ptr[tm]).sum())
    return r.size * 16 + tm.size * 8 + nnz * 12


def phase_bytes(prog):
    D = prog.dim
    nf = sum(prog.nfacet[:D])
    nc = prog.ncell
    ve = prog.viscoelastic
    b = {}
    vel = sum(s.size for s in prog.vel_slots) * 4 + nf * (4 + 2)           # slots, flags, delta index
    vel += nf * 8 * 3 + nc * 8 * 2                                          # u (read), u* (write), FU; p, F
    if ve:
        vel += nc * 8 * D * D                                              # S
    vel += _row_bytes(prog, [s.ravel() for s in prog.vel_slots])
    b["velocity"] = vel
    nnz = prog.p_col.size + 1
    b["poisson_init"] = prog.div_slots.size * 4 + nc * 2 + nf * 8 + nc * (8 * 5 + 4) + nnz * 12 + \
        _row_bytes(prog, [prog.div_slots.ravel()])
    # one CG iteration = 2 launches: (z, p_old, matrix) -> (p_new, q) ; (x, p_new, q, r, dinv) -> (x, r, z)
    b["poisson_iter"] = (nc * 4 + nnz * 12 + nc * 8 * 4 + nc * 8 * 8) / 2.0
    b["final"] = sum(s[1:3].size for s in prog.vel_slots) * 4 + nf * (8 * 2 + 2) + nc * 8 * 3
    if ve:
        cs = prog.cell_slots
        b["ve_cell"] = cs.size * 4 + nc * 4 + nf * 8 + nc * 8 * D * D * 5 + _row_bytes(prog, [cs.ravel()])
    return b


# ---------------------------------------------------------------------------
def run_b200(args, rank, world, device):
    import torch
    from higflow_b200 import engine
    from higflow_b200 import program as hp

    wl = WORKLOADS[args.workload]
    prog = load_program(wl)
    opts = engine.options(rtol=1e-10, atol=1e-10, device=device)
    case = engine.Case(prog, opts)
    stream = torch.cuda.ExternalStream(case.stream(), device=device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")

    for _ in range(args.warmup):
        case.step(1)
    case.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    launches0 = case.stats().kernel_launches
    iters0 = case.stats().total_iters
    case.profile(True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(device) as clk:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))          # L2 flush, outside the timed events
                evs[k][0].record(stream)
            case.step(1)
            with torch.cuda.stream(stream):
                evs[k][1].record(stream)
        case.synchronize()
        torch.cuda.synchronize(device)
        t_wall = time.perf_counter() - t_wall
    barrier()
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    st = case.stats()
    launches = st.kernel_launches - launches0
    iters = st.total_iters - iters0
    phases = case.phase_times()
    case.profile(False)

    # slowest rank decides
    t_s = dev_ms / 1e3
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([t_s], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_s = float(t.item())
    cells = prog.ncell
    value = cells * args.steps * world / t_s

    # roofline of the dominant phase (device time inside the timed region)
    pb = phase_bytes(prog)
    dom = max((p for p in phases if phases[p][1] > 0), key=lambda p: phases[p][0])
    dom_ms, dom_launch = phases[dom]
    per_launch_s = dom_ms / 1e3 / dom_launch
    achieved = pb[dom] / per_launch_s / 1e9
    peak, peak_kind = _peaks()
    traffic = None
    tfile = os.path.join(REPO, "profiles", f"traffic_{args.workload}.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get(dom)
        except Exception:
            traffic = None

    # end to end through the C ABI with pinned host buffers, copies every step
    pinned = {}
    names = [(hp.FIELD_U, d) for d in range(prog.dim)] + [(hp.FIELD_P, 0)]
    for fid, comp in names:
        n = prog.field_size(fid, comp)
        pinned[(fid, comp)] = torch.empty(n, dtype=torch.float64, pin_memory=True)
        src = case.get(fid, comp)
        pinned[(fid, comp)].numpy()[:] = src
    h2d = sum(v.numel() * 8 for v in pinned.values())
    import ctypes as C
    L = engine.lib()
    barrier()
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
    t_e2e = time.perf_counter() - t0
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([t_e2e], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = {"value": cells * args.steps * world / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d}
    case.close()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["name"], "cells": cells, "facets": sum(prog.nfacet[:prog.dim]),
                   "precision": "plain FP64", "poisson": "Jacobi-PCG, rtol 1e-10",
                   "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write, outside the step events)",
                   "parallelism": f"replicas x{world}", "program": "recorded from the reference flattener"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "bytes_per_launch": pb[dom], "launch_us": per_launch_s * 1e6, "peak_source": peak_kind},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "poisson_iters_per_step": iters / args.steps,
        "phases_ms_per_step": {p: v[0] / args.steps for p, v in phases.items()},
        "wall_s": t_wall,
        "clocks": clk.summary(),
    }
    return line


def reference_step_rate(wl, steps, warmup):
    """Time the reference's own higflow_solver_step on the workload (oracle build)."""
    from oracle import refpy
    spec = refpy.cavity(wl["dim"], wl["n"], Re=wl["Re"], dt=wl["dt"])
    c = refpy.RefCase(spec)
    c.step(warmup)
    el = c.step(steps)
    cells = c.ncell
    c.close()
    return cells * steps / el, el


def cpu_baseline(wl, budget_s=20.0):
    try:
        from oracle import refpy
        if not refpy.available(wl["dim"]):
            return None
        r, el = reference_step_rate(wl, 5, 1)
        steps = max(5, min(400, int(budget_s / max(el / 5, 1e-6))))
        rate, el = reference_step_rate(wl, steps, 2)
        return {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"{steps} steps of the same case from rest, reference higflow_solver_step "
                          f"(oracle build, single process; the reference is serial per MPI rank) in {el:.1f} s"}
    except Exception as e:  # pragma: no cover
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}


def run_reference(args):
    wl = WORKLOADS[args.workload]
    from oracle import refpy
    if not refpy.available(wl["dim"]):
        print(json.dumps({"impl": "reference", "unavailable": "oracle build of the reference not present"}))
        return
    rate, el = reference_step_rate(wl, args.steps, args.warmup)
    cb = {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
          "sample": f"{args.steps} timed steps after {args.warmup} warm-up steps, reference higflow_solver_step, "
                    "single process (serial per MPI rank)"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["name"], "cells": wl["n"] ** wl["dim"]},
        "cpu_baseline": cb, "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU reference sample")
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
        if world == 1 and not args.no_cpu_baseline and not WORKLOADS[args.workload].get("tiled"):
            line["cpu_baseline"] = cpu_baseline(WORKLOADS[args.workload])
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

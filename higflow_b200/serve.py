"""Serving by continuous batching into the batched engine kernels.

Requests (a recorded step program, a step count, optional initial fields)
arrive at any time.  The scheduler groups the waiting requests that can share a
batch (same dimension, flow type and time schemes) into a cohort: their
programs are concatenated into one batch program and run as one engine case
(hf_case_*: every kernel of a step covers all of the cohort's instances, one
CUDA graph launch per step), each instance with its own step limit
(hf_case_set_step_limits), so an instance that has taken its steps is frozen
while the others go on.  Several cohorts step at once, each on its own CUDA
stream, so a cohort formed from new arrivals overlaps the ones already running;
a cohort is admitted while the device memory the running ones hold plus its
estimate fits the HBM budget.  Fields stay on the device from admission until
the request's steps are done; a finished request's fields are read back
between chunks of steps, when its cohort's stream is idle.  A request whose
step fails (a NaN, a Poisson solve that does not converge) is frozen by the
engine at that step and fails alone; the rest of its cohort goes on.

Each instance's reductions are deterministic and per instance (see
hf_pcg.cuh), so a request's result does not depend on the other requests of
its cohort: the same alone and in any mix (tests/test_gpu_serve.py).

No counterpart in the reference, which runs one case per job.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import engine
from . import program as hp


def batch_key(prog: hp.Program):
    """Requests with equal keys can share one batch program."""
    p = prog.par
    return (prog.dim, int(p["flowtype"]), int(p.get("tempdiscrtype", 0)), int(p.get("ve_discrtype", 0)))



@dataclass
class _Request:
    rid: int
    prog: hp.Program
    steps: int
    fields: Dict[tuple, np.ndarray]
    t_submit: float
    t_admit: float = 0.0
    t_done: float = 0.0
    status: int = 0
    error: str = ""
    done: bool = False
    result: Dict[tuple, np.ndarray] = field(default_factory=dict)


class _Cohort:
    def __init__(self, reqs: List[_Request], opts, keep):
        self.reqs = reqs
        self.prog = hp.Program.concatenate([r.prog for r in reqs]) if len(reqs) > 1 else _as_batch(reqs[0].prog)
        self.case = engine.Case(self.prog, opts)
        for key in keep:
            fid, comp = key
            if not any(key in r.fields for r in reqs):
                continue
            whole = self.case.get(fid, comp)
            off = self.prog.cell_off if fid not in (hp.FIELD_U, hp.FIELD_USTAR, hp.FIELD_FU) else \
                self.prog.facet_off[comp]
            for i, r in enumerate(reqs):
                if key in r.fields:
                    whole[off[i]:off[i + 1]] = r.fields[key]
            self.case.set(fid, comp, whole)
        self.case.set_step_limits([r.steps for r in reqs])
        self.total = max(r.steps for r in reqs)
        self.done_steps = 0
        self.inflight = 0
        self.event = None
        self.nbytes = int(self.case.stats().device_bytes)


def _as_batch(prog: hp.Program) -> hp.Program:
    """A one-instance batch program (so step limits and instance offsets apply)."""
    return hp.Program.concatenate([prog])


class BatchServer:
    """Continuous batching of independent cases on one device (see module
    docstring).  ``max_cohorts``: cohorts stepping at once; ``max_cells``:
    cells per cohort; ``chunk``: steps queued per cohort between checks."""

    def __init__(self, device: int = 0, budget_gb: float = 150.0, max_cohorts: int = 8,
                 max_cells: int = 8_000_000, chunk: int = 32, opts: Optional[hp.HFOptions] = None,
                 window_s: float = 0.25):
        import torch
        self.torch = torch
        self.device = device
        self.budget = int(budget_gb * 1e9)
        self.max_cohorts = max_cohorts
        self.max_cells = max_cells
        self.chunk = chunk
        self.window_s = window_s
        self.opts = opts or engine.options(rtol=1e-10, atol=1e-300, device=device)
        self.mu = threading.Lock()
        self.cv = threading.Condition(self.mu)
        self.queue: deque = deque()
        self.reqs: Dict[int, _Request] = {}
        self.cohorts: List[_Cohort] = []
        self.next_id = 1
        self.stop = False
        self.t0 = time.perf_counter()
        self.cell_steps = 0
        self.cohorts_formed = 0
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    # ------------------------------------------------------------------ api
    def submit(self, prog: hp.Program, steps: int, fields: Optional[Dict[tuple, np.ndarray]] = None) -> int:
        if steps <= 0:
            raise ValueError("steps must be positive")
        with self.cv:
            rid = self.next_id
            self.next_id += 1
            r = _Request(rid, prog, int(steps), dict(fields or {}), time.perf_counter())
            self.reqs[rid] = r
            self.queue.append(r)
            self.cv.notify_all()
        return rid

    def wait(self, rid: int, timeout: Optional[float] = None):
        """(status, queue seconds, submission-to-completion seconds)."""
        with self.cv:
            r = self.reqs[rid]
            if not self.cv.wait_for(lambda: r.done, timeout=timeout):
                raise TimeoutError(rid)
            return r.status, r.t_admit - r.t_submit, r.t_done - r.t_submit

    def error(self, rid: int) -> str:
        """The engine's message for a failed request ('' when it succeeded)."""
        with self.cv:
            return self.reqs[rid].error

    def get(self, rid: int, fid: int, comp: int = 0) -> np.ndarray:
        with self.cv:
            r = self.reqs[rid]
            if not r.done:
                raise RuntimeError("request not finished")
            return r.result[(fid, comp)].copy()

    def release(self, rid: int) -> None:
        with self.cv:
            self.reqs.pop(rid, None)

    def close(self) -> None:
        with self.cv:
            self.stop = True
            self.cv.notify_all()
        self.thread.join()
        for c in self.cohorts:
            c.case.close()
        self.cohorts = []

    # ------------------------------------------------------------ scheduler
    @staticmethod
    def _field_keys(prog: hp.Program):
        keys = [(hp.FIELD_U, d) for d in range(prog.dim)] + [(hp.FIELD_P, 0), (hp.FIELD_DP, 0)]
        if prog.viscoelastic:
            keys += [(hp.FIELD_KERNEL, k) for k in range(prog.dim ** 2)]
            keys += [(hp.FIELD_S, k) for k in range(prog.dim ** 2)]
        return keys

    def _form(self) -> Optional[List[_Request]]:
        """The next cohort from the queue head's group (lock held).  Waiting
        requests gather for ``window_s`` after the head's arrival (or until
        they reach a quarter of ``max_cells``) so that a cohort is a batch
        rather than a single request: a cohort runs until its longest request
        is done, and a cohort of one long request would hold a stream at the
        step's latency floor for all of its steps."""
        if not self.queue or len(self.cohorts) >= self.max_cohorts:
            return None
        waited = time.perf_counter() - self.queue[0].t_submit
        cells = sum(r.prog.ncell for r in self.queue)
        if waited < self.window_s and cells < self.max_cells // 4 and not self.stop:
            return None
        held = sum(c.nbytes for c in self.cohorts)
        key = batch_key(self.queue[0].prog)
        pick, cells, est = [], 0, 0
        for r in list(self.queue):
            if batch_key(r.prog) != key:
                continue
            need = engine.device_bytes(r.prog, self.opts) * 3 // 2
            if pick and (cells + r.prog.ncell > self.max_cells or held + est + need > self.budget):
                break
            if not pick and held + need > self.budget and self.cohorts:
                return None            # wait for memory
            pick.append(r)
            cells += r.prog.ncell
            est += need
        for r in pick:
            self.queue.remove(r)
        return pick

    def _finish(self, c: _Cohort, i: int, r: _Request, status: int = 0, error: str = "") -> None:
        if status == 0:
            for key in self._field_keys(c.prog):
                r.result[key] = c.case.get_instance(key[0], key[1], i).copy()
        with self.cv:
            r.status, r.error = status, error
            r.t_done = time.perf_counter()
            r.done = True
            r.prog = None
            if status == 0:
                self.cell_steps += int(r.steps) * int(c.prog.cell_off[i + 1] - c.prog.cell_off[i])
            self.cv.notify_all()

    def _run(self) -> None:
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            with self.cv:
                if self.stop and not self.cohorts:
                    return
                pick = self._form()
                if pick is None and not self.cohorts:
                    self.cv.wait(timeout=0.05)
                    continue
            if pick:
                now = time.perf_counter()
                for r in pick:
                    r.t_admit = now
                try:
                    c = _Cohort(pick, self.opts, self._field_keys(pick[0].prog))
                except engine.EngineError as e:
                    for r in pick:
                        with self.cv:
                            r.status, r.error, r.t_done, r.done = e.code, str(e), time.perf_counter(), True
                            self.cv.notify_all()
                    continue
                self.cohorts.append(c)
                self.cohorts_formed += 1
            progressed = False
            for c in list(self.cohorts):
                if c.inflight:
                    if not c.event.query():
                        continue
                    status, error, failures = 0, "", None
                    try:
                        c.case.synchronize()
                    except engine.EngineError as e:
                        status, error = e.code, str(e)
                        try:
                            failures = c.case.instance_failures()
                        except engine.EngineError:
                            failures = None
                    c.done_steps += c.inflight
                    c.inflight = 0
                    progressed = True
                    # a failed instance is frozen by the engine and fails its
                    # request alone; any other error ends the cohort
                    whole = status != 0 and (failures is None or not failures.any())
                    for i, r in enumerate(c.reqs):
                        if r.done:
                            continue
                        if whole:
                            self._finish(c, i, r, status, error)
                        elif failures is not None and failures[i]:
                            self._finish(c, i, r, int(failures[i]), error)
                        elif r.steps <= c.done_steps:
                            self._finish(c, i, r)
                    c.total = max([r.steps for r in c.reqs if not r.done], default=c.done_steps)
                    if c.done_steps >= c.total:
                        c.case.close()
                        self.cohorts.remove(c)
                        continue
                n = min(self.chunk, c.total - c.done_steps)
                c.case.step(n, sync=False)
                stream = torch.cuda.ExternalStream(c.case.stream(), device=self.device)
                c.event = torch.cuda.Event()
                c.event.record(stream)
                c.inflight = n
                progressed = True
            if not progressed:
                time.sleep(2e-4)

    def stats(self):
        with self.cv:
            return {"cell_steps": self.cell_steps, "seconds": time.perf_counter() - self.t0,
                    "cohorts": self.cohorts_formed, "queued": len(self.queue), "running": len(self.cohorts)}

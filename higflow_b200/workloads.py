"""Synthetic case populations for the batched and served benchmark configurations.

Seeded draws in a fixed order (numpy.random.default_rng(seed)).  Every case is
a lid-driven cavity on the unit square or a channel [0,8] x [-1,1] (the
geometry of the shipped higflow/example2d_Newt case), and its step program is
recorded by the HigFlow host (higflow_b200/host.py): HigTree's own stencils,
ids and weights.  The explicit time step of each case is a fixed fraction of
its explicit stability bound, recorded with the case.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

from . import host
from . import program as hp


@dataclass
class CaseDraw:
    n: int                 # cells per side (channel: 2n x n/2 cells, the same count)
    model: int             # hp.OLDROYD_B / hp.GIESEKUS (viscoelastic) or -1 (Newtonian)
    De: float              # Weissenberg number (De in HigFlow's parameters)
    alpha: float           # Giesekus mobility
    beta: float
    Re: float
    dt: float
    steps: int
    geometry: str = "cavity"   # "cavity" or "channel"

    @property
    def cells(self) -> int:
        return self.n * self.n


def explicit_dt(n: int, Re: float, frac: float = 0.2) -> float:
    """frac times the explicit bound min(Re h^2 / 4, h) of a unit-lid cavity."""
    h = 1.0 / n
    return frac * min(Re * h * h / 4.0, h)


def batched_giesekus(count: int = 256, seed: int = 0) -> List[CaseDraw]:
    """256 cavities, side N log-uniform in [32, 256], Wi uniform [0.1, 2.0],
    Giesekus alpha uniform [0, 0.5], beta 0.1, Re 1, 2000 steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(32), math.log(256)))))
        wi = float(rng.uniform(0.1, 2.0))
        alpha = float(rng.uniform(0.0, 0.5))
        out.append(CaseDraw(n=n, model=hp.GIESEKUS, De=wi, alpha=alpha, beta=0.1, Re=1.0,
                            dt=explicit_dt(n, 1.0), steps=2000))
    return out


def served_stream(seed: int = 0, rate: float = 50.0, window_s: float = 60.0):
    """Poisson arrivals at ``rate`` per second over ``window_s``: 40% Newtonian
    cavities, 40% Oldroyd-B cavities (Wi uniform [0.1, 1.5]), 20% Giesekus
    channels (alpha uniform [0, 0.5], Wi uniform [0.1, 1.5]; the channel of the
    shipped example2d_Newt case); side N log-uniform in [64, 512] (a channel
    has 2N x N/2 cells); 500-5000 steps.  Inter-arrival times are drawn
    first; the time step of every draw is the cavity's explicit bound at its
    side (the channel's cells are larger, so it is within the channel's)."""
    rng = np.random.default_rng(seed)
    t, times = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > window_s:
            break
        times.append(t)
    cases = []
    for _ in times:
        kind = float(rng.uniform())
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(512)))))
        steps = int(rng.integers(500, 5001))
        if kind < 0.4:
            cases.append(CaseDraw(n=n, model=-1, De=0.0, alpha=0.0, beta=1.0, Re=100.0,
                                  dt=explicit_dt(n, 100.0), steps=steps))
        elif kind < 0.8:
            cases.append(CaseDraw(n=n, model=hp.OLDROYD_B, De=float(rng.uniform(0.1, 1.5)), alpha=0.0,
                                  beta=0.1, Re=1.0, dt=explicit_dt(n, 1.0), steps=steps))
        else:
            cases.append(CaseDraw(n=n, model=hp.GIESEKUS, De=float(rng.uniform(0.1, 1.5)),
                                  alpha=float(rng.uniform(0.0, 0.5)), beta=0.1, Re=1.0,
                                  dt=explicit_dt(n, 1.0), steps=steps, geometry="channel"))
    return times, cases


def served_requests(count: int = 48, step_scale: float = 1.0, seed: int = 0):
    """The first ``count`` requests of the served stream, step counts scaled by
    ``step_scale`` (at least 1): [(arrival s, CaseDraw)].  The stream's offered
    load (about 8.5e9 cell-steps/s over its 60 s window, some 5e11 cell-steps)
    is far above one device; the bounded prefix keeps arrivals, sizes, step
    counts and the mix of the stream and makes the run finish."""
    times, cases = served_stream(seed=seed)
    out = []
    for t, c in list(zip(times, cases))[:count]:
        c = CaseDraw(**{**c.__dict__, "steps": max(1, int(round(c.steps * step_scale)))})
        out.append((t, c))
    return out


def contraction_c2(per_unit: int = 32) -> host.TreesSpec:
    """The 2D Oldroyd-B 4:1 planar contraction configuration: two trees of the
    shipped contraction case at ``per_unit`` cells per unit length (32: 163,840
    cells plus the refined corner squares), Re 0.01, Wi 1.0, beta 1/9,
    log-conformation from the identity, parabolic inflow of mean 1, dt 5e-5.
    The velocity is semi-implicit Euler: explicit Euler at this dt violates the
    explicit viscous bound dt <= Re h^2 / 4 (about 2.4e-6 at h = 1/32) and
    diverges in the reference too."""
    return host.contraction(per_unit, Re=0.01, dt=5e-5, flowtype=hp.VISCOELASTIC, ve_model=hp.OLDROYD_B, De=1.0,
                            beta=1.0 / 9.0, kernel=hp.KERNEL_LOG, kernel_tol=1e-2,
                            tempdiscrtype=hp.SEMI_IMPLICIT_EULER)


def partition(costs, parts: int) -> List[List[int]]:
    """Indices of ``costs`` split into ``parts`` groups by greedy longest-first
    assignment (each item, largest cost first, to the group with the smallest
    total so far; ties to the lowest group).  Every index is in exactly one
    group, groups keep ascending index order, and the largest group total is at
    most 4/3 of the optimum (Graham's bound for this rule)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * parts
    groups: List[List[int]] = [[] for _ in range(parts)]
    for i in order:
        g = min(range(parts), key=lambda k: (load[k], k))
        groups[g].append(i)
        load[g] += costs[i]
    return [sorted(g) for g in groups]


def spec(c: CaseDraw) -> host.CaseSpec:
    """The HigFlow case of one draw: a unit lid-driven cavity of n x n cells, or
    a channel [0,8] x [-1,1] of 2n x n/2 square cells with the shipped case's
    parabolic inflow (mean 1) and outflow; CUBISTA convection, incremental
    projection, and for viscoelastic draws the log-conformation kernel from
    identity with CUBISTA cell convection."""
    par = dict(Re=c.Re, dt=c.dt)
    if c.model >= 0:
        par.update(flowtype=hp.VISCOELASTIC, ve_model=c.model, De=c.De, alpha=c.alpha, beta=c.beta,
                   kernel=hp.KERNEL_LOG, kernel_tol=1e-2, ve_convecdiscrtype=hp.CELL_CUBISTA)
    if c.geometry == "channel":
        return host.channel(2 * c.n, max(2, c.n // 2), length=8.0, half=1.0, umax=1.5, **par)
    return host.cavity(2, c.n, **par)


def programs(draws: List[CaseDraw], procs=None) -> List[hp.Program]:
    """Recorded programs of the draws (host processes in parallel, cached on disk)."""
    return host.record_many([spec(c) for c in draws], procs=procs)


def program(c: CaseDraw) -> hp.Program:
    return programs([c], procs=1)[0]


def batch(draws: List[CaseDraw], procs=None) -> hp.Program:
    return hp.Program.concatenate(programs(draws, procs=procs))

"""Algorithmic bytes of one HigFlow time step, from its step program.

The convention (fixed by the reference's data layout, the same for every
implementation that runs the step): per step

    B_step = sum over the reference's kernels of (F_k + S_k)  +  n_it * B_it

* F_k: the field arrays the reference's kernel reads (each once) plus those it
  writes (once), at their stored width (8 bytes: the fields are FP64 in both
  precision forms).
* S_k: the stencil bytes of the kernel's distinct queries,
  4 R_k + sum over their entries of (4 + w [entry is not a centre hit]),
  R_k = distinct (field, query) pairs and w the width of a stencil weight
  (8 plain, 4 mixed).  A centre hit is one 4-byte id; a general row carries
  its ids and weights (dp_interpolate_from_stencil, pdomain.c:1026-1053).
  The recorder merges identical queries of a field, so distinct recorded rows
  per field are the distinct queries.
* Poisson, per iteration of Jacobi-style PCG on the CSR operator:
  B_it = 4 (N_c + 1) + nnz_P (4 + w) + 13 w N_c (SpMV reads p, writes q;
  update reads x, p, r, q, D^-1 and writes x, r, z; direction reads z, p and
  writes p), n_it the measured iterations; the mixed form's FP32 inner
  iterations count at w = 4 and each FP64 refinement sweep as one more SpMV
  pass at w = 8.

The reference kernels and the fields they move (hig-flow-step.c,
hig-flow-step-viscoelastic.c, hig-flow-step-generalized-newtonian.c):

  velocity  (higflow_explicit_euler_intermediate_velocity[_viscoelastic],
             :613-660 / :931-980): reads u[d], FU[d] per facet direction, p,
             F per cell (and S per component, viscoelastic); writes u*[d]
  ve_cell   (velocity-derivative tensor :14-97, constitutive update :352-544,
             polymeric tensor :212-347): reads u[d], Du, S, K; writes Du, K, S
  divergence (higflow_pressure :48-131): reads u*[d]; writes the rhs b
  final     (higflow_final_velocity / _pressure :242-340): reads u*[d], dp,
             p; writes u[d], p
"""
from __future__ import annotations

from typing import Dict, Iterable, Tuple

import numpy as np

from . import program as hp


def _vel_tag(D: int, d: int, s: int) -> Tuple[str, int]:
    """(field family, component) a velocity slot reads."""
    if s == hp.V_FU:
        return ("FU", d)
    if s in (hp.V_PL, hp.V_PR):
        return ("p", 0)
    if s in (hp.V_FL, hp.V_FR):
        return ("F", 0)
    if s < hp.v_nslot(D, False):
        d2, k = divmod(s - hp.V_BLK0, hp.V_NB)
        return ("u", d2 if (k < 4 or k >= 8) else d)
    d2 = (s - hp.v_nslot(D, False)) // hp.V_NS
    return ("S", d * D + d2)


def _cell_tag(D: int, s: int) -> Tuple[str, int]:
    if s == hp.C_SELF:
        return ("cellself", 0)
    if s < hp.C_BLK0 + hp.C_NB * D:
        dim, k = divmod(s - hp.C_BLK0, hp.C_NB)
        return ("u", dim) if k < 2 else ("K", 0)
    pair = (s - hp.C_BLK0 - hp.C_NB * D) // hp.C_NQ
    return ("u", pair // (D - 1))


def query_bytes(prog: hp.Program, slots: Iterable[Tuple[Tuple[str, int], np.ndarray]], w: int) -> Dict[str, int]:
    """S_k of a kernel whose queries are the given slot rows (field tag, codes)."""
    lens = np.diff(prog.tmpl_ptr)[prog.row_tmpl] if prog.row_tmpl.size else np.zeros(0, np.int64)
    centre: Dict[Tuple[str, int], np.ndarray] = {}
    rows: Dict[Tuple[str, int], np.ndarray] = {}
    for tag, codes in slots:
        c = np.asarray(codes).ravel()
        hit = c[c >= 0]
        gen = -c[c < 0].astype(np.int64) - 1
        if hit.size:
            m = centre.get(tag)
            if m is None:
                m = centre[tag] = np.zeros(int(hit.max()) + 1, dtype=bool)
            elif m.size <= hit.max():
                m = centre[tag] = np.concatenate([m, np.zeros(int(hit.max()) + 1 - m.size, dtype=bool)])
            m[hit] = True
        if gen.size:
            m = rows.get(tag)
            if m is None:
                m = rows[tag] = np.zeros(prog.row_rhs.size, dtype=bool)
            m[gen] = True
    r_centre = int(sum(int(m.sum()) for m in centre.values()))
    r_rows = int(sum(int(m.sum()) for m in rows.values()))
    entries = int(sum(int(lens[m].sum()) for m in rows.values()))
    return {"queries": r_centre + r_rows, "centre_hits": r_centre, "rows": r_rows, "row_entries": entries,
            "bytes": 4 * (r_centre + r_rows) + 4 * r_centre + entries * (4 + w)}


def step_bytes(prog: hp.Program, mixed: bool) -> Dict[str, Dict[str, int]]:
    """F_k + S_k of every reference kernel of one step (no Poisson
    iterations), with the stencil weights at 4 bytes in the mixed form."""
    D = prog.dim
    w = 4 if mixed else 8
    nf = int(sum(prog.nfacet[:D]))
    nc = int(prog.ncell)
    ve = prog.viscoelastic
    out = {}
    vel_slots = []
    for d in range(D):
        for s in range(prog.vel_slots[d].shape[0]):
            b0 = hp.V_BLK0 + hp.V_NB * d
            if b0 <= s < b0 + 4:      # the facet's own u[d] corners are not queried
                continue
            if not ve and s >= hp.v_nslot(D, False):
                continue
            vel_slots.append((_vel_tag(D, d, s), prog.vel_slots[d][s]))
    q = query_bytes(prog, vel_slots, w)
    f = 8 * (nf * 3 + nc * 2 + (nc * D * D if ve else 0))
    out["velocity"] = {"F": f, "S": q["bytes"], **{k: v for k, v in q.items() if k != "bytes"}}
    if ve:
        cs = [(_cell_tag(D, s), prog.cell_slots[s]) for s in range(prog.cell_slots.shape[0])]
        q = query_bytes(prog, cs, w)
        f = 8 * nf + 8 * D * D * nc * (1 + 4 + 3)
        out["ve_cell"] = {"F": f, "S": q["bytes"], **{k: v for k, v in q.items() if k != "bytes"}}
    ds = [(("us", s // 2), prog.div_slots[s]) for s in range(prog.div_slots.shape[0])]
    q = query_bytes(prog, ds, 8)
    out["divergence"] = {"F": 8 * (nf + nc), "S": q["bytes"], **{k: v for k, v in q.items() if k != "bytes"}}
    fs = [(("dp", 0), prog.vel_slots[d][s]) for d in range(D) for s in (hp.V_PL, hp.V_PR)]
    q = query_bytes(prog, fs, 8)
    out["final"] = {"F": 8 * (2 * nf + 3 * nc), "S": q["bytes"], **{k: v for k, v in q.items() if k != "bytes"}}
    return out


def poisson_iter_bytes(prog: hp.Program, w: int) -> int:
    """B_it of one Jacobi-PCG iteration on the CSR Poisson operator."""
    nc = int(prog.ncell)
    return 4 * (nc + 1) + int(prog.p_col.size) * (4 + w) + 13 * w * nc


def whole_step(prog: hp.Program, mixed: bool, iters: float, sweeps: float = 0.0) -> Dict[str, float]:
    """B_step with ``iters`` Poisson iterations (for the mixed form: inner FP32
    iterations) and ``sweeps`` FP64 refinement sweeps, averaged per step."""
    parts = step_bytes(prog, mixed)
    fixed = sum(v["F"] + v["S"] for v in parts.values())
    nc = int(prog.ncell)
    spmv64 = 4 * (nc + 1) + int(prog.p_col.size) * 12 + 2 * 8 * nc
    pois = iters * poisson_iter_bytes(prog, 4 if mixed else 8) + sweeps * spmv64
    return {"bytes": fixed + pois, "fixed": fixed, "poisson": pois,
            "parts": {k: v["F"] + v["S"] for k, v in parts.items()}}

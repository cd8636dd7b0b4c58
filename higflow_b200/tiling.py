"""Step programs for large uniform meshes, tiled from a small recorded seed.

On a uniform single-level box mesh every stencil HigTree builds for an element
depends on where the element sits relative to the walls: once an element is
``R`` or more cells from a wall along an axis, moving it along that axis
translates its stencil.  A seed program recorded by the flattener on a mesh of
``2R+2`` cells per axis contains every stencil class, and a program for a
larger mesh of the same box, boundary conditions and cell aspect ratio follows
by mapping each element to its class in the seed and translating ids.
Translated general rows reuse the seed row as a template with a base offset
(row-major ids make a translation a constant index shift).

One caveat is inherited from HigTree itself: its interpolation stencils keep
the nearest candidates by distances computed in absolute coordinates, so where
several candidates are equidistant the reference's choice can differ with the
element's position.  A tiled program uses the seed's choice for every element
of a class, which gives the same discretisation up to that tie-break.  Programs
that must match the reference bit for bit are recorded, not tiled.

The id layouts are HigTree's for a single uniform tree: cells row-major with
the last axis fastest (higtree/src/higtree.c:23-37); interior facets normal to
``d`` row-major over the grid with ``n[d]-1`` positions along ``d``
(sfd_get_domain_facetiterator, higtree/src/domain.c:1834-1867).  Poisson
coefficients are rescaled from the seed's cell size to the target's.
"""
from __future__ import annotations

import os
from typing import List, Sequence

import numpy as np

from . import program as hp

SEEDS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "seeds")


def _strides(ext: Sequence[int]) -> np.ndarray:
    D = len(ext)
    s = np.ones(D, dtype=np.int64)
    for k in range(D - 2, -1, -1):
        s[k] = s[k + 1] * ext[k + 1]
    return s


def _coords(lin: np.ndarray, ext: Sequence[int]) -> np.ndarray:
    lin = np.asarray(lin, dtype=np.int64)
    out = np.empty(lin.shape + (len(ext),), dtype=np.int64)
    for k in range(len(ext) - 1, -1, -1):
        out[..., k] = lin % ext[k]
        lin = lin // ext[k]
    return out


def _lin(c: np.ndarray, ext: Sequence[int]) -> np.ndarray:
    return (c * _strides(ext)).sum(axis=-1)


def _grid_ext(n: Sequence[int], g: int) -> List[int]:
    """Extent of field grid g: -1 = cells, d >= 0 = facets normal to d."""
    e = list(n)
    if g >= 0:
        e[g] -= 1
    return e


def _classify(tc: np.ndarray, te: Sequence[int], se: Sequence[int], R: int):
    """Seed element coords and translation for target element coords tc."""
    te = np.asarray(te)
    se = np.asarray(se)
    low = tc < R
    high = (te - 1 - tc) < R
    sc = np.where(low, tc, np.where(high, se - (te - tc), R))
    return sc, tc - sc


class _Remap:
    """Seed id -> target id for translation zero, per field grid, and the
    linear shift of each element's translation, per grid."""

    def __init__(self, D, sn, tn):
        self.D, self.sn, self.tn = D, sn, tn
        self.map = {}
        self.strides = {}
        for g in range(-1, D):
            se, te = _grid_ext(sn, g), _grid_ext(tn, g)
            self.map[g] = _lin(_coords(np.arange(int(np.prod(se))), se), te)
            self.strides[g] = _strides(te)

    def shifts(self, off: np.ndarray):
        return {g: off @ self.strides[g] for g in range(-1, self.D)}


class _Rows:
    """General-row references: (seed row, grid, linear shift) -> target rows."""

    def __init__(self, seed: hp.Program, remap: _Remap):
        self.seed, self.remap = seed, remap
        self.rows, self.grids, self.shifts = [], [], []
        self.count = 0

    def add(self, seed_rows: np.ndarray, grid: int, shift: np.ndarray) -> np.ndarray:
        """Register references; returns their new (negative) codes."""
        n = seed_rows.size
        self.rows.append(seed_rows)
        self.grids.append(np.full(n, grid + 1, dtype=np.int64))
        self.shifts.append(shift)
        codes = -(np.arange(self.count, self.count + n, dtype=np.int64) + 1)
        self.count += n
        return codes

    def emit(self, kw: dict):
        seed = self.seed
        if not self.rows:
            kw.update(row_tmpl=np.zeros(0, np.int32), row_base=np.zeros(0, np.int32), row_rhs=np.zeros(0),
                      tmpl_ptr=np.zeros(1, np.int64), tmpl_col=np.zeros(0, np.int32), tmpl_w=np.zeros(0))
            return
        r = np.concatenate(self.rows)
        g1 = np.concatenate(self.grids)
        base = np.concatenate(self.shifts)
        # one template per distinct (seed row, grid); small key range -> table
        tk = r * 4 + g1
        present = np.zeros(int(tk.max()) + 1, dtype=bool)
        present[tk] = True
        keys = np.nonzero(present)[0]
        table = np.full(present.size, -1, dtype=np.int64)
        table[keys] = np.arange(keys.size)
        tptr = [0]
        tcol, tw = [], []
        for key in keys.tolist():
            sr, g = key // 4, key % 4 - 1
            st = seed.row_tmpl[sr]
            a, b = seed.tmpl_ptr[st], seed.tmpl_ptr[st + 1]
            sc = seed.tmpl_col[a:b].astype(np.int64) + seed.row_base[sr]
            tcol.append(self.remap.map[g][sc])
            tw.append(seed.tmpl_w[a:b])
            tptr.append(tptr[-1] + (b - a))
        if base.max(initial=0) > np.iinfo(np.int32).max:
            raise ValueError("mesh too large for int32 row bases")
        kw.update(
            row_tmpl=table[tk].astype(np.int32), row_base=base.astype(np.int32),
            row_rhs=seed.row_rhs[r].astype(np.float64),
            tmpl_ptr=np.array(tptr, dtype=np.int64),
            tmpl_col=np.concatenate(tcol).astype(np.int32), tmpl_w=np.concatenate(tw).astype(np.float64),
        )


def _remap_slots(seed_slots, sel, grid_of_slot, shifts, remap: _Remap, rows: _Rows, skip=()):
    """Translate a (nslot, seed elements) slot table to target elements."""
    ns = seed_slots.shape[0]
    ne = sel.size
    out = np.empty((ns, ne), dtype=np.int32)
    for s in range(ns):
        if s in skip:
            out[s] = 0
            continue
        g = grid_of_slot(s)
        codes = seed_slots[s][sel].astype(np.int64)
        direct = codes >= 0
        res = np.empty(ne, dtype=np.int64)
        res[direct] = remap.map[g][codes[direct]] + shifts[g][direct]
        gen = ~direct
        if gen.any():
            res[gen] = rows.add(-codes[gen] - 1, g, shifts[g][gen])
        out[s] = res
    return out


def tile(seed: hp.Program, seed_n: Sequence[int], R: int, n: Sequence[int], lengths: Sequence[float],
         seed_lengths: Sequence[float], newtonian: bool = False) -> hp.Program:
    """Program for a uniform mesh with ``n`` cells per axis on a box with edge
    ``lengths`` from a seed recorded on ``seed_n`` cells of a box with edge
    ``seed_lengths`` (same boundary conditions and cell aspect ratio)."""
    D = seed.dim
    sn, tn = list(seed_n), list(n)
    if len(tn) != D or any(t < s for t, s in zip(tn, sn)) or any(s < 2 * R + 2 for s in sn):
        raise ValueError("target must be at least the seed size, seed at least 2R+2 per axis")
    sdelta = np.array([seed_lengths[k] / sn[k] for k in range(D)])
    tdelta = np.array([lengths[k] / tn[k] for k in range(D)])
    ratio = sdelta / tdelta
    if not np.allclose(ratio, ratio[0], rtol=1e-12, atol=0):
        raise ValueError("cell aspect ratio differs from the seed's")
    scale = float(ratio[0]) ** 2
    ve = seed.viscoelastic and not newtonian
    remap = _Remap(D, sn, tn)
    rows = _Rows(seed, remap)
    kw = {}

    # velocity stage
    nsv = hp.v_nslot(D, ve)
    vel_slots, vel_flags, vel_delta = [], [], []
    for d in range(D):
        se, te = _grid_ext(sn, d), _grid_ext(tn, d)
        nf = int(np.prod(te))
        tc = _coords(np.arange(nf), te)
        sc, off = _classify(tc, te, se, R)
        sel = _lin(sc, se)
        b0 = hp.V_BLK0 + hp.V_NB * d
        vel_slots.append(_remap_slots(seed.vel_slots[d][:nsv], sel, lambda s, d=d: hp.vel_slot_grid(D, d, s),
                                      remap.shifts(off), remap, rows, skip=set(range(b0, b0 + 4))))
        vel_flags.append(seed.vel_flags[d][sel].copy())
        vel_delta.append(np.zeros(nf, dtype=np.uint16))

    # cells: divergence slots, viscoelastic cell slots, Poisson rows
    nc = int(np.prod(tn))
    tc = _coords(np.arange(nc), tn)
    sc, off = _classify(tc, tn, sn, R)
    sel = _lin(sc, sn)
    sh = remap.shifts(off)
    div = _remap_slots(seed.div_slots, sel, lambda s: s // 2, sh, remap, rows)
    cell_slots = cell_flags = None
    if ve:
        cell_slots = _remap_slots(seed.cell_slots, sel, lambda s: hp.cell_slot_grid(D, s), sh, remap, rows)
        cell_flags = seed.cell_flags[sel].copy()
    rows.emit(kw)

    # pressure pin: the cell holding the box centre (remove_pressure_singularity,
    # hig-flow-step.c:14-45); its Poisson row is empty in every program
    pin = -1
    if seed.pin_row >= 0:
        ps = _coords(np.array([seed.pin_row]), sn)[0]
        pt = np.array([(tn[k] // 2 + (ps[k] - sn[k] // 2)) if tn[k] % 2 == 0 else (tn[k] - 1) // 2
                       for k in range(D)])
        pin = int(_lin(pt, tn))

    # Poisson rows: seed row of the class, columns translated, 1/delta^2 rescaled.
    # The seed's own pinned row is empty, so a class represented by it is taken
    # from the next interior cell instead (index R+1 is also R from both walls).
    psc, poff = sc.copy(), off.copy()
    hit = sel == seed.pin_row
    if hit.any():
        psc[hit] = np.where(psc[hit] == R, R + 1, psc[hit])
        poff[hit] = tc[hit] - psc[hit]
    psel = _lin(psc, sn)
    if np.any(psel == seed.pin_row):
        raise ValueError("seed pin lies in a boundary class; record a larger seed")
    lens = (seed.p_ptr[1:] - seed.p_ptr[:-1])[psel]
    if pin >= 0:
        lens[pin] = 0
    p_ptr = np.zeros(nc + 1, dtype=np.int64)
    np.cumsum(lens, out=p_ptr[1:])
    rep = np.repeat(np.arange(nc), lens)
    first = np.repeat(seed.p_ptr[:-1][psel], lens)
    k = first + (np.arange(p_ptr[-1]) - np.repeat(p_ptr[:-1], lens))
    pshift = poff @ remap.strides[-1]
    p_col = (remap.map[-1][seed.p_col[k].astype(np.int64)] + pshift[rep]).astype(np.int32)
    p_val = seed.p_val[k] * scale
    p_brhs = seed.p_brhs[psel] * scale

    par = dict(seed.par)
    if not ve:
        par["flowtype"] = hp.NEWTONIAN
    return hp.Program(
        par=par, ncell=nc, nfacet=[int(np.prod(_grid_ext(tn, d))) for d in range(D)] + [0] * (3 - D),
        delta=tdelta.reshape(1, D), vel_slots=vel_slots, vel_flags=vel_flags, vel_delta=vel_delta,
        div_slots=div, cell_delta=np.zeros(nc, dtype=np.uint16),
        p_ptr=p_ptr, p_col=p_col, p_val=p_val, p_brhs=p_brhs,
        pin_row=pin, pin_value=seed.pin_value,
        cell_slots=cell_slots, cell_flags=cell_flags, **kw,
    )


def load_seed(name: str):
    """A committed seed: (program, seed_n, R, seed_lengths)."""
    z = np.load(os.path.join(SEEDS, f"{name}.meta.npz"))
    prog = hp.Program.load(os.path.join(SEEDS, f"{name}.prog.npz"))
    return prog, [int(x) for x in z["n"]], int(z["R"]), [float(x) for x in z["lengths"]]


_seed_cache = {}


def cavity(dim: int, n: int, viscoelastic: bool = False, **par) -> hp.Program:
    """Lid-driven cavity program on the unit square/cube with n cells per axis
    (lid u_0 = 1 on the top face, no-slip walls, pinned Neumann pressure)."""
    name = f"cavity{dim}d"
    if name not in _seed_cache:
        _seed_cache[name] = load_seed(name)
    seed, sn, R, sl = _seed_cache[name]
    prog = tile(seed, sn, R, [n] * dim, [1.0] * dim, sl, newtonian=not viscoelastic)
    for k, v in par.items():
        if k not in prog.par:
            raise KeyError(k)
        prog.par[k] = v
    return prog

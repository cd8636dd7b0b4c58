"""Step programs for large uniform meshes, tiled from a small recorded seed.

On a uniform single-level box mesh every stencil HigTree builds for an element
depends only on where the element sits relative to the walls: once an element is
``R`` or more cells from a wall along an axis, moving it along that axis just
translates its stencil.  A seed program recorded by the flattener on a mesh of
``2R+2`` cells per axis therefore contains every distinct stencil class, and a
program for any larger mesh of the same box, boundary conditions and cell
aspect ratio follows by mapping each element to its class in the seed and
translating ids.  Translated general rows reuse the seed row as a template with
a base offset (row-major ids make a translation a constant index shift), so
interior interpolation weights are stored once however large the mesh is.

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


def _vel_slot_grid(D: int, d: int, s: int) -> int:
    if s == hp.V_FU:
        return d
    if s <= hp.V_FR:
        return -1
    if s < hp.v_nslot(D, False):
        d2, k = divmod(s - hp.V_BLK0, hp.V_NB)
        return d2 if (k < 4 or k >= 8) else d
    return -1


def _cell_slot_grid(D: int, s: int) -> int:
    if s == hp.C_SELF:
        return -1
    if s < hp.C_BLK0 + hp.C_NB * D:
        dim, k = divmod(s - hp.C_BLK0, hp.C_NB)
        return dim if k < 2 else -1
    pair = (s - hp.C_BLK0 - hp.C_NB * D) // hp.C_NQ
    return pair // (D - 1)


class _Rows:
    """Collects (seed row, grid, offset) references and emits target rows."""

    def __init__(self, seed: hp.Program, sn, tn):
        self.seed, self.sn, self.tn = seed, sn, tn
        self.keys = []      # arrays (M, 2 + D): seed row, grid, offset...
        self.where = []     # (array to write, flat positions)

    def add(self, rows: np.ndarray, grid: int, off: np.ndarray, out: np.ndarray, pos: np.ndarray):
        if rows.size == 0:
            return
        k = np.empty((rows.size, 2 + off.shape[1]), dtype=np.int64)
        k[:, 0] = rows
        k[:, 1] = grid
        k[:, 2:] = off
        self.keys.append(k)
        self.where.append((out, pos))

    def emit(self, prog_kw: dict):
        seed, D = self.seed, self.seed.dim
        if not self.keys:
            prog_kw.update(row_tmpl=np.zeros(0, np.int32), row_base=np.zeros(0, np.int32),
                           row_rhs=np.zeros(0), tmpl_ptr=np.zeros(1, np.int64),
                           tmpl_col=np.zeros(0, np.int32), tmpl_w=np.zeros(0))
            return
        K = np.concatenate(self.keys)
        # one int64 key per reference: ((row * 4 + grid + 1) * cells + linear offset);
        # offsets are non-negative and smaller than the target extent on every axis
        P = int(np.prod(self.tn))
        key = (K[:, 0] * 4 + (K[:, 1] + 1)) * P + (K[:, 2:] * _strides(self.tn)).sum(axis=1)
        ukey, first, inv = np.unique(key, return_index=True, return_inverse=True)
        uniq = K[first]
        inv = inv.reshape(-1)
        # write the new codes back
        start = 0
        for (out, pos), k in zip(self.where, self.keys):
            out.reshape(-1)[pos] = -(inv[start:start + len(k)] + 1)
            start += len(k)
        # one template per distinct (seed row, grid)
        tkeys, tinv = np.unique(uniq[:, :2], axis=0, return_inverse=True)
        tinv = tinv.reshape(-1)
        tptr = [0]
        tcol, tw = [], []
        for sr, g in tkeys:
            st = seed.row_tmpl[sr]
            a, b = seed.tmpl_ptr[st], seed.tmpl_ptr[st + 1]
            sc = seed.tmpl_col[a:b].astype(np.int64) + seed.row_base[sr]
            se, te = _grid_ext(self.sn, int(g)), _grid_ext(self.tn, int(g))
            tcol.append(_lin(_coords(sc, se), te))
            tw.append(seed.tmpl_w[a:b])
            tptr.append(tptr[-1] + (b - a))
        base = np.empty(len(uniq), dtype=np.int64)
        for g in np.unique(uniq[:, 1]):
            m = uniq[:, 1] == g
            base[m] = (uniq[m, 2:] * _strides(_grid_ext(self.tn, int(g)))).sum(axis=1)
        if base.max(initial=0) > np.iinfo(np.int32).max:
            raise ValueError("mesh too large for int32 row bases")
        prog_kw.update(
            row_tmpl=tinv.astype(np.int32), row_base=base.astype(np.int32),
            row_rhs=seed.row_rhs[uniq[:, 0]].astype(np.float64),
            tmpl_ptr=np.array(tptr, dtype=np.int64),
            tmpl_col=(np.concatenate(tcol) if tcol else np.zeros(0)).astype(np.int32),
            tmpl_w=(np.concatenate(tw) if tw else np.zeros(0)).astype(np.float64),
        )


def _classify(tc: np.ndarray, te: Sequence[int], se: Sequence[int], R: int):
    """Seed element coords and translation for target element coords tc."""
    te = np.asarray(te)
    se = np.asarray(se)
    low = tc < R
    high = (te - 1 - tc) < R
    sc = np.where(low, tc, np.where(high, se - (te - tc), R))
    return sc, tc - sc


def _remap_codes(codes, grid, off, sn, tn, rows: _Rows, out, pos_base):
    """Direct codes translate; general codes become (row, grid, offset) refs."""
    direct = codes >= 0
    res = out.reshape(-1)
    if direct.any():
        se, te = _grid_ext(sn, grid), _grid_ext(tn, grid)
        c = _coords(codes[direct], se) + off[direct]
        res[pos_base[direct]] = _lin(c, te)
    gen = ~direct
    if gen.any():
        rows.add(-codes[gen].astype(np.int64) - 1, grid, off[gen], out, pos_base[gen])


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
    rows = _Rows(seed, sn, tn)
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
        out = np.empty((nsv, nf), dtype=np.int32)
        for s in range(nsv):
            b0 = hp.V_BLK0 + hp.V_NB * d
            if b0 <= s < b0 + 4:
                out[s] = 0          # the tangential-average slots are unused for d2 == d
                continue
            codes = seed.vel_slots[d][s][sel]
            _remap_codes(codes, _vel_slot_grid(D, d, s), off, sn, tn, rows, out, s * nf + np.arange(nf))
        vel_slots.append(out)
        vel_flags.append(seed.vel_flags[d][sel].copy())
        vel_delta.append(np.zeros(nf, dtype=np.uint16))

    # cells: divergence slots, viscoelastic cell slots, Poisson rows
    nc = int(np.prod(tn))
    tc = _coords(np.arange(nc), tn)
    sc, off = _classify(tc, tn, sn, R)
    sel = _lin(sc, sn)
    div = np.empty((2 * D, nc), dtype=np.int32)
    for s in range(2 * D):
        _remap_codes(seed.div_slots[s][sel], s // 2, off, sn, tn, rows, div, s * nc + np.arange(nc))
    cell_slots = cell_flags = None
    if ve:
        ncs = hp.c_nslot(D)
        cell_slots = np.empty((ncs, nc), dtype=np.int32)
        for s in range(ncs):
            _remap_codes(seed.cell_slots[s][sel], _cell_slot_grid(D, s), off, sn, tn, rows, cell_slots,
                         s * nc + np.arange(nc))
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
        mid = (psc[hit] == R)
        psc[hit] = np.where(mid, R + 1, psc[hit])
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
    scol = seed.p_col[k].astype(np.int64)
    p_col = _lin(_coords(scol, sn) + poff[rep], tn).astype(np.int32)
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


def cavity(dim: int, n: int, viscoelastic: bool = False, **par) -> hp.Program:
    """Lid-driven cavity program on the unit square/cube with n cells per axis
    (lid u_0 = 1 on the top face, no-slip walls, pinned Neumann pressure)."""
    seed, sn, R, sl = load_seed(f"cavity{dim}d")
    prog = tile(seed, sn, R, [n] * dim, [1.0] * dim, sl, newtonian=not viscoelastic)
    for k, v in par.items():
        if k not in prog.par:
            raise KeyError(k)
        prog.par[k] = v
    return prog

"""Step programs: the flattened stencil tables one HigFlow time step reads.

``Program`` holds an ``hf_program`` (``include/higflow_b200.h``) as numpy
arrays.  It converts to the C struct for the engine (``to_c``), copies out of a
C struct written by a flattener (``from_c``) and round-trips through ``.npz``
files for fixtures.  Slot semantics are documented in the header; in short a
slot code >= 0 is a direct field index (a stencil centre hit) and a code < 0
names a general stencil row ``-code-1`` whose value is
``-rhs + sum(w * field[col])`` accumulated in row order
(``higtree/src/pdomain.c:1026-1053``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

# enumerations (include/higflow_b200.h)
NEWTONIAN, VISCOELASTIC = 0, 3
GPTT, FENE_P, E_FENE = 3, 4, 5
VE_EXPLICIT, VE_IMPLICIT = 0, 1
EXPLICIT_EULER, EXPLICIT_RK2, EXPLICIT_RK3, SEMI_IMPLICIT_EULER, SEMI_IMPLICIT_CN, SEMI_IMPLICIT_BDF2 = 0, 1, 2, 3, 4, 5
NON_INCREMENTAL, INCREMENTAL = 0, 1
CENTRAL, FIRST_ORDER, SECOND_ORDER = 0, 1, 2
MCU, CUBISTA, QUICK = 0, 1, 2
OLDROYD_B, GIESEKUS, LPTT = 0, 1, 2
CELL_CENTRAL, CELL_CUBISTA = 0, 1
KERNEL_IDENTITY, KERNEL_LOG, KERNEL_SQRT = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
POISSON_AUTO, POISSON_CG, POISSON_BICGSTAB = 0, 1, 2
PRECOND_AUTO, PRECOND_JACOBI, PRECOND_AMG = 0, 1, 2

FIELD_U, FIELD_USTAR, FIELD_P, FIELD_DP, FIELD_F, FIELD_FU, FIELD_KERNEL, FIELD_S, FIELD_DU = range(9)

# slot layout constants
V_FU, V_PL, V_PR, V_FL, V_FR, V_BLK0, V_NB = 0, 1, 2, 3, 4, 5, 10
V_V4, V_UL, V_UR, V_ULL, V_URR, V_VCR, V_VCL = 0, 4, 5, 6, 7, 8, 9
V_NS = 4
C_SELF, C_BLK0, C_NB = 0, 1, 6
C_UVL, C_UVR, C_KL, C_KR, C_KLL, C_KRR = range(6)
C_NQ = 4


def v_nslot(dim: int, ve: bool) -> int:
    n = V_BLK0 + V_NB * dim
    return n + V_NS * dim if ve else n


def c_nslot(dim: int) -> int:
    return C_BLK0 + C_NB * dim + C_NQ * dim * (dim - 1)


def vel_slot_grid(D: int, d: int, s: int) -> int:
    """Field grid a velocity-stage slot reads: -1 cells, k >= 0 facets normal to k."""
    if s == V_FU:
        return d
    if s <= V_FR:
        return -1
    if s < v_nslot(D, False):
        d2, k = divmod(s - V_BLK0, V_NB)
        return d2 if (k < 4 or k >= 8) else d
    return -1


def cell_slot_grid(D: int, s: int) -> int:
    """Field grid a viscoelastic cell-stage slot reads."""
    if s == C_SELF:
        return -1
    if s < C_BLK0 + C_NB * D:
        dim, k = divmod(s - C_BLK0, C_NB)
        return dim if k < 2 else -1
    pair = (s - C_BLK0 - C_NB * D) // C_NQ
    return pair // (D - 1)


class HFParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("flowtype", C.c_int32), ("projtype", C.c_int32),
        ("convecdiscrtype", C.c_int32), ("secondconvecdiscrtype", C.c_int32),
        ("ve_model", C.c_int32), ("ve_convecdiscrtype", C.c_int32), ("kernel", C.c_int32),
        ("Re", C.c_double), ("dt", C.c_double),
        ("De", C.c_double), ("beta", C.c_double), ("kernel_tol", C.c_double),
        ("alpha", C.c_double), ("epsilon", C.c_double), ("xi", C.c_double),
        ("tempdiscrtype", C.c_int32), ("pad_", C.c_int32),
        ("L2_fene", C.c_double), ("lambda_fene", C.c_double), ("E_fene", C.c_double),
        ("ve_discrtype", C.c_int32), ("pad2_", C.c_int32),
        ("alpha_gptt", C.c_double), ("beta_gptt", C.c_double), ("gamma_gptt", C.c_double),
    ]


_P = C.POINTER


class HFProgram(C.Structure):
    _fields_ = [
        ("par", HFParams),
        ("ncell", C.c_int32),
        ("nfacet", C.c_int32 * 3),
        ("ndelta", C.c_int32),
        ("delta", _P(C.c_double)),
        ("nrows", C.c_int64),
        ("row_tmpl", _P(C.c_int32)), ("row_base", _P(C.c_int32)), ("row_rhs", _P(C.c_double)),
        ("ntmpl", C.c_int64), ("nnz", C.c_int64),
        ("tmpl_ptr", _P(C.c_int64)), ("tmpl_col", _P(C.c_int32)), ("tmpl_w", _P(C.c_double)),
        ("vel_nslot", C.c_int32),
        ("vel_slots", _P(C.c_int32) * 3),
        ("vel_flags", _P(C.c_uint32) * 3),
        ("vel_delta", _P(C.c_uint16) * 3),
        ("div_slots", _P(C.c_int32)),
        ("cell_delta", _P(C.c_uint16)),
        ("pnnz", C.c_int64),
        ("p_ptr", _P(C.c_int64)), ("p_col", _P(C.c_int32)), ("p_val", _P(C.c_double)),
        ("p_brhs", _P(C.c_double)),
        ("pin_row", C.c_int32), ("pin_value", C.c_double),
        ("cell_nslot", C.c_int32),
        ("cell_slots", _P(C.c_int32)),
        ("cell_flags", _P(C.c_uint32)),
        ("ninst", C.c_int32),
        ("inst_par", _P(HFParams)),
        ("cell_off", _P(C.c_int32)),
        ("facet_off", _P(C.c_int32) * 3),
        ("inst_pin", _P(C.c_int32)),
        ("inst_pin_value", _P(C.c_double)),
    ]


class HFOptions(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("poisson", C.c_int32),
        ("poisson_rtol", C.c_double), ("poisson_atol", C.c_double),
        ("poisson_maxit", C.c_int32), ("device", C.c_int32), ("precond", C.c_int32),
        ("eager", C.c_int32), ("tuning", C.c_int32),
    ]


class HFStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int64), ("last_iters", C.c_int32), ("last_outer", C.c_int32),
        ("last_residual", C.c_double), ("total_iters", C.c_int64),
        ("kernel_launches", C.c_int64), ("device_bytes", C.c_double),
    ]


_PARAM_NAMES = [n for n, _ in HFParams._fields_]
# parameters that programs written before they existed do not carry
_PARAM_DEFAULTS = {"tempdiscrtype": 0, "pad_": 0, "L2_fene": 0.0, "lambda_fene": 0.0, "E_fene": 0.0,
                   "ve_discrtype": 0, "pad2_": 0, "alpha_gptt": 1.0, "beta_gptt": 1.0, "gamma_gptt": 1.0}
_INT_PARAMS = ("dim", "flowtype", "projtype", "convecdiscrtype", "secondconvecdiscrtype", "ve_model",
               "ve_convecdiscrtype", "kernel", "tempdiscrtype", "pad_", "ve_discrtype", "pad2_")


def _np_from(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class Program:
    """A flattened step program with numpy storage (see module docstring)."""

    par: Dict[str, float]
    ncell: int
    nfacet: list
    delta: np.ndarray                     # (ndelta, dim) float64
    row_tmpl: np.ndarray                  # int32, per general row
    row_base: np.ndarray                  # int32, per general row
    row_rhs: np.ndarray                   # float64, per general row
    tmpl_ptr: np.ndarray                  # int64, ntmpl + 1
    tmpl_col: np.ndarray                  # int32
    tmpl_w: np.ndarray                    # float64
    vel_slots: list                       # per dim: (nslot, nfacet) int32
    vel_flags: list                       # per dim: (nfacet,) uint32
    vel_delta: list                       # per dim: (nfacet,) uint16
    div_slots: np.ndarray                 # (2*dim, ncell) int32
    cell_delta: np.ndarray                # (ncell,) uint16
    p_ptr: np.ndarray
    p_col: np.ndarray
    p_val: np.ndarray
    p_brhs: np.ndarray
    pin_row: int
    pin_value: float
    cell_slots: Optional[np.ndarray] = None   # (nslot, ncell) int32
    cell_flags: Optional[np.ndarray] = None
    # batches (see include/higflow_b200.h): per-instance parameters and offsets
    inst_par: Optional[list] = None
    cell_off: Optional[np.ndarray] = None
    facet_off: Optional[list] = None
    inst_pin: Optional[np.ndarray] = None
    inst_pin_value: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def ninst(self) -> int:
        return 0 if self.inst_par is None else len(self.inst_par)

    @property
    def dim(self) -> int:
        return int(self.par["dim"])

    @property
    def viscoelastic(self) -> bool:
        return int(self.par["flowtype"]) == VISCOELASTIC

    # ------------------------------------------------------------------
    @classmethod
    def from_c(cls, p: HFProgram) -> "Program":
        par = {n: getattr(p.par, n) for n in _PARAM_NAMES}
        dim = par["dim"]
        ncell = p.ncell
        nf = [p.nfacet[d] for d in range(3)]
        ns = p.vel_nslot
        vel_slots, vel_flags, vel_delta = [], [], []
        for d in range(dim):
            vel_slots.append(_np_from(p.vel_slots[d], ns * nf[d], np.int32).reshape(ns, nf[d]))
            vel_flags.append(_np_from(p.vel_flags[d], nf[d], np.uint32))
            vel_delta.append(_np_from(p.vel_delta[d], nf[d], np.uint16))
        cell_slots = cell_flags = None
        if p.cell_nslot:
            cell_slots = _np_from(p.cell_slots, p.cell_nslot * ncell, np.int32).reshape(p.cell_nslot, ncell)
            cell_flags = _np_from(p.cell_flags, ncell, np.uint32)
        return cls(
            par=par, ncell=ncell, nfacet=nf,
            delta=_np_from(p.delta, p.ndelta * dim, np.float64).reshape(p.ndelta, dim),
            row_tmpl=_np_from(p.row_tmpl, p.nrows, np.int32),
            row_base=_np_from(p.row_base, p.nrows, np.int32),
            row_rhs=_np_from(p.row_rhs, p.nrows, np.float64),
            tmpl_ptr=_np_from(p.tmpl_ptr, p.ntmpl + 1, np.int64),
            tmpl_col=_np_from(p.tmpl_col, p.nnz, np.int32),
            tmpl_w=_np_from(p.tmpl_w, p.nnz, np.float64),
            vel_slots=vel_slots, vel_flags=vel_flags, vel_delta=vel_delta,
            div_slots=_np_from(p.div_slots, 2 * dim * ncell, np.int32).reshape(2 * dim, ncell),
            cell_delta=_np_from(p.cell_delta, ncell, np.uint16),
            p_ptr=_np_from(p.p_ptr, ncell + 1, np.int64),
            p_col=_np_from(p.p_col, p.pnnz, np.int32),
            p_val=_np_from(p.p_val, p.pnnz, np.float64),
            p_brhs=_np_from(p.p_brhs, ncell, np.float64),
            pin_row=p.pin_row, pin_value=p.pin_value,
            cell_slots=cell_slots, cell_flags=cell_flags,
        )

    def to_c(self) -> HFProgram:
        """C view of this program; valid while this object is alive."""
        keep = []

        def a(x, dtype, ctype):
            x = np.ascontiguousarray(x, dtype=dtype)
            if x.size == 0:
                x = np.zeros(1, dtype=dtype)
            keep.append(x)
            return _ptr(x, ctype)

        p = HFProgram()
        for n in _PARAM_NAMES:
            setattr(p.par, n, self.par.get(n, _PARAM_DEFAULTS.get(n, 0)))
        p.ncell = self.ncell
        for d in range(3):
            p.nfacet[d] = self.nfacet[d] if d < self.dim else 0
        p.ndelta = self.delta.shape[0]
        p.delta = a(self.delta.ravel(), np.float64, C.c_double)
        p.nrows = self.row_rhs.size
        p.row_tmpl = a(self.row_tmpl, np.int32, C.c_int32)
        p.row_base = a(self.row_base, np.int32, C.c_int32)
        p.row_rhs = a(self.row_rhs, np.float64, C.c_double)
        p.ntmpl = self.tmpl_ptr.size - 1
        p.nnz = self.tmpl_col.size
        p.tmpl_ptr = a(self.tmpl_ptr, np.int64, C.c_int64)
        p.tmpl_col = a(self.tmpl_col, np.int32, C.c_int32)
        p.tmpl_w = a(self.tmpl_w, np.float64, C.c_double)
        p.vel_nslot = self.vel_slots[0].shape[0]
        for d in range(self.dim):
            p.vel_slots[d] = a(self.vel_slots[d].ravel(), np.int32, C.c_int32)
            p.vel_flags[d] = a(self.vel_flags[d], np.uint32, C.c_uint32)
            p.vel_delta[d] = a(self.vel_delta[d], np.uint16, C.c_uint16)
        p.div_slots = a(self.div_slots.ravel(), np.int32, C.c_int32)
        p.cell_delta = a(self.cell_delta, np.uint16, C.c_uint16)
        p.pnnz = self.p_col.size
        p.p_ptr = a(self.p_ptr, np.int64, C.c_int64)
        p.p_col = a(self.p_col, np.int32, C.c_int32)
        p.p_val = a(self.p_val, np.float64, C.c_double)
        p.p_brhs = a(self.p_brhs, np.float64, C.c_double)
        p.pin_row = self.pin_row
        p.pin_value = self.pin_value
        if self.cell_slots is not None:
            p.cell_nslot = self.cell_slots.shape[0]
            p.cell_slots = a(self.cell_slots.ravel(), np.int32, C.c_int32)
            p.cell_flags = a(self.cell_flags, np.uint32, C.c_uint32)
        else:
            p.cell_nslot = 0
        if self.inst_par is not None:
            n = len(self.inst_par)
            pars = (HFParams * n)()
            for i, ip in enumerate(self.inst_par):
                for nm in _PARAM_NAMES:
                    setattr(pars[i], nm, ip.get(nm, _PARAM_DEFAULTS.get(nm, 0)))
            keep.append(pars)
            p.ninst = n
            p.inst_par = C.cast(pars, C.POINTER(HFParams))
            p.cell_off = a(self.cell_off, np.int32, C.c_int32)
            for d in range(self.dim):
                p.facet_off[d] = a(self.facet_off[d], np.int32, C.c_int32)
            p.inst_pin = a(self.inst_pin, np.int32, C.c_int32)
            p.inst_pin_value = a(self.inst_pin_value, np.float64, C.c_double)
        else:
            p.ninst = 0
        self._keep = keep
        return p

    # ------------------------------------------------------------------
    @staticmethod
    def concatenate(progs) -> "Program":
        """One batch program holding independent cases side by side."""
        progs = list(progs)
        p0 = progs[0]
        D = p0.dim
        ve = p0.viscoelastic
        for q in progs:
            if q.dim != D or q.viscoelastic != ve or q.ninst:
                raise ValueError("batch members must share dim and flow type and not be batches")
        ni = len(progs)
        co = np.zeros(ni + 1, dtype=np.int64)
        fo = [np.zeros(ni + 1, dtype=np.int64) for _ in range(D)]
        for i, q in enumerate(progs):
            co[i + 1] = co[i] + q.ncell
            for d in range(D):
                fo[d][i + 1] = fo[d][i] + q.nfacet[d]
        if co[-1] > np.iinfo(np.int32).max or any(f[-1] > np.iinfo(np.int32).max for f in fo):
            raise ValueError("batch too large for int32 ids")

        def goff(i, g):
            return int(co[i]) if g < 0 else int(fo[g][i])

        # distinct deltas across the batch
        dtab, dmap = [], {}
        delta_remap = []
        for q in progs:
            m = np.empty(q.delta.shape[0], dtype=np.int64)
            for k, row in enumerate(q.delta):
                key = tuple(row.tolist())
                if key not in dmap:
                    dmap[key] = len(dtab)
                    dtab.append(row)
                m[k] = dmap[key]
            delta_remap.append(m)
        if len(dtab) > 65535:
            raise ValueError("too many distinct cell sizes in the batch")

        row_tmpl, row_base, row_rhs = [], [], []
        tptr, tcol, tw = [np.zeros(1, dtype=np.int64)], [], []
        nrow = ntm = nnz = 0
        vel = [[] for _ in range(D)]
        div, cells = [], []

        for i, q in enumerate(progs):
            # slot arrays of this instance with the field grid each slot reads
            arrays = []   # (output array, grid per slot row)
            for d in range(D):
                s = q.vel_slots[d].astype(np.int64)
                arrays.append((s, [vel_slot_grid(D, d, k) for k in range(s.shape[0])]))
            arrays.append((q.div_slots.astype(np.int64), [k // 2 for k in range(q.div_slots.shape[0])]))
            if ve:
                arrays.append((q.cell_slots.astype(np.int64), [cell_slot_grid(D, k) for k in range(q.cell_slots.shape[0])]))
            # rows keep their order; a row read through slots of two different field
            # grids (possible when recorded rows were merged by content) gets a copy
            # per extra grid
            nr = q.row_rhs.size
            grid_of = np.full(nr, -9, dtype=np.int64)
            extra = {}   # (row, grid) -> new index of the copy
            for a, gs in arrays:
                for k in range(len(gs)):
                    r = -a[k][a[k] < 0] - 1
                    g = gs[k]
                    unset = grid_of[r] == -9
                    grid_of[r[unset]] = g
                    clash = np.unique(r[grid_of[r] != g])
                    for rr in clash.tolist():
                        extra.setdefault((rr, g), None)
            base_off = np.array([goff(i, int(g)) if g != -9 else 0 for g in range(-1, D)], dtype=np.int64)
            gidx = np.where(grid_of == -9, -1, grid_of) + 1
            row_tmpl.append(q.row_tmpl.astype(np.int64) + ntm)
            row_base.append(q.row_base.astype(np.int64) + base_off[gidx] * (grid_of != -9))
            row_rhs.append(q.row_rhs)
            first_new = nrow
            nrow += nr
            for key in list(extra):
                rr, g = key
                extra[key] = nrow
                row_tmpl.append(np.array([int(q.row_tmpl[rr]) + ntm]))
                row_base.append(np.array([int(q.row_base[rr]) + goff(i, g)]))
                row_rhs.append(np.array([q.row_rhs[rr]]))
                nrow += 1
            for a, gs in arrays:
                for k in range(len(gs)):
                    row = a[k]
                    g = gs[k]
                    gen = row < 0
                    r = -row[gen] - 1
                    new = r + first_new
                    if extra:
                        for j in np.nonzero(grid_of[r] != g)[0].tolist():
                            new[j] = extra[(int(r[j]), g)]
                    row[gen] = -(new + 1)
                    row[~gen] += goff(i, g)
            for d in range(D):
                vel[d].append(arrays[d][0].astype(np.int32))
            div.append(arrays[D][0].astype(np.int32))
            if ve:
                cells.append(arrays[D + 1][0].astype(np.int32))
            tptr.append(q.tmpl_ptr[1:] + nnz)
            tcol.append(q.tmpl_col)
            tw.append(q.tmpl_w)
            ntm += q.tmpl_ptr.size - 1
            nnz += q.tmpl_col.size

        p_ptr = [np.zeros(1, dtype=np.int64)]
        p_col, p_val, p_brhs = [], [], []
        pn = 0
        for i, q in enumerate(progs):
            p_ptr.append(q.p_ptr[1:] + pn)
            p_col.append(q.p_col.astype(np.int64) + co[i])
            p_val.append(q.p_val)
            p_brhs.append(q.p_brhs)
            pn += q.p_col.size
        par = dict(p0.par)
        return Program(
            par=par, ncell=int(co[-1]), nfacet=[int(f[-1]) for f in fo] + [0] * (3 - D),
            delta=np.array(dtab, dtype=np.float64).reshape(-1, D),
            row_tmpl=np.concatenate(row_tmpl).astype(np.int32) if row_tmpl else np.zeros(0, np.int32),
            row_base=np.concatenate(row_base).astype(np.int32) if row_base else np.zeros(0, np.int32),
            row_rhs=np.concatenate(row_rhs).astype(np.float64) if row_rhs else np.zeros(0),
            tmpl_ptr=np.concatenate(tptr),
            tmpl_col=np.concatenate(tcol).astype(np.int32), tmpl_w=np.concatenate(tw),
            vel_slots=[np.concatenate(v, axis=1) for v in vel],
            vel_flags=[np.concatenate([q.vel_flags[d] for q in progs]) for d in range(D)],
            vel_delta=[np.concatenate([delta_remap[i][q.vel_delta[d]] for i, q in enumerate(progs)]).astype(np.uint16)
                       for d in range(D)],
            div_slots=np.concatenate(div, axis=1),
            cell_delta=np.concatenate([delta_remap[i][q.cell_delta] for i, q in enumerate(progs)]).astype(np.uint16),
            p_ptr=np.concatenate(p_ptr), p_col=np.concatenate(p_col).astype(np.int32),
            p_val=np.concatenate(p_val), p_brhs=np.concatenate(p_brhs),
            pin_row=-1, pin_value=0.0,
            cell_slots=np.concatenate(cells, axis=1) if ve else None,
            cell_flags=np.concatenate([q.cell_flags for q in progs]) if ve else None,
            inst_par=[dict(q.par) for q in progs],
            cell_off=co.astype(np.int32), facet_off=[f.astype(np.int32) for f in fo],
            inst_pin=np.array([(q.pin_row + int(co[i])) if q.pin_row >= 0 else -1 for i, q in enumerate(progs)],
                              dtype=np.int32),
            inst_pin_value=np.array([q.pin_value for q in progs], dtype=np.float64),
        )

    # ------------------------------------------------------------------
    def save(self, path: str, compress: bool = True) -> None:
        arrs = dict(
            par_keys=np.array(_PARAM_NAMES),
            par_vals=np.array([float(self.par.get(n, _PARAM_DEFAULTS.get(n, 0))) for n in _PARAM_NAMES]),
            ncell=np.int64(self.ncell), nfacet=np.array(self.nfacet, dtype=np.int64),
            delta=self.delta, row_tmpl=self.row_tmpl, row_base=self.row_base, row_rhs=self.row_rhs,
            tmpl_ptr=self.tmpl_ptr, tmpl_col=self.tmpl_col, tmpl_w=self.tmpl_w, div_slots=self.div_slots, cell_delta=self.cell_delta,
            p_ptr=self.p_ptr, p_col=self.p_col, p_val=self.p_val, p_brhs=self.p_brhs,
            pin=np.array([self.pin_row], dtype=np.int64), pin_value=np.float64(self.pin_value),
        )
        for d in range(self.dim):
            arrs[f"vel_slots{d}"] = self.vel_slots[d]
            arrs[f"vel_flags{d}"] = self.vel_flags[d]
            arrs[f"vel_delta{d}"] = self.vel_delta[d]
        if self.cell_slots is not None:
            arrs["cell_slots"] = self.cell_slots
            arrs["cell_flags"] = self.cell_flags
        (np.savez_compressed if compress else np.savez)(path, **arrs)

    @classmethod
    def load(cls, path: str) -> "Program":
        z = np.load(path)
        par = {}
        for k, v in zip(z["par_keys"], z["par_vals"]):
            k = str(k)
            par[k] = int(v) if k in _INT_PARAMS else float(v)
        for k, v in _PARAM_DEFAULTS.items():
            par.setdefault(k, v)
        dim = par["dim"]
        return cls(
            par=par, ncell=int(z["ncell"]), nfacet=[int(x) for x in z["nfacet"]],
            delta=z["delta"], row_tmpl=z["row_tmpl"], row_base=z["row_base"], row_rhs=z["row_rhs"],
            tmpl_ptr=z["tmpl_ptr"], tmpl_col=z["tmpl_col"], tmpl_w=z["tmpl_w"],
            vel_slots=[z[f"vel_slots{d}"] for d in range(dim)],
            vel_flags=[z[f"vel_flags{d}"] for d in range(dim)],
            vel_delta=[z[f"vel_delta{d}"] for d in range(dim)],
            div_slots=z["div_slots"], cell_delta=z["cell_delta"],
            p_ptr=z["p_ptr"], p_col=z["p_col"], p_val=z["p_val"], p_brhs=z["p_brhs"],
            pin_row=int(z["pin"][0]), pin_value=float(z["pin_value"]),
            cell_slots=z["cell_slots"] if "cell_slots" in z else None,
            cell_flags=z["cell_flags"] if "cell_flags" in z else None,
        )

    # ------------------------------------------------------------------
    def nbytes(self) -> int:
        n = 0
        for v in self.__dict__.values():
            if isinstance(v, np.ndarray):
                n += v.nbytes
            elif isinstance(v, list):
                n += sum(x.nbytes for x in v if isinstance(x, np.ndarray))
        return n

    def field_size(self, fid: int, comp: int = 0) -> int:
        if fid in (FIELD_U, FIELD_USTAR, FIELD_FU):
            return int(self.nfacet[comp])
        return int(self.ncell)

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
NON_INCREMENTAL, INCREMENTAL = 0, 1
CENTRAL, FIRST_ORDER, SECOND_ORDER = 0, 1, 2
MCU, CUBISTA, QUICK = 0, 1, 2
OLDROYD_B, GIESEKUS, LPTT = 0, 1, 2
CELL_CENTRAL, CELL_CUBISTA = 0, 1
KERNEL_IDENTITY, KERNEL_LOG, KERNEL_SQRT = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
POISSON_AUTO, POISSON_CG, POISSON_BICGSTAB = 0, 1, 2

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


class HFParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("flowtype", C.c_int32), ("projtype", C.c_int32),
        ("convecdiscrtype", C.c_int32), ("secondconvecdiscrtype", C.c_int32),
        ("ve_model", C.c_int32), ("ve_convecdiscrtype", C.c_int32), ("kernel", C.c_int32),
        ("Re", C.c_double), ("dt", C.c_double),
        ("De", C.c_double), ("beta", C.c_double), ("kernel_tol", C.c_double),
        ("alpha", C.c_double), ("epsilon", C.c_double), ("xi", C.c_double),
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
    ]


class HFOptions(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("poisson", C.c_int32),
        ("poisson_rtol", C.c_double), ("poisson_atol", C.c_double),
        ("poisson_maxit", C.c_int32), ("device", C.c_int32),
    ]


class HFStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int64), ("last_iters", C.c_int32), ("last_outer", C.c_int32),
        ("last_residual", C.c_double), ("total_iters", C.c_int64),
        ("kernel_launches", C.c_int64), ("device_bytes", C.c_double),
    ]


_PARAM_NAMES = [n for n, _ in HFParams._fields_]


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
    _keep: list = field(default_factory=list, repr=False)

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
            setattr(p.par, n, self.par[n])
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
        self._keep = keep
        return p

    # ------------------------------------------------------------------
    def save(self, path: str) -> None:
        arrs = dict(
            par_keys=np.array(_PARAM_NAMES), par_vals=np.array([float(self.par[n]) for n in _PARAM_NAMES]),
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
        np.savez_compressed(path, **arrs)

    @classmethod
    def load(cls, path: str) -> "Program":
        z = np.load(path)
        par = {}
        for k, v in zip(z["par_keys"], z["par_vals"]):
            k = str(k)
            par[k] = int(v) if k in ("dim", "flowtype", "projtype", "convecdiscrtype",
                                     "secondconvecdiscrtype", "ve_model",
                                     "ve_convecdiscrtype", "kernel") else float(v)
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

"""ctypes wrapper of the CPU restatement (oracle/restate/hf_restate.c).

Test infrastructure: runs the restated HigFlow step over a flattened program
(``higflow_b200.program.Program``) on the host, in FP64.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict

import numpy as np

from higflow_b200 import program as hp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libhf_restate.so")

_lib = None

_D = C.POINTER(C.c_double)


class Fields(C.Structure):
    _fields_ = [("u", _D * 3), ("us", _D * 3), ("p", _D), ("dp", _D), ("F", _D), ("FU", _D * 3),
                ("K", _D * 9), ("S", _D * 9), ("Du", _D * 9)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"restatement library missing: {LIB} (run make -C oracle restate)")
        L = C.CDLL(LIB)
        L.hfr_step.argtypes = [C.POINTER(hp.HFProgram), C.POINTER(Fields), C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.hfr_velocity.argtypes = [C.POINTER(hp.HFProgram), C.POINTER(Fields)]
        L.hfr_pressure.argtypes = [C.POINTER(hp.HFProgram), C.POINTER(Fields), C.c_double, C.POINTER(C.c_int)]
        L.hfr_final.argtypes = [C.POINTER(hp.HFProgram), C.POINTER(Fields)]
        L.hfr_ve_cell.argtypes = [C.POINTER(hp.HFProgram), C.POINTER(Fields)]
        L.hfr_divergence_rhs.argtypes = [C.POINTER(hp.HFProgram), C.POINTER(Fields), _D]
        L.hfr_cfl.argtypes = [C.POINTER(hp.HFProgram), C.POINTER(Fields)]
        L.hfr_cfl.restype = C.c_double
        L.hfr_mittag_leffler.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _D]
        L.hfr_mittag_leffler.restype = None
        _lib = L
    return _lib


def available() -> bool:
    return os.path.exists(LIB)


def mittag_leffler(alpha: float, beta: float, z, fi: int = 6) -> np.ndarray:
    """The restated E_{alpha,beta} (hf_restate.c, ml_eval) at every point of z."""
    zc = np.asarray(z, dtype=np.complex128)
    out = np.empty(zc.shape, dtype=np.complex128)
    r = (C.c_double * 2)()
    for i, v in np.ndenumerate(zc):
        lib().hfr_mittag_leffler(alpha, beta, v.real, v.imag, fi, r)
        out[i] = complex(r[0], r[1])
    return out


class State:
    """Host field storage in the engine's numbering, stepped by the restatement."""

    def __init__(self, prog: hp.Program):
        self.prog = prog
        self.cprog = prog.to_c()
        D = prog.dim
        nc = prog.ncell
        self.a: Dict[str, np.ndarray] = {}
        for d in range(D):
            self.a[f"u{d}"] = np.zeros(prog.nfacet[d])
            self.a[f"us{d}"] = np.zeros(prog.nfacet[d])
            self.a[f"FU{d}"] = np.zeros(prog.nfacet[d])
        for k in ("p", "dp", "F"):
            self.a[k] = np.zeros(nc)
        if prog.viscoelastic:
            for i in range(D * D):
                self.a[f"K{i}"] = np.zeros(nc)
                self.a[f"S{i}"] = np.zeros(nc)
                self.a[f"Du{i}"] = np.zeros(nc)
        self._bind()

    def _bind(self):
        f = Fields()
        p = lambda k: self.a[k].ctypes.data_as(_D)
        D = self.prog.dim
        for d in range(D):
            f.u[d] = p(f"u{d}")
            f.us[d] = p(f"us{d}")
            f.FU[d] = p(f"FU{d}")
        f.p, f.dp, f.F = p("p"), p("dp"), p("F")
        if self.prog.viscoelastic:
            for i in range(D * D):
                f.K[i], f.S[i], f.Du[i] = p(f"K{i}"), p(f"S{i}"), p(f"Du{i}")
        self.f = f

    def key(self, fid: int, comp: int = 0) -> str:
        return {hp.FIELD_U: f"u{comp}", hp.FIELD_USTAR: f"us{comp}", hp.FIELD_P: "p",
                hp.FIELD_DP: "dp", hp.FIELD_F: "F", hp.FIELD_FU: f"FU{comp}",
                hp.FIELD_KERNEL: f"K{comp}", hp.FIELD_S: f"S{comp}", hp.FIELD_DU: f"Du{comp}"}[fid]

    def set(self, fid: int, comp: int, v: np.ndarray) -> None:
        self.a[self.key(fid, comp)][:] = v

    def get(self, fid: int, comp: int = 0) -> np.ndarray:
        return self.a[self.key(fid, comp)].copy()

    def step(self, n: int = 1, rtol: float = 1e-13) -> int:
        it = C.c_int()
        rc = lib().hfr_step(C.byref(self.cprog), C.byref(self.f), n, rtol, C.byref(it))
        if rc != 0:
            raise RuntimeError(f"restatement step failed: {rc}")
        return it.value

    def velocity(self):
        lib().hfr_velocity(C.byref(self.cprog), C.byref(self.f))

    def pressure(self, rtol: float = 1e-13) -> int:
        it = C.c_int()
        rc = lib().hfr_pressure(C.byref(self.cprog), C.byref(self.f), rtol, C.byref(it))
        if rc != 0:
            raise RuntimeError(f"restatement pressure failed: {rc}")
        return it.value

    def final(self):
        lib().hfr_final(C.byref(self.cprog), C.byref(self.f))

    def ve_cell(self):
        lib().hfr_ve_cell(C.byref(self.cprog), C.byref(self.f))

    def divergence_rhs(self) -> np.ndarray:
        b = np.zeros(self.prog.ncell)
        lib().hfr_divergence_rhs(C.byref(self.cprog), C.byref(self.f), b.ctypes.data_as(_D))
        return b

    def cfl(self) -> float:
        """CFL number of the current velocity (higflow_compute_CFL)."""
        return lib().hfr_cfl(C.byref(self.cprog), C.byref(self.f))

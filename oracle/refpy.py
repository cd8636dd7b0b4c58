"""ctypes wrapper of the oracle harness (test infrastructure only).

Loads ``oracle/_ref/libhigflow_ref{2,3}d.so`` — the reference HigFlow C sources
built in place with single-rank shims (``oracle/Makefile``) — and drives the
reference's own time step, field storage and the HigFlow-side flattener.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
arm use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import tempfile
from typing import Dict, Optional, Sequence

import numpy as np

from higflow_b200 import program as hp
from higflow_b200.host import CaseSpec, HostParams, cavity, channel  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_libs: Dict[int, C.CDLL] = {}


RefParams = HostParams


def available(dim: int = 2) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libhigflow_ref{dim}d.so"))


def lib(dim: int) -> C.CDLL:
    if dim not in _libs:
        path = os.path.join(REF_DIR, f"libhigflow_ref{dim}d.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
        L = C.CDLL(path, mode=C.RTLD_LOCAL)
        L.hfref_create.argtypes = [C.c_char_p, C.POINTER(RefParams), C.POINTER(C.c_void_p)]
        L.hfref_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.hfref_get_field.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.c_int64]
        L.hfref_set_field.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.c_int64]
        L.hfref_centers.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
        L.hfref_step.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
        L.hfref_step_phased.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
        L.hfref_solver_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.hfref_time.argtypes = [C.c_void_p]
        L.hfref_time.restype = C.c_double
        L.hfref_flatten.argtypes = [C.c_void_p, C.POINTER(C.POINTER(hp.HFProgram))]
        L.hfref_program_free.argtypes = [C.POINTER(hp.HFProgram)]
        L.hfref_flatten_error.restype = C.c_char_p
        L.hfref_destroy.argtypes = [C.c_void_p]
        L.hfref_set_quiet.argtypes = [C.c_int]
        L.hfref_last_system.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.hfref_last_system_copy.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int),
                                             C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.hfref_ns.argtypes = [C.c_void_p]
        L.hfref_ns.restype = C.c_void_p
        L.hfref_dt.argtypes = [C.c_void_p]
        L.hfref_dt.restype = C.c_double
        L.hfref_set_dt.argtypes = [C.c_void_p, C.c_double]
        L.hfref_set_dt.restype = None
        L.hfref_cfl.argtypes = [C.c_void_p]
        L.hfref_cfl.restype = C.c_double
        L.hfref_adjust_timestep.argtypes = [C.c_void_p]
        L.hfref_adjust_timestep.restype = None
        L.hf_adjust_timestep.argtypes = [C.c_void_p]
        # the drop-in binding linked into the same library (product code under test)
        L.hf_attach.argtypes = [C.c_void_p, C.POINTER(hp.HFOptions)]
        L.hf_step.argtypes = [C.c_void_p]
        L.hf_sync_to_host.argtypes = [C.c_void_p]
        L.hf_sync_to_device.argtypes = [C.c_void_p]
        L.hf_detach.argtypes = [C.c_void_p]
        L.hf_detach.restype = None
        L.hf_last_error.restype = C.c_char_p
        _libs[dim] = L
    return _libs[dim]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class _Numc(C.Structure):
    _fields_ = [("real", C.c_double), ("imag", C.c_double)]


def mlfv(alpha: float, beta: float, z: complex, fi: int = 6) -> complex:
    """The reference's own Mittag-Leffler evaluation (hig-flow-mittag-leffler.c:117),
    from the 2D build."""
    L = lib(2)
    if not getattr(L, "_mlfv_set", False):
        L.mlfv.argtypes = [C.c_double, C.c_double, _Numc, C.c_int]
        L.mlfv.restype = _Numc
        L._mlfv_set = True
    r = L.mlfv(alpha, beta, _Numc(z.real, z.imag), fi)
    return complex(r.real, r.imag)


class RefCase:
    """One reference HigFlow case built from text inputs in a temp directory."""

    def __init__(self, spec: "CaseSpec"):
        self.spec = spec
        self.dim = spec.dim
        self.L = lib(self.dim)
        self.tmp = tempfile.mkdtemp(prefix="hfref_")
        name = spec.write(self.tmp)
        p = spec.host_params()
        h = C.c_void_p()
        rc = self.L.hfref_create(name.encode(), C.byref(p), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"hfref_create failed: {rc}")
        self._p = p
        self.h = h
        nc = C.c_int32()
        nf = (C.c_int32 * 3)()
        self.L.hfref_sizes(h, C.byref(nc), nf)
        self.ncell = nc.value
        self.nfacet = [nf[d] for d in range(self.dim)]

    def close(self):
        if self.h:
            self.L.hfref_destroy(self.h)
            self.h = None
        if self.tmp and os.path.isdir(self.tmp):
            shutil.rmtree(self.tmp, ignore_errors=True)
            self.tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def size(self, fid: int, comp: int = 0) -> int:
        if fid in (hp.FIELD_U, hp.FIELD_USTAR, hp.FIELD_FU):
            return self.nfacet[comp]
        return self.ncell

    def get(self, fid: int, comp: int = 0) -> np.ndarray:
        out = np.empty(self.size(fid, comp), dtype=np.float64)
        if self.L.hfref_get_field(self.h, fid, comp, _dp(out), out.size) != 0:
            raise ValueError("bad field")
        return out

    def set(self, fid: int, comp: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        if self.L.hfref_set_field(self.h, fid, comp, _dp(v), v.size) != 0:
            raise ValueError("bad field")

    def centers(self, facet_dim: int = -1) -> np.ndarray:
        n = self.ncell if facet_dim < 0 else self.nfacet[facet_dim]
        out = np.empty(n * self.dim, dtype=np.float64)
        self.L.hfref_centers(self.h, facet_dim, _dp(out))
        return out.reshape(n, self.dim)

    def step(self, n: int = 1) -> float:
        s = C.c_double()
        self.L.hfref_step(self.h, n, C.byref(s))
        return s.value

    def step_phased(self, n: int = 1) -> np.ndarray:
        t = np.zeros(5, dtype=np.float64)
        self.L.hfref_step_phased(self.h, n, _dp(t))
        return t

    def solver_stats(self):
        it = C.c_int32()
        res = C.c_double()
        self.L.hfref_solver_stats(self.h, C.byref(it), C.byref(res))
        return it.value, res.value

    def last_system(self):
        n = C.c_int()
        nnz = C.c_int()
        if self.L.hfref_last_system(C.byref(n), C.byref(nnz)) != 0:
            return None
        ptr = np.empty(n.value + 1, dtype=np.int32)
        col = np.empty(nnz.value, dtype=np.int32)
        val = np.empty(nnz.value, dtype=np.float64)
        b = np.empty(n.value, dtype=np.float64)
        self.L.hfref_last_system_copy(ptr.ctypes.data_as(C.POINTER(C.c_int)),
                                      col.ctypes.data_as(C.POINTER(C.c_int)), _dp(val), _dp(b))
        return ptr, col, val, b

    def flatten(self) -> hp.Program:
        pp = C.POINTER(hp.HFProgram)()
        rc = self.L.hfref_flatten(self.h, C.byref(pp))
        if rc != 0:
            raise RuntimeError(f"hf_flatten failed: {rc}: {self.L.hfref_flatten_error().decode()}")
        try:
            return hp.Program.from_c(pp.contents)
        finally:
            self.L.hfref_program_free(pp)

    @property
    def t(self) -> float:
        return self.L.hfref_time(self.h)

    @property
    def dt(self) -> float:
        return self.L.hfref_dt(self.h)

    @dt.setter
    def dt(self, value: float) -> None:
        self.L.hfref_set_dt(self.h, float(value))

    def cfl(self) -> float:
        """The reference's own CFL number of the current velocity."""
        return self.L.hfref_cfl(self.h)

    def adjust_timestep(self) -> None:
        """The reference's own adaptive time step (sets its dt)."""
        self.L.hfref_adjust_timestep(self.h)

    @property
    def ns(self) -> int:
        """The case's higflow_solver pointer (for the drop-in binding)."""
        return self.L.hfref_ns(self.h)

    def fields(self, names: Optional[Sequence[str]] = None) -> Dict[str, np.ndarray]:
        out = {}
        for d in range(self.dim):
            out[f"u{d}"] = self.get(hp.FIELD_U, d)
        out["p"] = self.get(hp.FIELD_P)
        if self.spec.flowtype == hp.VISCOELASTIC:
            for i in range(self.dim):
                for j in range(self.dim):
                    out[f"K{i}{j}"] = self.get(hp.FIELD_KERNEL, i * self.dim + j)
        return out


# case descriptions are the drop-in host's (higflow_b200/host.py)
__all__ = ["CaseSpec", "cavity", "channel", "RefCase", "available", "mlfv"]

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

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
MAXBC = 16

_libs: Dict[int, C.CDLL] = {}


class RefParams(C.Structure):
    _fields_ = [
        ("flowtype", C.c_int32), ("projtype", C.c_int32), ("convecdiscrtype", C.c_int32),
        ("secondconvecdiscrtype", C.c_int32), ("ve_model", C.c_int32),
        ("ve_convecdiscrtype", C.c_int32), ("kernel", C.c_int32), ("nbc", C.c_int32),
        ("Re", C.c_double), ("dt", C.c_double), ("t0", C.c_double),
        ("De", C.c_double), ("beta", C.c_double), ("kernel_tol", C.c_double),
        ("alpha", C.c_double), ("epsilon", C.c_double), ("xi", C.c_double),
        ("bc_u", (C.c_double * 3) * MAXBC), ("bc_upar", (C.c_double * 3) * MAXBC),
        ("bc_tdim", C.c_int32 * MAXBC), ("bc_c", C.c_double * MAXBC), ("bc_h", C.c_double * MAXBC),
        ("bc_p", C.c_double * MAXBC),
        ("k_init", (C.c_double * 3) * 3),
        ("tempdiscrtype", C.c_int32), ("pad_", C.c_int32),
        ("L2_fene", C.c_double), ("lambda_fene", C.c_double), ("E_fene", C.c_double),
        ("ve_discrtype", C.c_int32), ("pad2_", C.c_int32),
        ("alpha_gptt", C.c_double), ("beta_gptt", C.c_double),
    ]


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
        p = spec.ref_params()
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


# ----------------------------------------------------------------------
# case descriptions (text inputs in the reference's legacy formats)
# ----------------------------------------------------------------------
class CaseSpec:
    """A box domain with per-face boundary conditions, in the reference's
    legacy .domain/.bc text formats (hig-flow-ic.c:11-56, hig-flow-bc.c:572-614)
    and its .amr format (higtree-io.c:269-293)."""

    def __init__(self, dim: int, n: Sequence[int], lo: Sequence[float], hi: Sequence[float],
                 faces: Sequence[dict], **par):
        self.dim = dim
        self.n = list(n)
        self.lo = list(lo)
        self.hi = list(hi)
        self.faces = list(faces)   # per face: dict(axis, side, p='N'|'D', u='D'|'N', uval=[..], upar=.., p_val=)
        self.flowtype = par.get("flowtype", hp.NEWTONIAN)
        self.par = dict(par)
        self.refine: list = par.get("refine", [])   # extra levels: list of (delta, [(init, size)])

    def _amr(self, lo, hi, n, levels=()) -> str:
        s = " ".join(f"{lo[d]!r} {hi[d]!r}" for d in range(self.dim)) + "\n"
        s += f"{1 + len(levels)}\n"
        delta = [(hi[d] - lo[d]) / n[d] if n[d] > 0 else 0.0 for d in range(self.dim)]
        s += " ".join(repr(x) for x in delta) + " 1\n"
        s += " ".join("0" for _ in range(self.dim)) + " " + " ".join(str(x) for x in n) + "\n"
        for (ldelta, patches) in levels:
            s += " ".join(repr(x) for x in ldelta) + f" {len(patches)}\n"
            for (init, size) in patches:
                s += " ".join(str(x) for x in init) + " " + " ".join(str(x) for x in size) + "\n"
        return s

    def write(self, d: str) -> str:
        name = os.path.join(d, "case")
        with open(os.path.join(d, "dom0.amr"), "w") as f:
            f.write(self._amr(self.lo, self.hi, self.n, self.refine))
        with open(name + ".domain", "w") as f:
            f.write("1\n" + os.path.join(d, "dom0.amr") + "\n")
        lines = [str(len(self.faces))]
        for b, face in enumerate(self.faces):
            ax, side = face["axis"], face["side"]
            lo = list(self.lo)
            hi = list(self.hi)
            n = list(self.n)
            if side == 0:
                hi[ax] = lo[ax]
            else:
                lo[ax] = hi[ax]
            n[ax] = 1
            nb = [n[k] if k != ax else 1 for k in range(self.dim)]
            # degenerate axis: delta 0 (as in higflow/example2d_Newt/amrs/bc/*.amr)
            s = " ".join(f"{lo[k]!r} {hi[k]!r}" for k in range(self.dim)) + "\n1\n"
            delta = [0.0 if k == ax else (hi[k] - lo[k]) / nb[k] for k in range(self.dim)]
            s += " ".join(repr(x) for x in delta) + " 1\n"
            s += " ".join("0" for _ in range(self.dim)) + " " + " ".join(str(x) for x in nb) + "\n"
            path = os.path.join(d, f"bc{b}.amr")
            with open(path, "w") as f:
                f.write(s)
            ptype = 0 if face.get("p", "N") == "D" else 1
            lines.append(str(b))
            lines.append(path)
            lines.append(f"{ptype} 0")
            utype = 0 if face.get("u", "D") == "D" else 1
            for _ in range(self.dim):
                lines.append(f"{utype} 0")
        with open(name + ".bc", "w") as f:
            f.write("\n".join(lines) + "\n")
        return name

    def ref_params(self) -> RefParams:
        p = RefParams()
        g = self.par.get
        p.flowtype = self.flowtype
        p.projtype = g("projtype", hp.INCREMENTAL)
        p.convecdiscrtype = g("convecdiscrtype", hp.SECOND_ORDER)
        p.secondconvecdiscrtype = g("secondconvecdiscrtype", hp.CUBISTA)
        p.ve_model = g("ve_model", hp.OLDROYD_B)
        p.ve_convecdiscrtype = g("ve_convecdiscrtype", hp.CELL_CUBISTA)
        p.kernel = g("kernel", hp.KERNEL_LOG)
        p.nbc = len(self.faces)
        p.Re = g("Re", 100.0)
        p.dt = g("dt", 1e-4)
        p.t0 = g("t0", 0.0)
        p.De = g("De", 1.0)
        p.beta = g("beta", 1.0 / 9.0)
        p.kernel_tol = g("kernel_tol", 1e-2)
        p.alpha = g("alpha", 0.2)
        p.epsilon = g("epsilon", 0.25)
        p.xi = g("xi", 0.0)
        p.tempdiscrtype = g("tempdiscrtype", hp.EXPLICIT_EULER)
        p.L2_fene = g("L2_fene", 100.0)
        p.lambda_fene = g("lambda_fene", 1.0)
        p.E_fene = g("E_fene", 0.0)
        p.ve_discrtype = g("ve_discrtype", hp.VE_EXPLICIT)
        p.alpha_gptt = g("alpha_gptt", 1.0)
        p.beta_gptt = g("beta_gptt", 1.0)
        for b, face in enumerate(self.faces):
            for d, v in enumerate(face.get("uval", [0.0] * self.dim)):
                p.bc_u[b][d] = v
            for d, v in enumerate(face.get("upar", [0.0] * self.dim)):
                p.bc_upar[b][d] = v
            p.bc_tdim[b] = face.get("tdim", 0)
            p.bc_c[b] = face.get("c", 0.0)
            p.bc_h[b] = face.get("h", 1.0)
            p.bc_p[b] = face.get("p_val", 0.0)
        kin = g("k_init", None)
        if kin is None:
            # kernel of A = I: log -> 0, identity/sqrt -> I
            ident = p.kernel != hp.KERNEL_LOG
            for i in range(3):
                for j in range(3):
                    p.k_init[i][j] = 1.0 if (ident and i == j) else 0.0
        else:
            for i in range(3):
                for j in range(3):
                    p.k_init[i][j] = kin[i][j]
        return p


def cavity(dim: int = 2, n: int = 16, lid: float = 1.0, **par) -> CaseSpec:
    """Lid-driven cavity on the unit square/cube: no-slip walls, lid velocity
    u_0 = ``lid`` on the top face (y = 1 in 2D, z = 1 in 3D), Neumann pressure
    everywhere (so the pressure is pinned, hig-flow-bc.c:597-602)."""
    faces = []
    top = dim - 1
    for ax in range(dim):
        for side in (0, 1):
            uval = [0.0] * dim
            if ax == top and side == 1:
                uval[0] = lid
            faces.append(dict(axis=ax, side=side, p="N", u="D", uval=uval))
    return CaseSpec(dim, [n] * dim, [0.0] * dim, [1.0] * dim, faces, **par)


def channel(nx: int = 32, ny: int = 8, length: float = 8.0, half: float = 1.0, umax: float = 1.5,
            **par) -> CaseSpec:
    """2D channel [0,L] x [-h,h]: parabolic inflow umax*(1-(y/h)^2) at x = 0,
    no-slip walls, Dirichlet pressure / Neumann velocity outflow at x = L
    (the shipped higflow/example2d_Newt channel)."""
    faces = [
        dict(axis=0, side=0, p="N", u="D", uval=[0.0, 0.0], upar=[umax, 0.0], tdim=1, c=0.0, h=half),
        dict(axis=0, side=1, p="D", u="N", uval=[0.0, 0.0]),
        dict(axis=1, side=0, p="N", u="D", uval=[0.0, 0.0]),
        dict(axis=1, side=1, p="N", u="D", uval=[0.0, 0.0]),
    ]
    return CaseSpec(2, [nx, ny], [0.0, -half], [length, half], faces, **par)

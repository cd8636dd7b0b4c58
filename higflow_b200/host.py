"""HigFlow host of the drop-in, from Python: case descriptions and program recording.

A case is a box domain with per-face boundary conditions, written as the
reference's legacy text inputs (``.amr`` meshes, higtree-io.c:269-293; the
``.domain`` / ``.bc`` lists, hig-flow-ic.c:11-56, hig-flow-bc.c:572-614).  The
host library ``higflow_b200/lib/libhigflow_host{2,3}d.so`` (built by
``higflow_b200/host/Makefile`` from the HigFlow sources) builds the case the way
a HigFlow main program does and records its step program with the drop-in's
flattener, so every stencil id, weight and boundary term the GPU engine runs is
HigTree's own.  ``record_many`` records independent cases in parallel
processes (HigTree's stencil code is not reentrant, so one case per process at
a time).
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import shutil
import tempfile
import time
from typing import List, Optional, Sequence

import numpy as np

from . import program as hp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
MAXBC = 16

_libs = {}


class HostParams(C.Structure):
    """hfh_params (higflow_b200/host/hf_host.h)."""
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
        ("src_t", C.c_double),
    ]


def lib_path(dim: int) -> str:
    return os.path.join(LIB_DIR, f"libhigflow_host{dim}d.so")


def available(dim: int = 2) -> bool:
    return os.path.exists(lib_path(dim))


def lib(dim: int) -> C.CDLL:
    if dim not in _libs:
        path = lib_path(dim)
        if not os.path.exists(path):
            raise FileNotFoundError(f"HigFlow host library missing: {path} (make -C higflow_b200/host)")
        L = C.CDLL(path, mode=C.RTLD_LOCAL)
        L.hfh_record.argtypes = [C.c_char_p, C.POINTER(HostParams), C.POINTER(C.POINTER(hp.HFProgram))]
        L.hfh_program_free.argtypes = [C.POINTER(hp.HFProgram)]
        L.hfh_error.restype = C.c_char_p
        L.hfh_set_quiet.argtypes = [C.c_int]
        _libs[dim] = L
    return _libs[dim]


def record(spec: "CaseSpec") -> hp.Program:
    """The step program of one case, recorded by the host (HigTree's stencils)."""
    L = lib(spec.dim)
    tmp = tempfile.mkdtemp(prefix="hfh_")
    try:
        name = spec.write(tmp)
        p = spec.host_params()
        pp = C.POINTER(hp.HFProgram)()
        rc = L.hfh_record(name.encode(), C.byref(p), C.byref(pp))
        if rc != 0:
            raise RuntimeError(f"hfh_record failed ({rc}): {L.hfh_error().decode(errors='replace')}")
        try:
            return hp.Program.from_c(pp.contents)
        finally:
            L.hfh_program_free(pp)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# Physical parameters that enter no stencil: two cases that differ only in
# these record the same program up to its parameter block (tested against
# separate recordings in tests/test_host.py), so one recording serves both.
_PHYSICAL = ("Re", "dt", "t0", "De", "beta", "kernel_tol", "alpha", "epsilon", "xi", "L2_fene", "lambda_fene",
             "E_fene", "alpha_gptt", "beta_gptt")


_libm = None


def _tgamma(x: float) -> float:
    global _libm
    if _libm is None:
        import ctypes.util
        _libm = C.CDLL(ctypes.util.find_library("m"))
        _libm.tgamma.argtypes = [C.c_double]
        _libm.tgamma.restype = C.c_double
    return float(_libm.tgamma(x))


def with_parameters(prog: hp.Program, spec: "CaseSpec") -> hp.Program:
    """``prog`` (recorded for a case of the same geometry and controllers)
    with the physical parameters of ``spec``; arrays are shared."""
    p = spec.host_params()
    par = dict(prog.par)
    par["Re"], par["dt"] = float(p.Re), float(p.dt)
    # the flattener records the viscoelastic parameters of viscoelastic cases
    # only, with Gamma(beta_gptt) by the C library's tgamma (Python's
    # math.gamma can differ from it in the last bit)
    if int(par["flowtype"]) == hp.VISCOELASTIC:
        for k in _PHYSICAL:
            if k in par and k not in ("Re", "dt"):
                par[k] = float(getattr(p, k))
        par["gamma_gptt"] = _tgamma(par["beta_gptt"])
    out = hp.Program(**{k: v for k, v in prog.__dict__.items() if k != "_keep"})
    out.par = par
    return out


def _cache_dir() -> str:
    return os.environ.get("HF_PROGRAM_CACHE", os.path.join(tempfile.gettempdir(), "higflow_b200_programs"))


def _record_to_file(args):
    spec, path = args
    if not os.path.exists(path):
        prog = record(spec)
        tmp = path + f".{os.getpid()}.npz"
        prog.save(tmp, compress=False)
        os.replace(tmp, path)
    return path


def record_many(specs: Sequence["CaseSpec"], procs: Optional[int] = None, cache: bool = True) -> List[hp.Program]:
    """Programs of independent cases, recorded by ``procs`` host processes
    (default: every core) and kept in an on-disk cache keyed by the case's
    inputs (``HF_PROGRAM_CACHE``, default under the temp directory).  The pool
    is started with ``spawn``, so it may be used after CUDA is initialised."""
    import multiprocessing as mp
    d = _cache_dir()
    os.makedirs(d, exist_ok=True)
    # one recording per geometry (mesh, boundaries, controllers)
    groups = {}
    for sp in specs:
        groups.setdefault(sp.geometry_key(), sp)
    jobs = [(sp, os.path.join(d, k + ".npz")) for k, sp in groups.items()]
    todo = [j for j in jobs if not (cache and os.path.exists(j[1]))]
    # largest cases first, so the pool's tail is short
    todo.sort(key=lambda j: -j[0].cells())
    if todo:
        n = min(procs or os.cpu_count() or 1, len(todo))
        if n == 1:
            for j in todo:
                _record_to_file(j)
        else:
            with mp.get_context("spawn").Pool(n) as pool:
                for _ in pool.imap_unordered(_record_to_file, todo, chunksize=1):
                    pass
    loaded = {k: hp.Program.load(os.path.join(d, k + ".npz")) for k in groups}
    if not cache:
        for _, path in jobs:
            os.remove(path)
    return [with_parameters(loaded[sp.geometry_key()], sp) for sp in specs]


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

    def cells(self) -> int:
        """Leaf cells of the first level (a size for scheduling)."""
        return int(np.prod(self.n))

    def geometry_key(self) -> str:
        """A digest of what the recorded stencils depend on: mesh, boundaries and
        controllers, not the physical parameters (``_PHYSICAL``)."""
        p = self.host_params()
        for k in _PHYSICAL:
            setattr(p, k, 0.0)
        h = hashlib.sha256()
        h.update(repr((self.dim, self.n, self.lo, self.hi, self.faces, self.refine)).encode())
        h.update(bytes(p))
        return h.hexdigest()[:32]

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

    def trees(self):
        """(lo, hi, cells per axis, refinement levels) of each tree."""
        return [(self.lo, self.hi, self.n, self.refine)]

    def face_box(self, face):
        """(lo, hi, cells per axis, normal axis) of a boundary: a face of the box."""
        ax, side = face["axis"], face["side"]
        lo = list(self.lo)
        hi = list(self.hi)
        if side == 0:
            hi[ax] = lo[ax]
        else:
            lo[ax] = hi[ax]
        return lo, hi, [self.n[k] if k != ax else 1 for k in range(self.dim)], ax

    def write(self, d: str) -> str:
        name = os.path.join(d, "case")
        paths = []
        for t, (lo, hi, n, refine) in enumerate(self.trees()):
            paths.append(os.path.join(d, f"dom{t}.amr"))
            with open(paths[-1], "w") as f:
                f.write(self._amr(lo, hi, n, refine))
        with open(name + ".domain", "w") as f:
            f.write(f"{len(paths)}\n" + "".join(p + "\n" for p in paths))
        lines = [str(len(self.faces))]
        for b, face in enumerate(self.faces):
            lo, hi, nb, ax = self.face_box(face)
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

    def host_params(self) -> HostParams:
        p = HostParams()
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
        p.src_t = g("src_t", 0.0)
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


class TreesSpec(CaseSpec):
    """A domain of several trees (boxes, each with its own refinement levels)
    and explicit boundary boxes: ``trees`` = [dict(lo, hi, n, refine=[...])],
    ``faces`` = [dict(lo, hi, n, axis, p, u, uval, upar, tdim, c, h, p_val)]
    with ``n`` the boundary's cells per axis (1 along its normal ``axis``)."""

    def __init__(self, dim: int, trees: Sequence[dict], faces: Sequence[dict], **par):
        t0 = trees[0]
        super().__init__(dim, t0["n"], t0["lo"], t0["hi"], faces, **par)
        self.tree_list = [dict(t) for t in trees]

    def trees(self):
        return [(t["lo"], t["hi"], t["n"], t.get("refine", [])) for t in self.tree_list]

    def face_box(self, face):
        return list(face["lo"]), list(face["hi"]), list(face["n"]), face["axis"]

    def cells(self) -> int:
        return int(sum(int(np.prod(t["n"])) for t in self.tree_list))

    def geometry_key(self) -> str:
        p = self.host_params()
        for k in _PHYSICAL:
            setattr(p, k, 0.0)
        h = hashlib.sha256()
        h.update(repr((self.dim, self.tree_list, self.faces)).encode())
        h.update(bytes(p))
        return h.hexdigest()[:32]


def contraction(per_unit: int = 32, band: float = 0.125, refine: bool = True, umax: float = 1.5, **par) -> TreesSpec:
    """The 2D 4:1 planar contraction of higflow/example2d_Newt_contraction (two
    trees: upstream [-16,0] x [-4,4], downstream [0,16] x [-1,1]; its eight
    boundaries), at ``per_unit`` cells per unit length, with a second level
    (half the cell size) on squares of side 2 ``band`` centred on the
    contraction corners (0, +-1) (``band`` = 1/16 of the downstream width
    2 by default).  Parabolic inflow umax (1 - (y/4)^2) (mean umax 2/3) at
    x = -16, no-slip walls, outflow at x = 16 (pressure Dirichlet 0,
    velocity Neumann)."""
    h = 1.0 / per_unit
    up = dict(lo=[-16.0, -4.0], hi=[0.0, 4.0], n=[16 * per_unit, 8 * per_unit])
    dn = dict(lo=[0.0, -1.0], hi=[16.0, 1.0], n=[16 * per_unit, 2 * per_unit])
    if refine:
        b = int(round(band * 2 * per_unit))      # band in level-2 cells
        # level-2 patches (init, size) in level-2 cell units of each tree
        up["refine"] = [([h / 2, h / 2], [((32 * per_unit - b, (3 * per_unit) * 2 - b), (b, 2 * b)),
                                          ((32 * per_unit - b, (5 * per_unit) * 2 - b), (b, 2 * b))])]
        dn["refine"] = [([h / 2, h / 2], [((0, 4 * per_unit - b), (b, b)), ((0, 0), (b, b))])]
    wall = dict(p="N", u="D", uval=[0.0, 0.0])
    faces = [
        dict(lo=[-16.0, -4.0], hi=[-16.0, 4.0], n=[1, 8 * per_unit], axis=0, p="N", u="D", uval=[0.0, 0.0],
             upar=[umax, 0.0], tdim=1, c=0.0, h=4.0),
        dict(lo=[-16.0, 4.0], hi=[0.0, 4.0], n=[16 * per_unit, 1], axis=1, **wall),
        dict(lo=[0.0, 1.0], hi=[0.0, 4.0], n=[1, 3 * per_unit], axis=0, **wall),
        dict(lo=[0.0, 1.0], hi=[16.0, 1.0], n=[16 * per_unit, 1], axis=1, **wall),
        dict(lo=[16.0, -1.0], hi=[16.0, 1.0], n=[1, 2 * per_unit], axis=0, p="D", u="N", uval=[0.0, 0.0]),
        dict(lo=[0.0, -1.0], hi=[16.0, -1.0], n=[16 * per_unit, 1], axis=1, **wall),
        dict(lo=[0.0, -4.0], hi=[0.0, -1.0], n=[1, 3 * per_unit], axis=0, **wall),
        dict(lo=[-16.0, -4.0], hi=[0.0, -4.0], n=[16 * per_unit, 1], axis=1, **wall),
    ]
    return TreesSpec(2, [up, dn], faces, **par)

"""Python binding of the B200 step engine (``libhigflow_b200.so``).

``Case`` wraps ``hf_case_*`` from ``include/higflow_b200.h``: it uploads a
flattened step program, holds the fields in HBM and advances whole HigFlow
time steps on the GPU.  There is no CPU path: if the CUDA library or a device
is missing, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import program as hp

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "lib", "libhigflow_b200.so")

_lib: Optional[C.CDLL] = None


class EngineError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"higflow_b200 error {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load the in-tree engine library (built by ``higflow_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise EngineError(-7, f"engine library not built: {LIBPATH}")
        L = C.CDLL(LIBPATH)
        P, V = C.POINTER, C.c_void_p
        L.hf_last_error.restype = C.c_char_p
        L.hf_case_create.argtypes = [P(hp.HFProgram), P(hp.HFOptions), P(V)]
        L.hf_case_set_field.argtypes = [V, C.c_int32, C.c_int32, P(C.c_double), C.c_int64]
        L.hf_case_get_field.argtypes = [V, C.c_int32, C.c_int32, P(C.c_double), C.c_int64]
        L.hf_case_step.argtypes = [V, C.c_int32]
        L.hf_case_step_async.argtypes = [V, C.c_int32]
        L.hf_case_launch_counts.argtypes = [V, P(C.c_int32), P(C.c_int32)]
        L.hf_case_instance_iters.argtypes = [V, P(C.c_int64), C.c_int32]
        L.hf_case_adjust_timestep.argtypes = [V, P(C.c_double), P(C.c_double), C.c_int32]
        L.hf_case_set_timestep.argtypes = [V, P(C.c_double), C.c_int32]
        L.hf_case_set_step_limits.argtypes = [V, P(C.c_int64), C.c_int32]
        L.hf_case_instance_failures.argtypes = [V, P(C.c_int32), C.c_int32]
        L.hf_case_launch_shapes.argtypes = [V, P(C.c_int32), C.c_int32]
        L.hf_case_stats.argtypes = [V, P(hp.HFStats)]
        L.hf_case_synchronize.argtypes = [V]
        L.hf_case_destroy.argtypes = [V]
        L.hf_case_destroy.restype = None
        L.hf_case_device_bytes.argtypes = [P(hp.HFProgram), P(hp.HFOptions), P(C.c_int64)]
        L.hf_case_stream.argtypes = [V, P(C.c_void_p)]
        L.hf_case_instances.argtypes = [V, P(C.c_int32)]
        L.hf_case_instance_result.argtypes = [V, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_int32),
                                              P(C.c_double)]
        L.hf_case_solver_info.argtypes = [V, P(C.c_int32), P(C.c_int32), P(C.c_int64), P(C.c_int64),
                                          P(C.c_int64), P(C.c_int64), C.c_int32]
        L.hf_case_profile.argtypes = [V, C.c_int32]
        L.hf_case_phase_times.argtypes = [V, P(C.c_double), P(C.c_int64), C.c_int32]
        L.hf_mittag_leffler.argtypes = [C.c_double, C.c_double, P(C.c_double), C.c_int64, C.c_int32, P(C.c_double)]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise EngineError(rc, lib().hf_last_error().decode(errors="replace"))


def options(precision: int = hp.PREC_FP64, poisson: int = hp.POISSON_AUTO, rtol: float = 1e-10,
            atol: float = 1e-10, maxit: int = 20000, device: int = 0,
            precond: int = hp.PRECOND_AUTO, eager: bool = False, tune: bool = True) -> hp.HFOptions:
    o = hp.HFOptions()
    o.precision, o.poisson = precision, poisson
    o.poisson_rtol, o.poisson_atol, o.poisson_maxit, o.device = rtol, atol, maxit, device
    o.precond = precond
    o.eager = int(bool(eager))
    o.tuning = 0 if tune else 1
    return o


class Case:
    """One HigFlow case resident on the GPU."""

    def __init__(self, prog: hp.Program, opts: Optional[hp.HFOptions] = None):
        self.prog = prog
        self._cprog = prog.to_c()
        self._opts = opts or options()
        h = C.c_void_p()
        _check(lib().hf_case_create(C.byref(self._cprog), C.byref(self._opts), C.byref(h)))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().hf_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, fid: int, comp: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        _check(lib().hf_case_set_field(self.h, fid, comp, v.ctypes.data_as(C.POINTER(C.c_double)), v.size))

    def get(self, fid: int, comp: int = 0) -> np.ndarray:
        out = np.empty(self.prog.field_size(fid, comp), dtype=np.float64)
        _check(lib().hf_case_get_field(self.h, fid, comp, out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out

    def step(self, n: int = 1, sync: bool = True) -> None:
        """Advance n steps; with sync=False they are only queued on the case
        stream and a failure surfaces at the next synchronize()."""
        _check((lib().hf_case_step if sync else lib().hf_case_step_async)(self.h, n))

    def instance_iters(self) -> np.ndarray:
        """Poisson iterations of every instance summed over all steps so far."""
        n = self.instances()
        out = np.zeros(n, dtype=np.int64)
        _check(lib().hf_case_instance_iters(self.h, out.ctypes.data_as(C.POINTER(C.c_int64)), n))
        return out

    def adjust_timestep(self):
        """Adaptive time step of every instance (higflow_adjust_timestep):
        returns (CFL numbers, new time steps), one per instance."""
        n = self.instances()
        cfl = np.zeros(n)
        dt = np.zeros(n)
        _check(lib().hf_case_adjust_timestep(self.h, cfl.ctypes.data_as(C.POINTER(C.c_double)),
                                             dt.ctypes.data_as(C.POINTER(C.c_double)), n))
        return cfl, dt

    def set_step_limits(self, steps) -> None:
        """Instance i takes steps[i] more steps, then stays as it is (< 0: no limit)."""
        a = np.ascontiguousarray(steps, dtype=np.int64)
        _check(lib().hf_case_set_step_limits(self.h, a.ctypes.data_as(C.POINTER(C.c_int64)), a.size))

    def instance_failures(self) -> np.ndarray:
        """Under step limits: each instance's first failed step's status (0: none)."""
        a = np.zeros(self.instances(), dtype=np.int32)
        _check(lib().hf_case_instance_failures(self.h, a.ctypes.data_as(C.POINTER(C.c_int32)), a.size))
        return a

    def set_timestep(self, dt) -> None:
        a = np.ascontiguousarray(np.atleast_1d(dt), dtype=np.float64)
        _check(lib().hf_case_set_timestep(self.h, a.ctypes.data_as(C.POINTER(C.c_double)), a.size))

    def launch_shapes(self):
        """Block sizes of the tuned kernels: (k_vrows, k_velocity, k_ve_cell)."""
        a = (C.c_int32 * 3)()
        _check(lib().hf_case_launch_shapes(self.h, a, 3))
        return tuple(a)

    def launch_counts(self):
        """(kernels per step outside the Poisson loop, kernels per loop body)."""
        a, b = C.c_int32(), C.c_int32()
        _check(lib().hf_case_launch_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def synchronize(self) -> None:
        _check(lib().hf_case_synchronize(self.h))

    def stats(self) -> hp.HFStats:
        s = hp.HFStats()
        _check(lib().hf_case_stats(self.h, C.byref(s)))
        return s

    def instances(self) -> int:
        n = C.c_int32()
        _check(lib().hf_case_instances(self.h, C.byref(n)))
        return n.value

    def instance_result(self, inst: int):
        """Last step's Poisson result of one instance: (iters, outer, status, residual)."""
        it, ou, st, res = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        _check(lib().hf_case_instance_result(self.h, inst, C.byref(it), C.byref(ou), C.byref(st), C.byref(res)))
        return it.value, ou.value, st.value, res.value

    def get_instance(self, fid: int, comp: int, inst: int) -> np.ndarray:
        """Field values of one instance of a batch program."""
        a = self.get(fid, comp)
        if self.prog.ninst == 0:
            return a
        off = self.prog.cell_off if fid not in (hp.FIELD_U, hp.FIELD_USTAR, hp.FIELD_FU) else self.prog.facet_off[comp]
        return a[off[inst]:off[inst + 1]]

    def stream(self) -> int:
        """Handle of the cudaStream_t all of this case's kernels run on."""
        p = C.c_void_p()
        _check(lib().hf_case_stream(self.h, C.byref(p)))
        return p.value or 0

    def profile(self, enable: bool = True) -> None:
        """Turn per-phase CUDA-event timing on/off (resets the counters)."""
        _check(lib().hf_case_profile(self.h, 1 if enable else 0))

    def solver_info(self):
        """{'method', 'levels': [(rows, nnz_A, nnz_P, nnz_R), ...]} of the Poisson solver."""
        m, nl = C.c_int32(), C.c_int32()
        k = 32
        rows, na, npp, nr = (C.c_int64 * k)(), (C.c_int64 * k)(), (C.c_int64 * k)(), (C.c_int64 * k)()
        _check(lib().hf_case_solver_info(self.h, C.byref(m), C.byref(nl), rows, na, npp, nr, k))
        method = {hp.PRECOND_AMG: "amg-cg", hp.PRECOND_JACOBI: "jacobi-cg", -1: "bicgstab"}[m.value]
        return {"method": method, "levels": [(rows[i], na[i], npp[i], nr[i]) for i in range(nl.value)]}

    PHASES = ("ve_cell", "velocity", "poisson_init", "poisson_iter", "final", "velocity_rows", "ve_cell_main")

    def phase_times(self):
        """{phase: (device ms, kernel launches)} accumulated since profile()."""
        n = len(self.PHASES)
        ms = (C.c_double * n)()
        la = (C.c_int64 * n)()
        _check(lib().hf_case_phase_times(self.h, ms, la, n))
        return {p: (ms[i], la[i]) for i, p in enumerate(self.PHASES)}


def mittag_leffler(alpha: float, beta: float, z, fi: int = 6) -> np.ndarray:
    """E_{alpha,beta}(z) on the GPU at every point of ``z`` (the evaluation the
    GPTT model takes; the reference's ``mlfv``, hig-flow-mittag-leffler.c:117).
    Returns a complex array of the shape of ``z``."""
    zc = np.ascontiguousarray(np.asarray(z, dtype=np.complex128))
    zi = zc.reshape(-1).view(np.float64)
    out = np.empty_like(zi)
    _check(lib().hf_mittag_leffler(alpha, beta, zi.ctypes.data_as(C.POINTER(C.c_double)), zc.size, fi,
                                   out.ctypes.data_as(C.POINTER(C.c_double))))
    return out.view(np.complex128).reshape(zc.shape)


def device_bytes(prog: hp.Program, opts: Optional[hp.HFOptions] = None) -> int:
    b = C.c_int64()
    cp = prog.to_c()
    o = opts or options()
    _check(lib().hf_case_device_bytes(C.byref(cp), C.byref(o), C.byref(b)))
    return b.value


# ---------------------------------------------------------------------------
# serving (include/higflow_b200.h, hf_server_*)
class HFServerOptions(C.Structure):
    _fields_ = [("hbm_budget_gb", C.c_double), ("max_active", C.c_int32), ("chunk_steps", C.c_int32),
                ("setup_threads", C.c_int32), ("device", C.c_int32)]


class HFFieldData(C.Structure):
    _fields_ = [("field", C.c_int32), ("comp", C.c_int32), ("data", C.POINTER(C.c_double)), ("n", C.c_int64)]


class HFServerCounts(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("queued", C.c_int64),
                ("active", C.c_int64), ("reserved_bytes", C.c_int64), ("cell_steps", C.c_int64),
                ("seconds", C.c_double)]


def _server_lib() -> C.CDLL:
    L = lib()
    if not hasattr(L, "_server_ready"):
        P, V = C.POINTER, C.c_void_p
        L.hf_server_create.argtypes = [P(HFServerOptions), P(V)]
        L.hf_server_submit.argtypes = [V, P(hp.HFProgram), P(hp.HFOptions), C.c_int32, P(HFFieldData), C.c_int32,
                                       P(C.c_int64)]
        L.hf_server_wait.argtypes = [V, C.c_int64, C.c_int32, P(C.c_int32), P(C.c_double), P(C.c_double)]
        L.hf_server_get_field.argtypes = [V, C.c_int64, C.c_int32, C.c_int32, P(C.c_double), C.c_int64]
        L.hf_server_release.argtypes = [V, C.c_int64]
        L.hf_server_stats.argtypes = [V, P(HFServerCounts)]
        L.hf_server_destroy.argtypes = [V]
        L.hf_server_destroy.restype = None
        L.hf_server_last_error.restype = C.c_char_p
        L._server_ready = True
    return L


def _scheck(rc: int) -> None:
    if rc != 0:
        raise EngineError(rc, _server_lib().hf_server_last_error().decode(errors="replace"))


class Server:
    """Continuous batching of independent cases on one GPU (hf_server_*)."""

    def __init__(self, budget_gb: float = 150.0, max_active: int = 64, chunk_steps: int = 16,
                 setup_threads: int = 8, device: int = 0):
        o = HFServerOptions(budget_gb, max_active, chunk_steps, setup_threads, device)
        self.h = C.c_void_p()
        _scheck(_server_lib().hf_server_create(C.byref(o), C.byref(self.h)))
        self._sizes = {}

    def submit(self, prog: hp.Program, opts: Optional[hp.HFOptions] = None, steps: int = 1,
               fields: Optional[dict] = None) -> int:
        """Queue a case; fields: {(field, comp): values}.  Returns its id."""
        cp = prog.to_c()
        fl = list((fields or {}).items())
        arr = (HFFieldData * max(len(fl), 1))()
        keep = []
        for k, ((fid, comp), v) in enumerate(fl):
            v = np.ascontiguousarray(v, dtype=np.float64)
            keep.append(v)
            arr[k] = HFFieldData(fid, comp, v.ctypes.data_as(C.POINTER(C.c_double)), v.size)
        rid = C.c_int64()
        o = opts or options()
        _scheck(_server_lib().hf_server_submit(self.h, C.byref(cp), C.byref(o), steps, arr, len(fl), C.byref(rid)))
        self._sizes[rid.value] = prog
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1):
        """(status, queue seconds, submit-to-done seconds); None while still running."""
        st, q, t = C.c_int32(), C.c_double(), C.c_double()
        rc = _server_lib().hf_server_wait(self.h, rid, timeout_ms, C.byref(st), C.byref(q), C.byref(t))
        if rc == -8:
            return None
        _scheck(rc)
        return st.value, q.value, t.value

    def get(self, rid: int, fid: int, comp: int = 0) -> np.ndarray:
        out = np.empty(self._sizes[rid].field_size(fid, comp), dtype=np.float64)
        _scheck(_server_lib().hf_server_get_field(self.h, rid, fid, comp,
                                                  out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out

    def release(self, rid: int) -> None:
        _scheck(_server_lib().hf_server_release(self.h, rid))
        self._sizes.pop(rid, None)

    def stats(self) -> HFServerCounts:
        s = HFServerCounts()
        _scheck(_server_lib().hf_server_stats(self.h, C.byref(s)))
        return s

    def close(self) -> None:
        if self.h:
            _server_lib().hf_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""hf_slv_solve_device_noalloc against the allocating hf_slv_* entry points.

The system is a seeded sparse, non-symmetric, diagonally dominant matrix (the
shape of a Poisson row set with convection-like asymmetry).  Both entry points
run the same Jacobi-preconditioned BiCGStab to rtol 1e-12; the solutions must
agree to 1e-10 relative L2, on two no-alloc calls in a row, and the no-alloc
solution must satisfy ||b - A x|| / ||b|| <= 1e-10 when the residual is
recomputed on the host (scipy).  Sizes: a small system and one at the entry
point's 65536-row limit.
"""
import ctypes as C

import numpy as np
import pytest

from higflow_b200 import engine

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _system(n, seed=7):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        cols = {i}
        for d in (1, 2, 37):
            for j in (i - d, i + d):
                if 0 <= j < n:
                    cols.add(j)
        cols = sorted(cols)
        off = {j: -rng.uniform(0.5, 1.5) for j in cols if j != i}
        diag = sum(abs(v) for v in off.values()) + rng.uniform(0.5, 1.0)
        rows.append([(j, diag if j == i else off[j]) for j in cols])
    ptr = np.zeros(n + 1, dtype=np.int32)
    for i, r in enumerate(rows):
        ptr[i + 1] = ptr[i] + len(r)
    col = np.array([j for r in rows for j, _ in r], dtype=np.int32)
    val = np.array([v for r in rows for _, v in r], dtype=np.float64)
    b = rng.standard_normal(n)
    x0 = rng.standard_normal(n) * 1e-3
    return ptr, col, val, b, x0


def _lib():
    L = engine.lib()
    L.hf_slv_create.argtypes = [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.hf_slv_set_Ai.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    L.hf_slv_set_bi.argtypes = [C.c_void_p, C.c_int32, C.c_double]
    L.hf_slv_set_x.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.hf_slv_assemble_matrix.argtypes = [C.c_void_p]
    L.hf_slv_set_tolerances.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32]
    L.hf_slv_solve.argtypes = [C.c_void_p]
    L.hf_slv_get_x.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.hf_slv_destroy.argtypes = [C.c_void_p]
    L.hf_slv_destroy.restype = None
    L.hf_slv_solve_device_noalloc.argtypes = [
        C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
        C.c_int32, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    return L


def _dbl(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _allocating_solve(L, ptr, col, val, b, x0):
    n = b.size
    s = C.c_void_p()
    assert L.hf_slv_create(0, n, C.byref(s)) == 0
    for i in range(n):
        j = np.ascontiguousarray(col[ptr[i]:ptr[i + 1]])
        v = np.ascontiguousarray(val[ptr[i]:ptr[i + 1]])
        assert L.hf_slv_set_Ai(s, i, j.size, j.ctypes.data_as(C.POINTER(C.c_int32)), _dbl(v)) == 0
        assert L.hf_slv_set_bi(s, i, float(b[i])) == 0
    x = x0.copy()
    assert L.hf_slv_set_x(s, _dbl(x)) == 0
    assert L.hf_slv_assemble_matrix(s) == 0
    assert L.hf_slv_set_tolerances(s, 1e-12, 1e-300, 100000) == 0
    assert L.hf_slv_solve(s) == 0, L.hf_last_error()
    assert L.hf_slv_get_x(s, _dbl(x)) == 0
    L.hf_slv_destroy(s)
    return x


def _host_residual(ptr, col, val, x, b):
    import scipy.sparse as sp
    A = sp.csr_matrix((val, col, ptr), shape=(b.size, b.size))
    return float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))


@pytest.mark.parametrize("n", [3000, 65536])
def test_no_alloc_solve_matches_allocating_solver_twice(n):
    import torch
    L = _lib()
    ptr, col, val, b, x0 = _system(n)
    want = _allocating_solve(L, ptr, col, val, b, x0)
    dev = torch.device("cuda:0")
    d_ptr = torch.from_numpy(ptr).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    stream = torch.cuda.Stream(device=dev)
    for call in range(2):
        d_x = torch.from_numpy(x0.copy()).to(dev)
        torch.cuda.synchronize(dev)
        it, res = C.c_int32(), C.c_double()
        rc = L.hf_slv_solve_device_noalloc(n, d_ptr.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), d_b.data_ptr(),
                                           d_x.data_ptr(), 1e-12, 1e-300, 100000, stream.cuda_stream,
                                           C.byref(it), C.byref(res))
        assert rc == 0, (call, L.hf_last_error())
        got = d_x.cpu().numpy()
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < TOL, (call, err)
        assert it.value > 0 and res.value <= 1e-11
        assert _host_residual(ptr, col, val, got, b) <= 1e-10, call


def test_no_alloc_rejects_oversize_system():
    L = _lib()
    it, res = C.c_int32(), C.c_double()
    # the size check comes before any device access: the pointers are not read
    rc = L.hf_slv_solve_device_noalloc(65537, 1, 1, 1, 1, 1, 1e-10, 1e-10, 10, None, C.byref(it), C.byref(res))
    assert rc == -1   # HF_ERR_INVALID
    assert b"exceeds the static scratch" in L.hf_last_error()

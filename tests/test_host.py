"""The HigFlow host of the drop-in (higflow_b200/host): program recording.

Every benchmark and served workload runs programs recorded by the host, i.e.
by HigTree's own stencil builder through the drop-in's flattener.  These tests
pin that path on the CPU: the host records exactly what the oracle build of the
reference records, one recording serves cases that differ only in physical
parameters, and the parallel recorder returns the same programs.
"""
import math

import numpy as np
import pytest

from higflow_b200 import host
from higflow_b200 import program as hp

pytestmark = pytest.mark.skipif(not host.available(2), reason="HigFlow host library not built")


def _arrays_equal(a: hp.Program, b: hp.Program):
    for k, v in a.__dict__.items():
        if k in ("_keep", "par"):
            continue
        w = getattr(b, k)
        if isinstance(v, np.ndarray):
            assert v.dtype == w.dtype and np.array_equal(v, w), k
        elif isinstance(v, list) and v and isinstance(v[0], np.ndarray):
            assert len(v) == len(w) and all(np.array_equal(x, y) for x, y in zip(v, w)), k
        else:
            assert v == w, k


def _giesekus(n, **kw):
    par = dict(Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GIESEKUS, kernel=hp.KERNEL_LOG, De=1.5,
               alpha=0.3, beta=0.1)
    par.update(kw)
    return host.cavity(2, n, **par)


def test_host_records_what_the_reference_records():
    from oracle import refpy
    if not refpy.available(2):
        pytest.skip("oracle build not present")
    for spec in (_giesekus(14), host.channel(24, 6, Re=1.0, dt=1e-4)):
        a = host.record(spec)
        c = refpy.RefCase(spec)
        b = c.flatten()
        c.close()
        _arrays_equal(a, b)
        assert a.par == b.par


def test_one_recording_serves_every_physical_parameter_set():
    a = _giesekus(12, Re=1.0, dt=1e-4, De=0.5, alpha=0.1, beta=0.1)
    b = _giesekus(12, Re=2.5, dt=3e-5, De=1.7, alpha=0.45, beta=0.2, kernel_tol=1e-3)
    assert a.geometry_key() == b.geometry_key()
    ra, rb = host.record(a), host.record(b)
    _arrays_equal(ra, rb)
    moved = host.with_parameters(ra, b)
    _arrays_equal(moved, rb)
    assert moved.par == rb.par
    # geometry, boundary values and controllers are part of the key
    assert host.cavity(2, 12, lid=2.0).geometry_key() != host.cavity(2, 12).geometry_key()
    assert _giesekus(13).geometry_key() != a.geometry_key()
    assert _giesekus(12, kernel=hp.KERNEL_SQRT).geometry_key() != a.geometry_key()


def test_gptt_gamma_follows_the_parameters():
    a = _giesekus(10, ve_model=hp.GPTT, alpha_gptt=0.5, beta_gptt=1.0)
    b = _giesekus(10, ve_model=hp.GPTT, alpha_gptt=0.5, beta_gptt=1.3)
    moved = host.with_parameters(host.record(a), b)
    assert moved.par["gamma_gptt"] == pytest.approx(math.gamma(1.3), rel=1e-15)
    assert moved.par["gamma_gptt"] == host.record(b).par["gamma_gptt"]


def test_parallel_recorder_matches_single_recordings(tmp_path, monkeypatch):
    monkeypatch.setenv("HF_PROGRAM_CACHE", str(tmp_path))
    specs = [_giesekus(10), _giesekus(11, De=0.3), _giesekus(10, De=1.9), host.channel(16, 4, Re=1.0, dt=1e-4)]
    progs = host.record_many(specs, procs=2)
    assert len(list(tmp_path.glob("*.npz"))) == 3      # two specs share one geometry
    for sp, pr in zip(specs, progs):
        want = host.record(sp)
        _arrays_equal(pr, want)
        assert pr.par == want.par

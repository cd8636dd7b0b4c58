"""Host-side behaviour of the drop-in binding: configurations outside the GPU
path are refused at attach, before any device work, with HF_ERR_UNSUPPORTED
(the binding never falls back to the reference's CPU step)."""
import ctypes as C

import pytest

from higflow_b200 import program as hp

refpy = pytest.importorskip("oracle.refpy")


def test_attach_refuses_an_unsupported_model_without_a_gpu():
    if not refpy.available(2):
        pytest.skip("oracle build of the reference not present")
    # FENE-P (visc_model_type 4, hig-flow-kernel.h:301): not on the GPU path
    case = refpy.RefCase(refpy.cavity(2, 8, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.FENE_P))
    L = case.L
    assert L.hf_attach(case.ns, None) == -2   # HF_ERR_UNSUPPORTED
    assert b"FENE-P" in L.hfref_flatten_error()
    assert L.hf_step(case.ns) == -2            # stepping attaches first, and refuses the same way
    assert L.hf_sync_to_host(case.ns) == -1    # never attached
    case.close()


def test_attach_refuses_time_dependent_sources_without_a_gpu():
    """A case whose source callback depends on t (higflow_calculate_source_term
    evaluates it at ns->par.t every step, hig-flow-step.c:343-367) would run
    with frozen sources on the GPU path: refused at attach, before any device
    work.  The same case with a fixed source is not refused for that reason."""
    if not refpy.available(2):
        pytest.skip("oracle build of the reference not present")
    case = refpy.RefCase(refpy.cavity(2, 8, Re=10.0, dt=1e-3, src_t=2.5))
    L = case.L
    assert L.hf_attach(case.ns, None) == -2   # HF_ERR_UNSUPPORTED
    assert L.hf_sync_to_host(case.ns) == -1    # not attached
    case.close()

"""The step-level drop-in (hf_attach / hf_step / hf_sync_to_host / hf_detach,
higflow_b200/binding/hf_attach.c) driving the reference's own solver object.

Two instances of the same case are built by the reference harness; one is
stepped by the reference (higflow_solver_step[_viscoelastic]), the other is
attached to the GPU engine and stepped by hf_step, then synced back into its
own distributed properties.  The reference-side fields must agree to 1e-10
relative L2 (the plain-FP64 parity bar; the Poisson solves differ only in
their Krylov iterates, both to 1e-13)."""
import ctypes as C
import os

import numpy as np
import pytest

from higflow_b200 import engine
from higflow_b200 import program as hp

os.environ.setdefault("HF_ORACLE_RTOL", "1e-15")
refpy = pytest.importorskip("oracle.refpy")

pytestmark = pytest.mark.gpu

TOL = 1e-10

# Both copies start from the same seeded random u, p (and K) fields, as the
# golden fixtures do: from rest the pressure increments of the first steps are
# tiny next to the warm-start iterate, and both solvers stop at the rounding
# floor of that iterate rather than at the requested tolerance.
CASES = {
    "newtonian": lambda: refpy.cavity(2, 16, Re=100.0, dt=1e-3),
    "giesekus_log": lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GIESEKUS,
                                         kernel=hp.KERNEL_LOG, alpha=0.3, beta=0.1, De=0.5),
    # semi-implicit Euler velocity (the reference's own slvu solvers on its side)
    "oldroyd_sie": lambda: refpy.cavity(2, 12, Re=0.01, dt=1e-3, flowtype=hp.VISCOELASTIC, ve_model=hp.OLDROYD_B,
                                        kernel=hp.KERNEL_LOG, beta=1.0 / 9.0,
                                        tempdiscrtype=hp.SEMI_IMPLICIT_EULER),
    # GPTT (the Mittag-Leffler factor; gamma_gptt from the flattener's tgamma)
    "gptt_log": lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GPTT,
                                     kernel=hp.KERNEL_LOG, beta=1.0 / 9.0, De=0.5, epsilon=0.3, xi=0.1,
                                     alpha_gptt=0.8, beta_gptt=1.2),
    # semi-implicit BDF2 (two solves per direction)
    "newtonian_bdf2": lambda: refpy.cavity(2, 12, Re=0.1, dt=1e-3, tempdiscrtype=hp.SEMI_IMPLICIT_BDF2),
}


def _perturb(case, ve, seed=0):
    rng = np.random.default_rng(seed)
    for d in range(case.dim):
        case.set(hp.FIELD_U, d, 0.3 * rng.standard_normal(case.nfacet[d]))
    case.set(hp.FIELD_P, 0, 0.1 * rng.standard_normal(case.ncell))
    if ve:
        for i in range(case.dim):
            for j in range(i, case.dim):
                v = 0.2 * rng.standard_normal(case.ncell)
                case.set(hp.FIELD_KERNEL, i * case.dim + j, v)
                case.set(hp.FIELD_KERNEL, j * case.dim + i, v)


def _fields(case, ve):
    keys = [("u0", hp.FIELD_U, 0), ("u1", hp.FIELD_U, 1), ("p", hp.FIELD_P, 0)]
    if ve:
        keys += [(f"K{k}", hp.FIELD_KERNEL, k) for k in range(4)] + [(f"S{k}", hp.FIELD_S, k) for k in range(4)]
    return {name: case.get(fid, comp) for name, fid, comp in keys}


@pytest.mark.parametrize("name", sorted(CASES))
def test_hf_step_matches_reference_step(name):
    if not refpy.available(2):
        pytest.skip("oracle build of the reference not present")
    spec = CASES[name]()
    ve = spec.flowtype == hp.VISCOELASTIC
    steps = 4
    ref = refpy.RefCase(spec)
    gpu = refpy.RefCase(CASES[name]())
    _perturb(ref, ve)
    _perturb(gpu, ve)
    # HigTree caches interpolation stencils on first use and later steps read
    # the cached form, which is what the program records; walking the queries
    # once warms the reference copy's cache the same way (as the golden
    # fixtures are made)
    ref.flatten()
    ref.step(steps)
    L = gpu.L
    opts = engine.options(rtol=1e-13, atol=1e-300)
    assert L.hf_attach(gpu.ns, C.byref(opts)) == 0, L.hf_last_error()
    for _ in range(steps):
        assert L.hf_step(gpu.ns) == 0, L.hf_last_error()
    assert L.hf_sync_to_host(gpu.ns) == 0, L.hf_last_error()
    want, got = _fields(ref, ve), _fields(gpu, ve)
    for k in want:
        err = np.linalg.norm(got[k] - want[k]) / max(np.linalg.norm(want[k]), 1e-300)
        assert err < TOL, (name, k, err)
    # the reference solver object carries the engine's solve statistics
    it, res = gpu.solver_stats()
    assert it > 0 and res < 1e-11
    L.hf_detach(gpu.ns)
    ref.close()
    gpu.close()


def test_detach_leaves_the_gpu_fields_on_the_host():
    if not refpy.available(2):
        pytest.skip("oracle build of the reference not present")
    gpu = refpy.RefCase(CASES["newtonian"]())
    L = gpu.L
    assert L.hf_attach(gpu.ns, None) == 0, L.hf_last_error()
    assert L.hf_step(gpu.ns) == 0
    L.hf_detach(gpu.ns)          # syncs, then frees the engine case
    u = gpu.get(hp.FIELD_U, 0)
    assert np.abs(u).max() > 0.0  # the lid has started to drive the flow
    gpu.close()


def test_sync_to_device_after_a_host_side_restart():
    """A case that replaces its fields on the host between steps (as after
    higflow_load_properties) pushes them to the GPU with hf_sync_to_device;
    the GPU then steps from the new state exactly as the reference does."""
    if not refpy.available(2):
        pytest.skip("oracle build of the reference not present")
    ref = refpy.RefCase(CASES["giesekus_log"]())
    gpu = refpy.RefCase(CASES["giesekus_log"]())
    _perturb(ref, True)
    _perturb(gpu, True)
    ref.flatten()
    ref.step(2)
    L = gpu.L
    opts = engine.options(rtol=1e-13, atol=1e-300)
    assert L.hf_attach(gpu.ns, C.byref(opts)) == 0, L.hf_last_error()
    for _ in range(2):
        assert L.hf_step(gpu.ns) == 0, L.hf_last_error()
    # both copies load the same new u, p and K (a restart; the other fields
    # stay as the steps left them, so the GPU copy syncs them out first), then
    # step twice more
    assert L.hf_sync_to_host(gpu.ns) == 0, L.hf_last_error()
    _perturb(ref, True, seed=5)
    _perturb(gpu, True, seed=5)
    assert L.hf_sync_to_device(gpu.ns) == 0, L.hf_last_error()
    ref.step(2)
    for _ in range(2):
        assert L.hf_step(gpu.ns) == 0, L.hf_last_error()
    assert L.hf_sync_to_host(gpu.ns) == 0, L.hf_last_error()
    want, got = _fields(ref, True), _fields(gpu, True)
    for k in want:
        err = np.linalg.norm(got[k] - want[k]) / max(np.linalg.norm(want[k]), 1e-300)
        assert err < TOL, (k, err)
    L.hf_detach(gpu.ns)
    ref.close()
    gpu.close()


def test_adjust_timestep_through_the_binding_matches_the_reference():
    """hf_adjust_timestep (the target of -Wl,--wrap=higflow_adjust_timestep)
    sets ns->par.dt from the GPU state as the reference's own routine does
    from its host state."""
    if not refpy.available(2):
        pytest.skip("oracle build of the reference not present")
    ref = refpy.RefCase(CASES["newtonian"]())
    gpu = refpy.RefCase(CASES["newtonian"]())
    _perturb(ref, False)
    _perturb(gpu, False)
    ref.flatten()
    L = gpu.L
    opts = engine.options(rtol=1e-13, atol=1e-300)
    assert L.hf_attach(gpu.ns, C.byref(opts)) == 0, L.hf_last_error()
    ref.step(2)
    for _ in range(2):
        assert L.hf_step(gpu.ns) == 0, L.hf_last_error()
    ref.adjust_timestep()
    assert L.hf_adjust_timestep(gpu.ns) == 0, L.hf_last_error()
    assert abs(gpu.dt - ref.dt) <= 1e-10 * ref.dt, (gpu.dt, ref.dt)
    L.hf_detach(gpu.ns)
    ref.close()
    gpu.close()


def test_a_host_change_of_dt_reaches_the_gpu():
    """A case that sets ns->par.dt on the host between steps (a restart, or
    its own time-step control) syncs out, changes dt, and pushes the state
    back with hf_sync_to_device, which carries the new dt to the engine; the
    GPU then steps with it exactly as the reference does."""
    if not refpy.available(2):
        pytest.skip("oracle build of the reference not present")
    ref = refpy.RefCase(CASES["newtonian"]())
    gpu = refpy.RefCase(CASES["newtonian"]())
    _perturb(ref, False)
    _perturb(gpu, False)
    ref.flatten()
    L = gpu.L
    opts = engine.options(rtol=1e-13, atol=1e-300)
    assert L.hf_attach(gpu.ns, C.byref(opts)) == 0, L.hf_last_error()
    ref.step(2)
    for _ in range(2):
        assert L.hf_step(gpu.ns) == 0, L.hf_last_error()
    assert L.hf_sync_to_host(gpu.ns) == 0, L.hf_last_error()
    for c in (ref, gpu):
        c.dt = 0.6 * c.dt
    assert L.hf_sync_to_device(gpu.ns) == 0, L.hf_last_error()
    ref.step(3)
    for _ in range(3):
        assert L.hf_step(gpu.ns) == 0, L.hf_last_error()
    assert L.hf_sync_to_host(gpu.ns) == 0, L.hf_last_error()
    want, got = _fields(ref, False), _fields(gpu, False)
    for k in want:
        err = np.linalg.norm(got[k] - want[k]) / max(np.linalg.norm(want[k]), 1e-300)
        assert err < TOL, (k, err)
    L.hf_detach(gpu.ns)
    ref.close()
    gpu.close()

"""GPU parity of the B200 step engine against the oracle and the reference.

Every test goes through the C ABI (libhigflow_b200.so via higflow_b200.engine).
Tolerances: relative L2 1e-10 on velocity, pressure and kernel tensor after the
fixture's N steps (the plain-FP64 parity bar); the velocity stage is compared
bit for bit (same FP64 operation sequence, no FMA contraction).
"""
import numpy as np
import pytest

from higflow_b200 import engine
from higflow_b200 import program as hp
from oracle import restate
from tests.helpers import (ML_ALPHAS, ML_BETAS, ML_POINTS, compare, field_keys, golden_names, load_golden,
                           load_init)

pytestmark = pytest.mark.gpu

NAMES = golden_names()
TOL = 1e-10


def _opts(**kw):
    kw.setdefault("rtol", 1e-13)
    kw.setdefault("atol", 1e-300)
    return engine.options(**kw)


@pytest.mark.parametrize("name", NAMES)
def test_engine_matches_reference_after_n_steps(name):
    prog, data = load_golden(name)
    case = engine.Case(prog, _opts())
    load_init(case, prog, data)
    case.step(int(data["steps"]))
    keys = [k for k, _, _ in field_keys(prog) if k != "dp" and not k.startswith("S")]
    got = {k: case.get(fid, comp) for k, fid, comp in field_keys(prog)}
    err = compare(got, {k: data["ref_" + k] for k in keys}, keys)
    assert max(err.values()) < TOL, err
    case.close()


@pytest.mark.parametrize("name", NAMES)
def test_engine_matches_restatement(name):
    prog, data = load_golden(name)
    case = engine.Case(prog, _opts())
    st = restate.State(prog)
    load_init(case, prog, data)
    load_init(st, prog, data)
    n = int(data["steps"])
    case.step(n)
    st.step(n, rtol=1e-14)
    keys = [k for k, _, _ in field_keys(prog) if k != "dp"]
    got = {k: case.get(fid, comp) for k, fid, comp in field_keys(prog)}
    want = {k: st.get(fid, comp) for k, fid, comp in field_keys(prog)}
    err = compare(got, want, keys)
    assert max(err.values()) < TOL, err
    case.close()


@pytest.mark.parametrize("name", ["cav2d_cubista", "cav2d_quick", "cav2d_central", "cav3d_cubista", "chan2d_cubista"])
def test_velocity_stage_bit_exact(name):
    """One step: u* (the explicit velocity stage) is bit-identical to the
    oracle's, because both evaluate the same recorded rows in the reference's
    order with the same IEEE operations."""
    prog, data = load_golden(name)
    case = engine.Case(prog, _opts())
    st = restate.State(prog)
    load_init(case, prog, data)
    load_init(st, prog, data)
    case.step(1)
    st.velocity()
    for d in range(prog.dim):
        a = case.get(hp.FIELD_USTAR, d)
        b = st.get(hp.FIELD_USTAR, d)
        assert np.array_equal(a, b), (d, np.abs(a - b).max())
    case.close()


@pytest.mark.parametrize("name", ["cav2d_cubista", "cav3d_cubista", "ve2d_oldroyd_log"])
def test_amg_and_jacobi_preconditioners_agree(name):
    prog, data = load_golden(name)
    out = []
    for pc in (hp.PRECOND_AMG, hp.PRECOND_JACOBI):
        case = engine.Case(prog, _opts(precond=pc))
        load_init(case, prog, data)
        case.step(int(data["steps"]))
        out.append(case.get(hp.FIELD_P))
        case.close()
    assert np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[0]) < 1e-10


def test_amg_iteration_count_is_small():
    """On a 128x128 cavity the AMG-preconditioned CG converges in far fewer
    iterations than diagonal scaling."""
    from higflow_b200 import host
    prog = host.record(host.cavity(2, 128, Re=100.0, dt=1e-4))
    iters = {}
    for pc in (hp.PRECOND_AMG, hp.PRECOND_JACOBI):
        case = engine.Case(prog, engine.options(precond=pc))
        u = np.zeros(prog.nfacet[0])
        case.step(2)
        iters[pc] = case.stats().last_iters
        case.close()
    assert iters[hp.PRECOND_AMG] * 10 < iters[hp.PRECOND_JACOBI], iters


def test_bicgstab_path_matches_cg():
    """Both Poisson solvers against the reference's fields after the golden
    steps.  BiCGStab stops on its recursive residual, which drifts from the true
    one near 1e-13, so the two agree to ~1e-9 rather than to the CG's 1e-10."""
    name = "cav2d_cubista"
    prog, data = load_golden(name)
    steps = int(data["steps"])
    out = []
    for solver in (hp.POISSON_CG, hp.POISSON_BICGSTAB):
        case = engine.Case(prog, _opts(poisson=solver))
        load_init(case, prog, data)
        case.step(steps)
        got = {k: case.get(fid, comp) for k, fid, comp in field_keys(prog)}
        err = compare(got, {k: data["ref_" + k] for k, _, _ in field_keys(prog)}, ["u0", "u1", "p"])
        assert max(err.values()) < 1e-9, (solver, err)
        out.append(got["p"])
        case.close()
    assert np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[0]) < 1e-9


def test_invalid_program_rejected_on_host():
    prog, _ = load_golden("cav2d_cubista")
    bad = hp.Program.load(__import__("os").path.join(__import__("tests.helpers", fromlist=["GOLDEN"]).GOLDEN,
                                                       "cav2d_cubista.prog.npz"))
    bad.vel_slots[0] = bad.vel_slots[0].copy()
    bad.vel_slots[0][hp.V_PL, 0] = prog.ncell + 5   # direct index past the pressure field
    with pytest.raises(engine.EngineError) as e:
        engine.Case(bad)
    assert e.value.code == -1


def test_nan_is_reported():
    prog, data = load_golden("cav2d_cubista")
    case = engine.Case(prog, _opts())
    load_init(case, prog, data)
    u = data["init_u0"].copy()
    u[3] = np.nan
    case.set(hp.FIELD_U, 0, u)
    with pytest.raises(engine.EngineError) as e:
        case.step(1)
    assert e.value.code == -4
    case.close()


def test_solver_engine_known_answer():
    """higtree/atf-tests/test-solver-2d.c:9-49 through the solver-vtable engine:
    the 3x3 system solves to x = (1, 4, -2)."""
    import ctypes as C
    L = engine.lib()
    L.hf_slv_create.argtypes = [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.hf_slv_set_Ai.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    L.hf_slv_set_bi.argtypes = [C.c_void_p, C.c_int32, C.c_double]
    L.hf_slv_assemble_matrix.argtypes = [C.c_void_p]
    L.hf_slv_set_tolerances.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32]
    L.hf_slv_solve.argtypes = [C.c_void_p]
    L.hf_slv_get_x.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.hf_slv_destroy.argtypes = [C.c_void_p]
    L.hf_slv_destroy.restype = None
    m = [[-1.0, 3.0, 5.0], [3.0, -5.0, 7.0], [-1.0, 4.0, -10.0]]
    b = [1.0, -31.0, 35.0]
    s = C.c_void_p()
    assert L.hf_slv_create(0, 3, C.byref(s)) == 0
    j = (C.c_int32 * 3)(0, 1, 2)
    for i in range(3):
        assert L.hf_slv_set_Ai(s, i, 3, j, (C.c_double * 3)(*m[i])) == 0
        assert L.hf_slv_set_bi(s, i, b[i]) == 0
    assert L.hf_slv_assemble_matrix(s) == 0
    assert L.hf_slv_set_tolerances(s, 1e-8, 1e-8, 1000) == 0
    assert L.hf_slv_solve(s) == 0
    x = (C.c_double * 3)()
    assert L.hf_slv_get_x(s, x) == 0
    assert abs(x[0] - 1.0) < 1e-12 and abs(x[1] - 4.0) < 1e-12 and abs(x[2] + 2.0) < 1e-12
    L.hf_slv_destroy(s)


def test_semi_implicit_velocity_refused_in_a_batch():
    """The semi-implicit form solves each direction's velocity system on one
    instance; a batch of such programs is refused at create."""
    prog, _ = load_golden("sie2d_cubista")
    batch = hp.Program.concatenate([prog, prog])
    with pytest.raises(engine.EngineError) as e:
        engine.Case(batch, _opts())
    assert e.value.code == -2 and "semi-implicit" in str(e.value)   # HF_ERR_UNSUPPORTED


@pytest.mark.parametrize("name", ["sie2d_cubista", "bdf2_cav2d"])
def test_semi_implicit_velocity_iterates_and_counts_launches(name):
    """A semi-implicit step runs eagerly and its velocity solves' kernels are
    counted in the step statistics."""
    prog, data = load_golden(name)
    case = engine.Case(prog, _opts())
    load_init(case, prog, data)
    case.step(2)
    st = case.stats()
    assert st.steps == 2 and st.kernel_launches > 2 * 10
    case.close()


def _random_velocity(obj, prog, seed, amp=0.7):
    rng = np.random.default_rng(seed)
    for d in range(prog.dim):
        obj.set(hp.FIELD_U, d, amp * rng.standard_normal(prog.nfacet[d]))


@pytest.mark.parametrize("name", ["cav2d_cubista", "ve2d_oldroyd_log", "cav3d_cubista"])
def test_adaptive_timestep_matches_restatement(name):
    """hf_case_adjust_timestep: the CFL number of the device velocity against the
    restatement's (higflow_compute_CFL) and the reference's update of dt."""
    prog, _ = load_golden(name)
    case = engine.Case(prog, _opts())
    st = restate.State(prog)
    _random_velocity(case, prog, 1)
    _random_velocity(st, prog, 1)
    dt0 = prog.par["dt"]
    cfl, dt = case.adjust_timestep()
    want = st.cfl()
    assert abs(cfl[0] - want) <= 1e-13 * want, (cfl, want)
    assert abs(dt[0] - min(min(0.1 / (want + 1e-12), 1.1) * dt0, 32 * dt0)) <= 1e-15 * dt[0]
    case.close()


def test_adaptive_timestep_per_instance_in_a_batch():
    """Each instance of a batch adapts its own dt from its own CFL number, and
    the next step uses it: a batch member steps as a case created with the new dt."""
    names = ["cav2d_cubista", "cav2d_lid"]
    progs = [load_golden(n)[0] for n in names]
    batch = hp.Program.concatenate(progs)
    case = engine.Case(batch, _opts())
    alone = []
    for i, p in enumerate(progs):
        c = engine.Case(p, _opts())
        _random_velocity(c, p, 10 + i, 0.7 * (1 + 9 * i))   # the second one's CFL limits its step
        alone.append((c, c.adjust_timestep()))
    # the same velocity per instance in the batch
    for i, p in enumerate(progs):
        rng = np.random.default_rng(10 + i)
        for d in range(p.dim):
            u = case.get(hp.FIELD_U, d)
            off = batch.facet_off[d]
            u[off[i]:off[i + 1]] = 0.7 * (1 + 9 * i) * rng.standard_normal(p.nfacet[d])
            case.set(hp.FIELD_U, d, u)
    cfl, dt = case.adjust_timestep()
    for i, (c, (ca, dta)) in enumerate(alone):
        assert abs(cfl[i] - ca[0]) <= 1e-14 * ca[0] and abs(dt[i] - dta[0]) <= 1e-15 * dta[0], (i, cfl, ca)
    assert dt[0] != dt[1]
    # one step with the adapted dt, against a fresh case created with that dt
    p2 = hp.Program.load(__import__("os").path.join(__import__("tests.helpers", fromlist=["GOLDEN"]).GOLDEN,
                                                      names[0] + ".prog.npz"))
    p2.par["dt"] = float(dt[0])
    ref = engine.Case(p2, _opts())
    _random_velocity(ref, p2, 10)
    case.step(1)
    ref.step(1)
    u = case.get_instance(hp.FIELD_U, 0, 0)
    ur = ref.get(hp.FIELD_U, 0)
    assert np.linalg.norm(u - ur) <= TOL * np.linalg.norm(ur)
    for c, _ in alone:
        c.close()
    ref.close()
    case.close()


def test_adaptive_timestep_refused_for_semi_implicit():
    prog, _ = load_golden("sie2d_cubista")
    case = engine.Case(prog, _opts())
    with pytest.raises(engine.EngineError):
        case.adjust_timestep()
    case.close()


def _ml_series_region(a, az):
    """The region where the evaluation sums the power series (the same bounds
    as hf::mittag_leffler and the reference's mlfv)."""
    return (a < 1 and az <= 1) or (1 <= a < 2 and az <= np.floor(20 / (2.1 - a) ** (5.5 - 2 * a))) or \
        (a >= 2 and az <= 50)


def _ml_scale(a, b, z):
    """Rounding scale of the evaluation at z: in the power-series region the
    sum of the terms' moduli, E_{a,b}(|z|); in the integral and asymptotic
    forms |E(z)|; through the reductions for a > 1 the mean over the reduced
    points, as the value itself is formed."""
    az = abs(z)
    if _ml_series_region(a, az):
        return abs(restate.mittag_leffler(a, b, [az])[0])
    if a <= 1:
        return abs(restate.mittag_leffler(a, b, [z])[0])
    th = np.angle(z)
    if a >= 2:
        m = int(np.floor(a / 2))
        pts = [az ** (1 / (m + 1)) * np.exp(1j * (2 * np.pi * h + th) / (m + 1)) for h in range(m + 1)]
        return float(np.mean([_ml_scale(a / (m + 1), b, p) for p in pts]))
    r = np.sqrt(az) * np.exp(1j * th / 2)
    return 0.5 * (_ml_scale(a / 2, b, r) + _ml_scale(a / 2, b, -r))


def test_mittag_leffler_device_matches_restatement():
    """hf_mittag_leffler (the GPTT model's E_{alpha,beta}, hf::mittag_leffler) on
    the GPU against the restatement over every region of the evaluation: real
    and imaginary parts to 1e-12 of the evaluation's rounding scale (CUDA's and
    the host's libm differ in the last bits), infinities where the restatement
    overflows.  The scale is |E|, and in the power-series region (also where
    the reductions for alpha > 1 land in it) the sum of the terms' moduli,
    E_{alpha,beta}(|z|): for z off the positive axis the series cancels terms
    up to that size (E_{1,0.4}(-12) = -0.027 from terms near 1e5), so the last
    bits of each term set the result's accuracy there, the reference's too."""
    pts = np.array(ML_POINTS)
    nfinite = 0
    for a in ML_ALPHAS:
        for b in ML_BETAS:
            got = engine.mittag_leffler(a, b, pts)
            want = restate.mittag_leffler(a, b, pts)
            for z, g, w in zip(ML_POINTS, got, want):
                if not np.isfinite(w.real):
                    assert np.isinf(g.real) and np.sign(g.real) == np.sign(w.real), (a, b, z, g, w)
                    continue
                scale = max(abs(w), _ml_scale(a, b, z))
                assert abs(g.real - w.real) <= 1e-12 * scale and abs(g.imag - w.imag) <= 1e-12 * scale, (a, b, z, g, w)
                nfinite += 1
    assert nfinite > 800


def test_mittag_leffler_rejects_out_of_range_arguments():
    with pytest.raises(engine.EngineError) as e:
        engine.mittag_leffler(6.0, 1.0, [1.0])
    assert e.value.code == -1
    with pytest.raises(engine.EngineError):
        engine.mittag_leffler(0.5, 1.0, [1.0], fi=0)
    assert engine.mittag_leffler(0.5, 1.0, np.zeros(0)).size == 0

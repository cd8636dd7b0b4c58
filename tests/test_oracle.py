"""The oracle (CPU restatement over flattened programs) pinned against the
reference HigFlow itself, plus the reference's own known-answer tests restated.

CPU only.  Tests that rebuild cases need the oracle build of the reference
(oracle/_ref/libhigflow_ref{2,3}d.so) and are skipped without it.
"""
import numpy as np
import pytest

from higflow_b200 import program as hp
from oracle import restate
from tests.helpers import (ML_ALPHAS, ML_BETAS, ML_POINTS, compare, field_keys, golden_names, load_golden,
                           load_init)

NAMES = golden_names()

try:
    from oracle import refpy
    HAVE_REF = refpy.available(2) and refpy.available(3)
except Exception:  # pragma: no cover
    HAVE_REF = False


@pytest.mark.parametrize("name", NAMES)
def test_restatement_matches_reference_fields(name):
    """hf_restate.c over the recorded program reproduces the reference's own
    N-step fields (tests/golden, written by higflow_solver_step[_viscoelastic])."""
    prog, data = load_golden(name)
    st = restate.State(prog)
    load_init(st, prog, data)
    st.step(int(data["steps"]), rtol=1e-14)
    keys = [k for k, _, _ in field_keys(prog) if k != "dp" and not k.startswith("S")]
    got = {k: st.get(fid, comp) for k, fid, comp in field_keys(prog)}
    want = {k: data["ref_" + k] for k in keys}
    err = compare(got, want, keys)
    assert max(err.values()) < 1e-10, err


def test_golden_fixtures_present():
    assert len(NAMES) >= 10


def _rebuild(name):
    from tests.golden.make_golden import CASES
    factory, steps, amps = CASES[name]
    return factory, steps, amps


@pytest.mark.skipif(not HAVE_REF, reason="oracle build of the reference not available")
@pytest.mark.parametrize("name", ["cav2d_cubista", "ve2d_oldroyd_log", "chan2d_cubista", "cav3d_cubista"])
def test_flattener_is_deterministic_and_bit_exact(name):
    """Flattening the same reference case again gives the committed program
    bit for bit: same slots, same row ids, same weights and boundary terms."""
    from tests.golden import make_golden
    import tempfile, os, shutil
    prog, _ = load_golden(name)
    d = tempfile.mkdtemp()
    try:
        old = make_golden.HERE
        make_golden.HERE = d
        make_golden.make(name)
        make_golden.HERE = old
        p2 = hp.Program.load(os.path.join(d, f"{name}.prog.npz"))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    for attr in ("row_tmpl", "row_base", "row_rhs", "tmpl_ptr", "tmpl_col", "tmpl_w", "div_slots", "p_ptr",
                 "p_col", "p_val", "p_brhs", "delta"):
        a, b = getattr(prog, attr), getattr(p2, attr)
        assert a.dtype == b.dtype and np.array_equal(a, b), attr
    for d_ in range(prog.dim):
        assert np.array_equal(prog.vel_slots[d_], p2.vel_slots[d_])
        assert np.array_equal(prog.vel_flags[d_], p2.vel_flags[d_])
    assert prog.pin_row == p2.pin_row


@pytest.mark.skipif(not HAVE_REF, reason="oracle build of the reference not available")
def test_poisson_rows_match_reference_assembly():
    """The flattened Poisson rows equal the system higflow_pressure assembles
    and hands to the solver plugin (captured inside the oracle's engine)."""
    spec = refpy.cavity(2, 10, Re=10.0, dt=1e-3)
    c = refpy.RefCase(spec)
    prog = c.flatten()
    c.step(1)
    ptr, col, val, b = c.last_system()
    n = prog.ncell
    for r in range(n):
        ref = dict(zip(col[ptr[r]:ptr[r + 1]], val[ptr[r]:ptr[r + 1]]))
        if r == prog.pin_row:
            assert ref == {r: 1.0}
            continue
        mine = {}
        for k in range(prog.p_ptr[r], prog.p_ptr[r + 1]):
            mine[int(prog.p_col[k])] = mine.get(int(prog.p_col[k]), 0.0) + prog.p_val[k]
        assert mine.keys() == ref.keys()
        for k in ref:
            assert mine[k] == ref[k]
    c.close()


@pytest.mark.skipif(not HAVE_REF, reason="oracle build of the reference not available")
def test_wls_rows_reproduce_linear_and_quadratic_fields():
    """Known answers of higtree/atf-tests/test-wls-2d.c:10-139 restated on the
    recorded interpolation rows: order-2 moving least squares reproduces
    f = 2 + 3x + 4y (2.0 at the origin, 5.5 at (0.5, 0.5), 9.0 at (1, 1)) and a
    quadratic exactly at every interior query point."""
    spec = refpy.cavity(2, 16, Re=10.0, dt=1e-3)
    c = refpy.RefCase(spec)
    prog = c.flatten()
    D = 2
    centers = [c.centers(d) for d in range(D)]
    fcent = [centers[d] for d in range(D)]
    lin = lambda x: 2.0 + 3.0 * x[..., 0] + 4.0 * x[..., 1]
    quad = lambda x: x[..., 0] ** 2 - 0.5 * x[..., 0] * x[..., 1] + 0.25 * x[..., 1] ** 2 - 0.25
    checked = 0
    for d in range(D):
        nf = prog.nfacet[d]
        for d2 in range(D):
            for slot, sign in ((hp.V_BLK0 + hp.V_NB * d2 + hp.V_VCR, 1.0), (hp.V_BLK0 + hp.V_NB * d2 + hp.V_VCL, -1.0)):
                codes = prog.vel_slots[d][slot]
                for f in range(nf):
                    code = int(codes[f])
                    if code >= 0:
                        continue
                    r = -code - 1
                    t = prog.row_tmpl[r]
                    a, b = prog.tmpl_ptr[t], prog.tmpl_ptr[t + 1]
                    w = prog.tmpl_w[a:b]
                    if prog.row_rhs[r] != 0.0 or abs(w.sum() - 1.0) > 1e-12:
                        continue  # row mixes in boundary samples
                    pts = fcent[d2][prog.row_base[r] + prog.tmpl_col[a:b]]
                    xq = fcent[d][f].copy()
                    delta = prog.delta[prog.vel_delta[d][f]]
                    xq[d2] += sign * 0.5 * delta[d2]
                    for fn in (lin, quad):
                        assert abs(np.dot(w, fn(pts)) - fn(xq)) < 1e-10
                    checked += 1
    assert checked > 100
    # the three known answers of the linear case at the reference's points
    pts = np.array([[-1, -1], [-1, 0], [-1, 1], [1, -1], [1, 0], [1, 1]], dtype=float)
    vals = lin(pts)
    assert list(vals) == [-5, -1, 3, 1, 5, 9]
    assert [lin(np.array(p)) for p in ([0.0, 0.0], [0.5, 0.5], [1.0, 1.0])] == [2.0, 5.5, 9.0]
    c.close()


def test_program_roundtrip(tmp_path):
    prog, _ = load_golden("ve2d_oldroyd_log")
    p = tmp_path / "x.prog.npz"
    prog.save(str(p))
    q = hp.Program.load(str(p))
    assert q.par == prog.par
    assert np.array_equal(q.cell_slots, prog.cell_slots)
    c = q.to_c()
    assert c.ncell == prog.ncell and c.vel_nslot == prog.vel_slots[0].shape[0]


@pytest.mark.skipif(not HAVE_REF, reason="oracle build of the reference not present")
@pytest.mark.parametrize("dim,ve", [(2, False), (2, True), (3, False)])
def test_cfl_matches_reference(dim, ve):
    """The restated CFL number (higflow_compute_CFL, hig-flow-timestep.c:7-40)
    against the reference's own on the same random velocity, and the adaptive
    step's formula against the reference's higflow_adjust_timestep."""
    kw = dict(Re=10.0, dt=1e-3)
    if ve:
        kw.update(flowtype=hp.VISCOELASTIC, ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG)
    c = refpy.RefCase(refpy.cavity(dim, 12 if dim == 2 else 6, **kw))
    rng = np.random.default_rng(3)
    for d in range(dim):
        c.set(hp.FIELD_U, d, 0.7 * rng.standard_normal(c.nfacet[d]))
    prog = c.flatten()   # also warms HigTree's stencil cache, as every step after the first reads it
    st = restate.State(prog)
    for d in range(dim):
        st.set(hp.FIELD_U, d, c.get(hp.FIELD_U, d))
    want = c.cfl()
    got = st.cfl()
    assert abs(got - want) <= 1e-14 * abs(want), (got, want)
    dt0 = c.dt
    c.adjust_timestep()
    expect = min(min(0.1 / (want + 1e-12), 1.1) * dt0, 32 * dt0)
    assert abs(c.dt - expect) <= 1e-15 * expect, (c.dt, expect)
    c.close()


@pytest.mark.skipif(not HAVE_REF, reason="oracle build of the reference not present")
@pytest.mark.skipif(not HAVE_REF, reason="oracle build of the reference not present")
def test_mittag_leffler_restatement_matches_reference():
    """E_{alpha,beta}(z) of the restatement (hf_restate.c, ml_eval) against the
    reference's own mlfv (hig-flow-mittag-leffler.c:117) over every region of
    the evaluation, fi = 6 as the GPTT model passes: real parts to 1e-13
    relative, overflow to inf on both sides together.  (Imaginary parts are
    not compared: the reference's asymptotic leading term has the sign of its
    sine wrong, which never reaches a real part.)"""
    pts = np.array(ML_POINTS)
    n_region = {"finite": 0, "inf": 0}
    for a in ML_ALPHAS:
        for b in ML_BETAS:
            mine = restate.mittag_leffler(a, b, pts)
            for z, m in zip(ML_POINTS, mine):
                r = refpy.mlfv(a, b, z)
                if not np.isfinite(r.real):
                    assert m.real == r.real, (a, b, z, r, m)
                    n_region["inf"] += 1
                    continue
                assert abs(m.real - r.real) <= 1e-13 * abs(r.real), (a, b, z, r, m)
                n_region["finite"] += 1
    assert n_region["finite"] > 800


def test_gptt_out_of_range_parameters_are_refused():
    """GPTT with alpha_gptt outside (0, 5] (the range the reference's
    Mittag-Leffler evaluation accepts) is refused at flatten with the reason."""
    if not HAVE_REF:
        pytest.skip("oracle build of the reference not present")
    c = refpy.RefCase(refpy.cavity(2, 8, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GPTT,
                                   kernel=hp.KERNEL_LOG, alpha_gptt=6.0, beta_gptt=1.0))
    with pytest.raises(Exception) as e:
        c.flatten()
    assert "alpha_gptt" in str(e.value)
    c.close()


def test_fene_p_is_refused_with_its_reason():
    """FENE-P stays off the GPU path: the reference's polymeric tensor reads xi
    without assigning it for this model, so there is no defined stress to match."""
    c = refpy.RefCase(refpy.cavity(2, 8, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.FENE_P,
                                   kernel=hp.KERNEL_LOG, L2_fene=100.0))
    with pytest.raises(Exception) as e:
        c.flatten()
    assert "FENE-P" in str(e.value)
    c.close()

"""Serving (hf_server_*): requests admitted while others run, each one the same
alone and in the mix, bit for bit (every request is an engine case of its own
with deterministic kernels; tolerance 0)."""
import time

import numpy as np
import pytest

from higflow_b200 import engine
from higflow_b200 import program as hp
from higflow_b200 import host

pytestmark = pytest.mark.gpu


def _requests():
    """(program, options, steps, initial fields): Newtonian and viscoelastic
    cavities of several sizes, step counts and parameters."""
    out = []
    rng = np.random.default_rng(3)
    for k, (n, ve, steps) in enumerate([(24, False, 7), (40, True, 5), (32, True, 9), (56, False, 4),
                                        (28, True, 6), (48, False, 8)]):
        par = dict(Re=1.0 if ve else 100.0, dt=1e-4 if ve else 2e-4)
        if ve:
            par.update(flowtype=hp.VISCOELASTIC, ve_model=hp.GIESEKUS if k % 2 else hp.OLDROYD_B, De=0.3 + 0.1 * k,
                       alpha=0.2, beta=0.1, kernel=hp.KERNEL_LOG, kernel_tol=1e-2)
        prog = host.record(host.cavity(2, n, **par))
        fields = {(hp.FIELD_U, d): 0.05 * rng.standard_normal(prog.nfacet[d]) for d in range(2)}
        out.append((prog, engine.options(rtol=1e-10, atol=1e-300, precision=hp.PREC_MIXED if ve else hp.PREC_FP64),
                    steps, fields))
    return out


def _fields(get, prog):
    keys = [(hp.FIELD_U, 0), (hp.FIELD_U, 1), (hp.FIELD_P, 0)]
    if prog.viscoelastic:
        keys += [(hp.FIELD_KERNEL, k) for k in range(4)]
    return {k: get(*k) for k in keys}


def test_requests_are_the_same_alone_and_in_the_mix():
    reqs = _requests()
    alone = []
    for prog, opts, steps, fields in reqs:
        case = engine.Case(prog, opts)
        for (fid, comp), v in fields.items():
            case.set(fid, comp, v)
        case.step(steps)
        alone.append(_fields(case.get, prog))
        case.close()
    # a budget that holds about two of these cases at a time: later requests
    # are admitted as earlier ones are released
    budget = 2.5 * max(engine.device_bytes(p) for p, *_ in reqs) * 1.5 / 1e9
    srv = engine.Server(budget_gb=budget, max_active=4, chunk_steps=2, setup_threads=2)
    ids = [srv.submit(prog, opts, steps, fields) for prog, opts, steps, fields in reqs]
    for k, rid in enumerate(ids):
        status, queue_s, total_s = srv.wait(rid)
        assert status == 0
        assert total_s >= queue_s >= 0.0
        got = _fields(lambda f, c: srv.get(rid, f, c), reqs[k][0])
        for key in got:
            assert np.array_equal(got[key], alone[k][key]), (k, key)
        srv.release(rid)
    st = srv.stats()
    assert st.submitted == len(reqs) and st.completed == len(reqs) and st.failed == 0
    assert st.cell_steps == sum(p.ncell * s for p, _, s, _ in reqs)
    srv.close()


def test_a_failing_request_does_not_disturb_the_others():
    reqs = _requests()[:3]
    srv = engine.Server(max_active=3, chunk_steps=1, setup_threads=2)
    prog, opts, steps, fields = reqs[0]
    bad = {k: v.copy() for k, v in fields.items()}
    bad[(hp.FIELD_U, 0)][5] = np.nan
    ids = [srv.submit(prog, opts, steps, bad)] + [srv.submit(p, o, s, f) for p, o, s, f in reqs[1:]]
    assert srv.wait(ids[0])[0] == -4          # HF_ERR_NAN, reported for that request only
    for rid in ids[1:]:
        assert srv.wait(rid)[0] == 0
    for rid in ids:
        srv.release(rid)
    srv.close()


def test_batch_server_results_are_the_same_alone_and_in_the_mix():
    """Continuous batching (higflow_b200.serve.BatchServer): requests submitted
    while others run are grouped into cohorts that step as one batch, each
    request frozen at its own step count.  Every result equals the request run
    alone as an engine case for its steps (1e-10 relative L2, plain FP64)."""
    from higflow_b200 import serve
    reqs = _requests()
    opts = engine.options(rtol=1e-13, atol=1e-300)
    srv = serve.BatchServer(opts=opts, max_cohorts=3, chunk=3)
    ids = []
    for k, (prog, _, steps, fields) in enumerate(reqs):
        ids.append(srv.submit(prog, steps, fields))
        if k == 2:
            time.sleep(0.05)       # the later ones arrive while the first cohort runs
    got = []
    for rid, (prog, _, _, _) in zip(ids, reqs):
        status, q, t = srv.wait(rid, timeout=300)
        assert status == 0
        got.append({k: srv.get(rid, *k) for k in _fields(lambda f, c: None, prog)})
        srv.release(rid)
    st = srv.stats()
    srv.close()
    assert st["cohorts"] >= 2
    for (prog, _, steps, fields), mix in zip(reqs, got):
        case = engine.Case(prog, opts)
        for key, v in fields.items():
            case.set(*key, v)
        case.step(steps)
        alone = _fields(case.get, prog)
        case.close()
        for k in alone:
            err = np.linalg.norm(alone[k] - mix[k]) / max(np.linalg.norm(alone[k]), 1e-300)
            assert err < 1e-10, (k, err)


def test_batch_server_failing_request_fails_alone():
    """A request whose fields hold a NaN fails with HF_ERR_NAN; the engine
    freezes its instance and the rest of its cohort finishes unchanged."""
    from higflow_b200 import serve
    reqs = _requests()[:4]
    opts = engine.options(rtol=1e-13, atol=1e-300)
    bad = {k: v.copy() for k, v in reqs[1][3].items()}
    bad[(hp.FIELD_U, 0)][7] = np.nan
    srv = serve.BatchServer(opts=opts, max_cohorts=1, chunk=2)
    ids = [srv.submit(prog, steps, bad if k == 1 else fields) for k, (prog, _, steps, fields) in enumerate(reqs)]
    statuses = [srv.wait(rid, timeout=300)[0] for rid in ids]
    assert statuses == [0, -4, 0, 0]
    got = {k: {key: srv.get(ids[k], *key) for key in _fields(lambda f, c: None, reqs[k][0])} for k in (0, 2, 3)}
    st = srv.stats()
    srv.close()
    assert st["cell_steps"] == sum(reqs[k][0].ncell * reqs[k][2] for k in (0, 2, 3))
    for k in (0, 2, 3):
        prog, _, steps, fields = reqs[k]
        case = engine.Case(prog, opts)
        for key, v in fields.items():
            case.set(*key, v)
        case.step(steps)
        alone = _fields(case.get, prog)
        case.close()
        for key in alone:
            err = np.linalg.norm(alone[key] - got[k][key]) / max(np.linalg.norm(alone[key]), 1e-300)
            assert err < 1e-10, (k, key, err)

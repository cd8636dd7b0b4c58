"""Batched cases on one GPU: each instance's result is the same alone and in a
batch, and the mixed-precision form agrees with the plain FP64 form.

Tolerances: plain FP64 alone vs in a batch 1e-10 relative L2 (both solve each
instance to its own 1e-13 Poisson residual); mixed vs plain 1e-6 relative L2
(the FP32 inner solve is refined in FP64 to the same residual test).
"""
import numpy as np
import pytest

from higflow_b200 import engine
from higflow_b200 import program as hp
from tests.helpers import compare, field_keys, load_golden, load_init

pytestmark = pytest.mark.gpu

# the models differ per instance (Oldroyd-B, Giesekus, LPTT, GPTT, e-FENE)
VE_NAMES = ["ve2d_oldroyd_log", "ve2d_giesekus_log", "ve2d_lptt_sqrt", "ve2d_oldroyd_central", "gptt2d_log",
            "efene2d_log"]
NEWT_NAMES = ["cav2d_cubista", "cav2d_quick", "cav2d_central", "chan2d_cubista", "cav2d_lid"]


def _run_alone(name, steps, **kw):
    prog, data = load_golden(name)
    case = engine.Case(prog, engine.options(rtol=1e-13, atol=1e-300, **kw))
    load_init(case, prog, data)
    case.step(steps)
    out = {k: case.get(fid, comp) for k, fid, comp in field_keys(prog)}
    case.close()
    return out


def _keys(prog):
    return [k for k, _, _ in field_keys(prog) if k != "dp"]


@pytest.mark.parametrize("names", [VE_NAMES, NEWT_NAMES])
def test_instances_same_alone_and_in_batch(names):
    steps = 3
    progs, datas = zip(*[load_golden(n) for n in names])
    batch = hp.Program.concatenate(progs)
    case = engine.Case(batch, engine.options(rtol=1e-13, atol=1e-300))
    assert case.instances() == len(names)
    # initial fields, instance by instance, in the concatenated arrays
    for key, fid, comp in field_keys(progs[0]):
        whole = np.concatenate([d["init_" + key] for d in datas])
        case.set(fid, comp, whole)
    case.step(steps)
    for i, (name, prog) in enumerate(zip(names, progs)):
        alone = _run_alone(name, steps)
        got = {k: case.get_instance(fid, comp, i) for k, fid, comp in field_keys(prog)}
        err = compare(got, alone, _keys(prog))
        assert max(err.values()) < 1e-10, (name, err)
        # CG accepts a breakdown once ||r|| <= 100 rtol ||b|| (the recurrence has
        # lost its last digits there); that is the bound on the reported residual
        it, outer, status, res = case.instance_result(i)
        assert status == 0 and res < 1e-11
    case.close()


@pytest.mark.parametrize("name", ["cav2d_cubista", "ve2d_oldroyd_log", "cav3d_cubista"])
def test_mixed_precision_matches_plain(name):
    prog, data = load_golden(name)
    steps = int(data["steps"])
    plain = _run_alone(name, steps)
    mixed = _run_alone(name, steps, precision=hp.PREC_MIXED)
    err = compare(mixed, plain, _keys(prog))
    assert max(err.values()) < 1e-6, err


def test_mixed_precision_reaches_the_same_residual():
    prog, data = load_golden("cav2d_lid")
    case = engine.Case(prog, engine.options(rtol=1e-10, atol=1e-300, precision=hp.PREC_MIXED))
    load_init(case, prog, data)
    case.step(5)
    it, outer, status, res = case.instance_result(0)
    assert status == 0 and res <= 1e-10 and outer >= 1
    case.close()


def test_eager_launches_match_the_step_graph():
    """The same kernels launched one by one (host-driven iteration loop) give
    the graph's results bit for bit."""
    names = VE_NAMES[:2]
    progs, datas = zip(*[load_golden(n) for n in names])
    batch = hp.Program.concatenate(progs)
    out = []
    for eager in (False, True):
        case = engine.Case(batch, engine.options(rtol=1e-13, atol=1e-300, precision=hp.PREC_MIXED, eager=eager))
        for key, fid, comp in field_keys(progs[0]):
            case.set(fid, comp, np.concatenate([d["init_" + key] for d in datas]))
        case.step(3)
        out.append({k: case.get(fid, comp) for k, fid, comp in field_keys(progs[0])})
        assert case.stats().total_iters > 0
        case.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("precision", [hp.PREC_FP64, hp.PREC_MIXED])
def test_step_limits_freeze_each_instance_at_its_count(precision):
    """hf_case_set_step_limits: instance i takes limits[i] steps and is then
    frozen while the batch goes on; its fields equal the instance run alone
    for limits[i] steps (1e-10 relative L2), in both precision forms."""
    names = VE_NAMES[:4]
    limits = [1, 4, 2, 6]
    progs, datas = zip(*[load_golden(n) for n in names])
    batch = hp.Program.concatenate(progs)
    case = engine.Case(batch, engine.options(rtol=1e-13, atol=1e-300, precision=precision))
    for key, fid, comp in field_keys(progs[0]):
        case.set(fid, comp, np.concatenate([d["init_" + key] for d in datas]))
    case.set_step_limits(limits)
    case.step(max(limits) + 2)
    for i, (name, prog) in enumerate(zip(names, progs)):
        alone = _run_alone(name, limits[i], precision=precision)
        got = {k: case.get_instance(fid, comp, i) for k, fid, comp in field_keys(prog)}
        err = compare(got, alone, _keys(prog))
        assert max(err.values()) < 1e-10, (name, limits[i], err)
    case.close()


def test_launch_shape_tuning_changes_no_result():
    """hf_options.tuning: the tuned block sizes give the built-in sizes' fields
    bit for bit (each thread's work and order do not depend on the block
    size), and the sizes kept are among the candidates."""
    names = VE_NAMES[:3]
    progs, datas = zip(*[load_golden(n) for n in names])
    batch = hp.Program.concatenate(progs)
    out = []
    for tune in (True, False):
        case = engine.Case(batch, engine.options(rtol=1e-13, atol=1e-300, precision=hp.PREC_MIXED, tune=tune))
        for key, fid, comp in field_keys(progs[0]):
            case.set(fid, comp, np.concatenate([d["init_" + key] for d in datas]))
        case.step(3)
        out.append({k: case.get(fid, comp) for k, fid, comp in field_keys(progs[0])})
        shapes = case.launch_shapes()
        if tune:
            assert shapes[0] in (128, 256, 512) and shapes[1] in (64, 128, 256) and shapes[2] in (64, 128)
        else:
            assert shapes == (256, 128, 128)
        case.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_a_failed_instance_under_step_limits_is_frozen_alone():
    """Under step limits an instance whose step fails (here a NaN in its
    initial velocity) is frozen at that step and reported by
    hf_case_instance_failures; the step call returns the failure; the other
    instances go on and equal their runs alone (1e-10 relative L2)."""
    names = VE_NAMES[:3]
    progs, datas = zip(*[load_golden(n) for n in names])
    batch = hp.Program.concatenate(progs)
    case = engine.Case(batch, engine.options(rtol=1e-13, atol=1e-300))
    for key, fid, comp in field_keys(progs[0]):
        whole = np.concatenate([d["init_" + key] for d in datas])
        if key == "u0":
            whole[batch.facet_off[0][1] + 3] = np.nan      # instance 1
        case.set(fid, comp, whole)
    case.set_step_limits([4, 4, 4])
    with pytest.raises(engine.EngineError) as e:
        case.step(4)
    assert e.value.code == -4
    assert list(case.instance_failures()) == [0, -4, 0]
    for i in (0, 2):
        alone = _run_alone(names[i], 4)
        got = {k: case.get_instance(fid, comp, i) for k, fid, comp in field_keys(progs[i])}
        err = compare(got, alone, _keys(progs[i]))
        assert max(err.values()) < 1e-10, (names[i], err)
    case.close()

"""The benchmark configurations against the reference itself, at their own sizes.

Programs are recorded by the HigFlow host (higflow_b200/host.py) exactly as the
benchmark records them; the reference fields come from the reference's own
step (tests/golden/make_configs.py).  Tolerances, relative L2 per field:
plain FP64 1e-10 (the parity bar), mixed form 1e-6 (the precision bar of the
mixed form against the FP64 oracle).

* C1: the 64x64 Newtonian lid-driven cavity, Re 100, dt 1e-4, 200 steps from
  rest (the whole configuration).
* C4 subset: six instances of the batched Giesekus population (sides 32 to
  129), 20 steps from rest with the conformation at the identity, run as one
  batch.  From the identity the reference's conformation is ill-conditioned
  (its spin term divides by an eigenvalue gap plus 1e-12,
  hig-flow-step-viscoelastic.c:1667): the fixture stores, per instance and
  field, how far the reference's own fields move when its Poisson tolerance
  goes from 1e-15 to 1e-13, and a field's bound is the larger of the
  tolerance above and three times that sensitivity (it exceeds 1e-10 for the
  side-129 instance's K, about 4e-6; every other field of every instance is
  held to the plain bar).  The mixed form's perturbations are of FP32 size,
  so its bound takes the reference's sensitivity to a Poisson tolerance of
  1e-6 instead; the K of an instance whose reference K moves by more than
  1e-9 under a 1e-13 Poisson change (the side-129 instance) is not bounded
  in the mixed form after 20 steps (a perturbation of FP32 size moves it by
  an amount no reference run bounds: about 3e-2 measured), and is held to
  the mixed bar over the configuration's full 2000 steps instead (C4
  instance test below).
* C4 instance: that side-129 instance alone over the configuration's 2000
  steps, after 200 and after 2000 steps, against the reference, both forms,
  the bounds built the same way from the reference's own sensitivity (the
  mixed form's K at the end only).
"""
import os

import numpy as np
import pytest

from higflow_b200 import engine, host, workloads
from higflow_b200 import program as hp
from tests.helpers import GOLDEN, rel_l2

PLAIN_TOL = 1e-10
MIXED_TOL = 1e-6


def _c1():
    prog = host.record(host.cavity(2, 64, Re=100.0, dt=1e-4))
    ref = dict(np.load(os.path.join(GOLDEN, "c1_64_200.npz")))
    return prog, ref


@pytest.mark.gpu
@pytest.mark.parametrize("precision, tol", [(hp.PREC_FP64, PLAIN_TOL), (hp.PREC_MIXED, MIXED_TOL)])
def test_c1_whole_configuration_matches_reference(precision, tol):
    prog, ref = _c1()
    case = engine.Case(prog, engine.options(rtol=1e-13 if precision == hp.PREC_FP64 else 1e-10, atol=1e-300,
                                            precision=precision))
    case.step(int(ref["steps"]))
    err = {"u0": rel_l2(ref["ref_u0"], case.get(hp.FIELD_U, 0)), "u1": rel_l2(ref["ref_u1"], case.get(hp.FIELD_U, 1)),
           "p": rel_l2(ref["ref_p"], case.get(hp.FIELD_P))}
    case.close()
    assert max(err.values()) < tol, err


def _c4_sub():
    ref = dict(np.load(os.path.join(GOLDEN, "c4_sub_20.npz")))
    draws = workloads.batched_giesekus()
    idx = [int(i) for i in ref["index"]]
    progs = [host.record(workloads.spec(draws[i])) for i in idx]
    return idx, progs, ref


@pytest.mark.gpu
@pytest.mark.parametrize("precision, tol", [(hp.PREC_FP64, PLAIN_TOL), (hp.PREC_MIXED, MIXED_TOL)])
def test_c4_subset_batch_matches_reference(precision, tol):
    idx, progs, ref = _c4_sub()
    batch = hp.Program.concatenate(progs)
    case = engine.Case(batch, engine.options(rtol=1e-13 if precision == hp.PREC_FP64 else 1e-10, atol=1e-300,
                                             precision=precision))
    case.step(int(ref["steps"]))
    worst = {}
    for j, i in enumerate(idx):
        got = {f"u{d}": case.get_instance(hp.FIELD_U, d, j) for d in range(2)}
        got["p"] = case.get_instance(hp.FIELD_P, 0, j)
        for k in range(4):
            got[f"K{k}"] = case.get_instance(hp.FIELD_KERNEL, k, j)
        if precision == hp.PREC_MIXED and max(float(ref[f"sens{i}_K{k}"]) for k in range(4)) > 1e-9:
            got = {k: v for k, v in got.items() if not k.startswith("K")}
        err = {k: rel_l2(ref[f"ref{i}_{k}"], v) for k, v in got.items()}
        sens = "sens" if precision == hp.PREC_FP64 else "sens6_"
        bound = {k: max(tol, 3.0 * float(ref[f"{sens}{i}_{k}"])) for k in got}
        worst[i] = max(err[k] / bound[k] for k in got)
        assert worst[i] < 1.0, (i, err, bound)
    case.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision, tol", [(hp.PREC_FP64, PLAIN_TOL), (hp.PREC_MIXED, MIXED_TOL)])
def test_c4_instance_full_steps_matches_reference(precision, tol):
    ref = dict(np.load(os.path.join(GOLDEN, "c4_61_2000.npz")))
    i = int(ref["index"])
    prog = host.record(workloads.spec(workloads.batched_giesekus()[i]))
    case = engine.Case(hp.Program.concatenate([prog]),
                       engine.options(rtol=1e-13 if precision == hp.PREC_FP64 else 1e-10, atol=1e-300,
                                      precision=precision))
    done = 0
    marks = [int(x) for x in ref["marks"]]
    for m in marks:
        case.step(m - done)
        done = m
        got = {f"u{d}": case.get(hp.FIELD_U, d) for d in range(2)}
        got["p"] = case.get(hp.FIELD_P)
        # the mixed form's K is held to its bound at the configuration's end;
        # after 200 steps it is still in the ill-conditioned start (measured:
        # 1.0e-4 in K0 against the reference's 2.3e-5 sensitivity to a 1e-6
        # Poisson tolerance, u and p within 1e-7)
        if precision == hp.PREC_FP64 or m == marks[-1]:
            for k in range(4):
                got[f"K{k}"] = case.get(hp.FIELD_KERNEL, k)
        err = {k: rel_l2(ref[f"ref{m}_{k}"], v) for k, v in got.items()}
        sens = "sens" if precision == hp.PREC_FP64 else "sens6_"
        bound = {k: max(tol, 3.0 * float(ref[f"{sens}{m}_{k}"])) for k in got}
        assert max(err[k] / bound[k] for k in got) < 1.0, (m, err, bound)
    case.close()


def test_fixture_instances_are_the_generator_selection():
    from tests.golden.make_configs import c4_subset
    ref = np.load(os.path.join(GOLDEN, "c4_sub_20.npz"))
    assert [int(i) for i in ref["index"]] == c4_subset()


@pytest.mark.gpu
def test_c2_reduced_contraction_matches_reference():
    """C2's case (4:1 contraction, two trees with refined corners, Oldroyd-B,
    Re 0.01, Wi 1, semi-implicit velocity, dt 5e-5) at 8 cells per unit
    length, on the BiCGStab Poisson path (the AMR rows are not symmetric).
    After one step every field is held to 1e-10; after ten the bound is the
    larger of 1e-10 and three times the reference's own sensitivity to its
    Poisson tolerance, which the constitutive update from the identity grows
    to about 1e-6 in u and 1e-2 in K within those ten steps."""
    from tests.golden.make_configs import c2_spec
    ref = dict(np.load(os.path.join(GOLDEN, "c2_8.npz")))
    prog = host.record(c2_spec(int(ref["per_unit"])))
    case = engine.Case(prog, engine.options(rtol=1e-13, atol=1e-300))
    done = 0
    for m in (int(x) for x in ref["marks"]):
        case.step(m - done)
        done = m
        got = {f"u{d}": case.get(hp.FIELD_U, d) for d in range(2)}
        got["p"] = case.get(hp.FIELD_P)
        for k in range(4):
            got[f"K{k}"] = case.get(hp.FIELD_KERNEL, k)
        err = {k: rel_l2(ref[f"ref{m}_{k}"], v) for k, v in got.items()}
        bound = {k: max(PLAIN_TOL, 3.0 * float(ref[f"sens{m}_{k}"])) for k in got}
        assert all(err[k] < bound[k] for k in got), (m, err, bound)
    case.close()

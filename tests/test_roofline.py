"""Algorithmic bytes of a step (higflow_b200/roofline.py), on recorded programs.

Checked against counts made directly on the program: distinct centre hits and
distinct rows per field, their entries, and the convention's arithmetic."""
import numpy as np
import pytest

from higflow_b200 import host, roofline
from higflow_b200 import program as hp

pytestmark = pytest.mark.skipif(not host.available(2), reason="HigFlow host library not built")


def _prog():
    return host.record(host.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GIESEKUS,
                                   kernel=hp.KERNEL_LOG))


def test_divergence_and_final_counts_by_hand():
    p = _prog()
    sb = roofline.step_bytes(p, mixed=False)
    # divergence: u*[d] at the cell faces; centre hits are distinct facet ids
    # per direction (UL and UR of one direction read the same field)
    hits = sum(np.unique(np.concatenate([p.div_slots[2 * d], p.div_slots[2 * d + 1]])[
        np.concatenate([p.div_slots[2 * d], p.div_slots[2 * d + 1]]) >= 0]).size for d in range(2))
    assert sb["divergence"]["centre_hits"] == hits
    nf = sum(p.nfacet[:2])
    assert sb["divergence"]["F"] == 8 * (nf + p.ncell)
    assert sb["final"]["F"] == 8 * (2 * nf + 3 * p.ncell)


def test_velocity_rows_and_widths():
    p = _prog()
    plain, mixed = roofline.step_bytes(p, False), roofline.step_bytes(p, True)
    v, vm = plain["velocity"], mixed["velocity"]
    assert v["rows"] == vm["rows"] and v["row_entries"] == vm["row_entries"] > 0
    # the weights are the only difference: 4 bytes per row entry
    assert v["S"] - vm["S"] == 4 * v["row_entries"]
    assert v["S"] == 4 * v["queries"] + 4 * v["centre_hits"] + 12 * v["row_entries"]
    ws = roofline.whole_step(p, False, iters=3.0)
    assert ws["bytes"] == pytest.approx(ws["fixed"] + 3.0 * roofline.poisson_iter_bytes(p, 8))
    assert roofline.poisson_iter_bytes(p, 8) == 4 * (p.ncell + 1) + p.p_col.size * 12 + 13 * 8 * p.ncell


def test_bench_phase_bytes_split_the_stages():
    """The per-kernel figures the bench line reports beside the phases:
    velocity_rows is the velocity stage's stencil rows alone, ve_cell_main the
    cell stage without its polymeric-tensor pass (8 D^2 x 3 bytes per cell)."""
    import bench
    p = _prog()
    for mixed in (False, True):
        pb, sb = bench.phase_bytes(p, mixed, iters_per_step=2.0, sweeps_per_step=1.0 if mixed else 0.0)
        w = 4 if mixed else 8
        v = sb["velocity"]
        assert pb["velocity_rows"] == 4 * v["rows"] + v["row_entries"] * (4 + w)
        assert 0 < pb["velocity_rows"] < pb["velocity"]
        assert pb["ve_cell_main"] == pb["ve_cell"] - 8 * 4 * p.ncell * 3
        assert pb["poisson_iter"] > 2.0 * roofline.poisson_iter_bytes(p, w) - 1

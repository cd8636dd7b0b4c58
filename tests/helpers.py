"""Shared test helpers: golden fixtures, oracle state set-up, comparisons."""
from __future__ import annotations

import glob
import os

import numpy as np

from higflow_b200 import program as hp

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    return sorted(os.path.basename(p)[:-len(".prog.npz")] for p in glob.glob(os.path.join(GOLDEN, "*.prog.npz")))


def load_golden(name: str):
    prog = hp.Program.load(os.path.join(GOLDEN, f"{name}.prog.npz"))
    data = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    return prog, data


def field_keys(prog: hp.Program):
    D = prog.dim
    keys = [(f"u{d}", hp.FIELD_U, d) for d in range(D)] + [("p", hp.FIELD_P, 0), ("dp", hp.FIELD_DP, 0)]
    if prog.viscoelastic:
        keys += [(f"K{k}", hp.FIELD_KERNEL, k) for k in range(D * D)]
        keys += [(f"S{k}", hp.FIELD_S, k) for k in range(D * D)]
    return keys


def load_init(target, prog: hp.Program, data: dict) -> None:
    """Copy the fixture's initial fields into an engine Case or oracle State."""
    for key, fid, comp in field_keys(prog):
        target.set(fid, comp, data["init_" + key])


# Mittag-Leffler parameters and points reaching every region of the
# evaluation: series near 0, the integral form's three sectors with beta <= 1
# and > 1, the asymptotic series, and the reductions for alpha >= 1
ML_ALPHAS = (0.3, 0.5, 0.8, 1.0, 1.3, 1.7, 2.0, 2.5, 3.7, 4.6)
ML_BETAS = (0.4, 1.0, 1.5, 2.2)
ML_POINTS = tuple(complex(x) for x in (-80, -30, -12, -5, -2.5, -1.0, -0.3, 0.0, 0.4, 1.0, 1.7, 3.0, 6.0, 9.0,
                                      14.0, 20.0, 40.0, 70.0)) + (3 + 4j, -2 + 1j, 0.5 - 0.7j, -9 - 9j, 12j)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    na = np.linalg.norm(a)
    return float(np.linalg.norm(a - b) / (na if na > 0 else 1.0))


def compare(got: dict, want: dict, keys) -> dict:
    return {k: rel_l2(want[k], got[k]) for k in keys}

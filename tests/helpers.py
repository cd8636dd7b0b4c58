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


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    na = np.linalg.norm(a)
    return float(np.linalg.norm(a - b) / (na if na > 0 else 1.0))


def compare(got: dict, want: dict, keys) -> dict:
    return {k: rel_l2(want[k], got[k]) for k in keys}

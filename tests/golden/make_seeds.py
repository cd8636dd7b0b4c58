"""Record the seed programs the tiler (higflow_b200/tiling.py) expands.

Each seed is the flattened program of a lid-driven cavity recorded from the
reference HigTree through the HigFlow-side flattener, on a mesh of n cells per
axis, written to higflow_b200/seeds/<name>.prog.npz with <name>.meta.npz
(n, R, box lengths).  Seeds are recorded viscoelastic (log kernel), which is a
superset of the Newtonian slots.  Needs the oracle build of the reference.

    python tests/golden/make_seeds.py [cavity2d|cavity3d]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from higflow_b200 import program as hp  # noqa: E402
from oracle import refpy  # noqa: E402

OUT = os.path.join(REPO, "higflow_b200", "seeds")

SEEDS = {
    # name: (dim, cells per axis, R)
    "cavity2d": (2, 18, 8),
    "cavity3d": (3, 16, 7),
}


def spec(dim: int, n: int):
    return refpy.cavity(dim, n, Re=100.0, dt=1e-3, flowtype=hp.VISCOELASTIC, ve_model=hp.OLDROYD_B,
                        kernel=hp.KERNEL_LOG)


def make(name: str) -> None:
    dim, n, R = SEEDS[name]
    t = time.time()
    c = refpy.RefCase(spec(dim, n))
    prog = c.flatten()
    c.close()
    os.makedirs(OUT, exist_ok=True)
    prog.save(os.path.join(OUT, f"{name}.prog.npz"))
    np.savez(os.path.join(OUT, f"{name}.meta.npz"), n=np.array([n] * dim), R=np.int64(R),
             lengths=np.ones(dim))
    print(f"{name}: n={n} R={R} rows={prog.row_rhs.size} nnz={prog.tmpl_col.size} in {time.time() - t:.1f}s")


def make_c1() -> None:
    """The 64x64 lid-driven cavity of the CPU-runnable benchmark configuration
    (Newtonian, Re 100, dt 1e-4), recorded whole: every stencil is HigTree's."""
    t = time.time()
    c = refpy.RefCase(refpy.cavity(2, 64, Re=100.0, dt=1e-4))
    prog = c.flatten()
    c.close()
    prog.save(os.path.join(OUT, "c1_cavity2d_64.prog.npz"))
    print(f"c1_cavity2d_64: rows={prog.row_rhs.size} nnz={prog.tmpl_col.size} in {time.time() - t:.1f}s")


if __name__ == "__main__":
    for nm in sys.argv[1:] or list(SEEDS) + ["c1"]:
        if nm == "c1":
            make_c1()
        else:
            make(nm)

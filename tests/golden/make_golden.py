"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a container where the reference tree is present and the oracle is built
(``make -C oracle``).  For each case below it builds the reference HigFlow case
from text inputs, sets seeded random initial fields, records the flattened step
program through the HigFlow-side flattener, runs the reference's own
``higflow_solver_step`` / ``higflow_solver_step_viscoelastic`` for ``steps``
steps, and stores program, initial fields and the reference's fields in
``<name>.npz`` plus ``<name>.prog.npz``.

    python tests/golden/make_golden.py            # all cases
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

os.environ.setdefault("HF_ORACLE_RTOL", "1e-15")

from higflow_b200 import program as hp  # noqa: E402
from oracle import refpy  # noqa: E402

# name -> (spec factory, steps, random-field amplitude for u, p, K)
CASES = {
    "cav2d_cubista": (lambda: refpy.cavity(2, 16, Re=100.0, dt=1e-3), 5, (0.3, 0.1, 0.0)),
    "cav2d_quick": (lambda: refpy.cavity(2, 12, Re=50.0, dt=1e-3, secondconvecdiscrtype=hp.QUICK), 4, (0.3, 0.1, 0.0)),
    "cav2d_central": (lambda: refpy.cavity(2, 12, Re=50.0, dt=1e-3, convecdiscrtype=hp.CENTRAL), 4, (0.3, 0.1, 0.0)),
    "cav2d_lid": (lambda: refpy.cavity(2, 16, Re=100.0, dt=1e-3), 10, (0.0, 0.0, 0.0)),
    "cav3d_cubista": (lambda: refpy.cavity(3, 6, Re=100.0, dt=1e-3), 3, (0.3, 0.1, 0.0)),
    "chan2d_cubista": (lambda: refpy.channel(32, 8, Re=1.0, dt=1e-4), 5, (0.3, 0.1, 0.0)),
    "ve2d_oldroyd_log": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC,
                                              ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG), 4, (0.3, 0.1, 0.2)),
    "ve2d_giesekus_log": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC,
                                               ve_model=hp.GIESEKUS, kernel=hp.KERNEL_LOG, alpha=0.3, beta=0.1,
                                               De=0.5), 4, (0.3, 0.1, 0.2)),
    "ve2d_lptt_sqrt": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC,
                                            ve_model=hp.LPTT, kernel=hp.KERNEL_SQRT, epsilon=0.25, xi=0.1),
                       4, (0.3, 0.1, 0.2)),
    "ve2d_oldroyd_central": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC,
                                                  ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_IDENTITY,
                                                  ve_convecdiscrtype=hp.CELL_CENTRAL), 4, (0.3, 0.1, 0.2)),
    "ve3d_oldroyd_log": (lambda: refpy.cavity(3, 5, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC,
                                              ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG), 2, (0.3, 0.1, 0.2)),
    # two-level quadtrees: a refined patch in the middle of the cavity (level-1
    # cells of half the size), so stencils cross coarse/fine interfaces and the
    # Poisson rows are not symmetric there
    "amr2d_cubista": (lambda: refpy.cavity(2, 16, Re=100.0, dt=1e-3,
                                           refine=[([0.5 / 16, 0.5 / 16], [((8, 8), (16, 16))])]), 4, (0.3, 0.1, 0.0)),
    "amr2d_oldroyd_log": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC,
                                               ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG, beta=1.0 / 9.0,
                                               refine=[([0.5 / 12, 0.5 / 12], [((6, 6), (12, 12))])]),
                          3, (0.3, 0.1, 0.2)),
    # semi-implicit Euler velocity (higflow_semi_implicit_euler_intermediate_velocity):
    # a low-Re Newtonian cavity, an Oldroyd-B log cavity and a two-level
    # Oldroyd-B case (the contraction configuration's form: non-symmetric
    # Poisson rows at the level interface)
    # explicit Runge-Kutta velocity (every stage evaluates E(u): the reference's
    # stages read ns->dpu, hig-flow-step.c:639)
    "rk2_cav2d": (lambda: refpy.cavity(2, 16, Re=10.0, dt=1e-3, tempdiscrtype=hp.EXPLICIT_RK2), 4, (0.3, 0.1, 0.0)),
    "rk3_giesekus_log": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC,
                                              ve_model=hp.GIESEKUS, kernel=hp.KERNEL_LOG, alpha=0.3, beta=0.1,
                                              De=0.5, tempdiscrtype=hp.EXPLICIT_RK3), 3, (0.3, 0.1, 0.2)),
    # e-FENE (the reference forms its stress with fA = a = 1: its model switch
    # falls through to the default case)
    "efene2d_log": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.E_FENE,
                                         kernel=hp.KERNEL_LOG, beta=1.0 / 9.0, De=0.5, L2_fene=100.0,
                                         lambda_fene=1.0, E_fene=0.1), 3, (0.3, 0.1, 0.2)),
    # implicit Euler constitutive step (per-cell Kronecker system in Omega)
    "ve2d_oldroyd_implicit": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-3, flowtype=hp.VISCOELASTIC,
                                                   ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG, beta=1.0 / 9.0,
                                                   De=0.5, ve_discrtype=hp.VE_IMPLICIT), 3, (0.3, 0.1, 0.2)),
    "ve2d_giesekus_implicit_central": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-3, flowtype=hp.VISCOELASTIC,
                                                            ve_model=hp.GIESEKUS, kernel=hp.KERNEL_LOG, alpha=0.3,
                                                            beta=0.1, De=0.5, ve_discrtype=hp.VE_IMPLICIT,
                                                            ve_convecdiscrtype=hp.CELL_CENTRAL), 3, (0.3, 0.1, 0.2)),
    "sie2d_cubista": (lambda: refpy.cavity(2, 16, Re=0.1, dt=1e-3, tempdiscrtype=hp.SEMI_IMPLICIT_EULER),
                      4, (0.3, 0.1, 0.0)),
    "sie2d_oldroyd_log": (lambda: refpy.cavity(2, 12, Re=0.01, dt=1e-3, flowtype=hp.VISCOELASTIC,
                                               ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG, beta=1.0 / 9.0,
                                               tempdiscrtype=hp.SEMI_IMPLICIT_EULER), 3, (0.3, 0.1, 0.2)),
    "cn2d_cubista": (lambda: refpy.cavity(2, 16, Re=0.1, dt=1e-3, tempdiscrtype=hp.SEMI_IMPLICIT_CN),
                     4, (0.3, 0.1, 0.0)),
    "cn2d_oldroyd_log": (lambda: refpy.cavity(2, 12, Re=0.01, dt=1e-3, flowtype=hp.VISCOELASTIC,
                                              ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG, beta=1.0 / 9.0,
                                              tempdiscrtype=hp.SEMI_IMPLICIT_CN), 3, (0.3, 0.1, 0.2)),
    # GPTT: Gamma(beta_g) E_{alpha_g,beta_g}(eps Re De tr S / (1 - beta)) in M;
    # the first steps' tr S reaches both sides of the Mittag-Leffler series /
    # integral boundary (|z| up to 1.5 and 3), beta_g > 1 takes the arc integral
    "gptt2d_log": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GPTT,
                                        kernel=hp.KERNEL_LOG, beta=1.0 / 9.0, De=0.5, epsilon=0.15, xi=0.1,
                                        alpha_gptt=0.5, beta_gptt=1.0), 3, (0.3, 0.1, 0.2)),
    "gptt2d_b12_implicit": (lambda: refpy.cavity(2, 12, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GPTT,
                                                 kernel=hp.KERNEL_LOG, beta=1.0 / 9.0, De=0.5, epsilon=0.3, xi=0.1,
                                                 alpha_gptt=0.8, beta_gptt=1.2, ve_discrtype=hp.VE_IMPLICIT),
                            3, (0.3, 0.1, 0.2)),
    # the same in 3D (D = 3 forms of the GPTT cell kernel and of BDF2)
    "gptt3d_log": (lambda: refpy.cavity(3, 5, Re=1.0, dt=1e-4, flowtype=hp.VISCOELASTIC, ve_model=hp.GPTT,
                                        kernel=hp.KERNEL_LOG, beta=1.0 / 9.0, De=0.5, epsilon=0.3, xi=0.1,
                                        alpha_gptt=0.8, beta_gptt=1.2), 3, (0.3, 0.1, 0.2)),
    "bdf2_cav3d": (lambda: refpy.cavity(3, 6, Re=0.1, dt=1e-3, tempdiscrtype=hp.SEMI_IMPLICIT_BDF2),
                   3, (0.3, 0.1, 0.0)),
    # semi-implicit BDF2 (two solves per direction: into uaux, then into u*)
    "bdf2_cav2d": (lambda: refpy.cavity(2, 16, Re=0.1, dt=1e-3, tempdiscrtype=hp.SEMI_IMPLICIT_BDF2),
                   4, (0.3, 0.1, 0.0)),
    "bdf2_oldroyd_log": (lambda: refpy.cavity(2, 12, Re=0.01, dt=1e-3, flowtype=hp.VISCOELASTIC,
                                              ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG, beta=1.0 / 9.0,
                                              tempdiscrtype=hp.SEMI_IMPLICIT_BDF2), 3, (0.3, 0.1, 0.2)),
    "amr2d_sie_oldroyd": (lambda: refpy.cavity(2, 12, Re=0.01, dt=1e-3, flowtype=hp.VISCOELASTIC,
                                               ve_model=hp.OLDROYD_B, kernel=hp.KERNEL_LOG, beta=1.0 / 9.0,
                                               tempdiscrtype=hp.SEMI_IMPLICIT_EULER,
                                               refine=[([0.5 / 12, 0.5 / 12], [((6, 6), (12, 12))])]),
                          3, (0.3, 0.1, 0.2)),
}


def field_keys(dim: int, ve: bool):
    keys = [(f"u{d}", hp.FIELD_U, d) for d in range(dim)] + [("p", hp.FIELD_P, 0), ("dp", hp.FIELD_DP, 0)]
    if ve:
        keys += [(f"K{k}", hp.FIELD_KERNEL, k) for k in range(dim * dim)]
        keys += [(f"S{k}", hp.FIELD_S, k) for k in range(dim * dim)]
    return keys


def make(name: str, seed: int = 0) -> None:
    factory, steps, (au, ap, ak) = CASES[name]
    spec = factory()
    c = refpy.RefCase(spec)
    dim = c.dim
    ve = spec.flowtype == hp.VISCOELASTIC
    rng = np.random.default_rng(seed)
    for d in range(dim):
        if au:
            c.set(hp.FIELD_U, d, au * rng.standard_normal(c.nfacet[d]))
    if ap:
        c.set(hp.FIELD_P, 0, ap * rng.standard_normal(c.ncell))
    if ve and ak:
        for i in range(dim):
            for j in range(i, dim):
                v = ak * rng.standard_normal(c.ncell)
                if spec.par.get("kernel", hp.KERNEL_LOG) != hp.KERNEL_LOG and i == j:
                    v = 1.0 + 0.5 * np.abs(v)   # identity/sqrt kernels need a positive-definite start
                c.set(hp.FIELD_KERNEL, i * dim + j, v)
                c.set(hp.FIELD_KERNEL, j * dim + i, v)
    prog = c.flatten()
    out = {"steps": np.int64(steps), "dim": np.int64(dim)}
    for key, fid, comp in field_keys(dim, ve):
        out["init_" + key] = c.get(fid, comp)
    c.step(steps)
    for key, fid, comp in field_keys(dim, ve):
        out["ref_" + key] = c.get(fid, comp)
    it, res = c.solver_stats()
    out["ref_last_iters"] = np.int64(it)
    prog.save(os.path.join(HERE, f"{name}.prog.npz"))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    c.close()
    print(f"{name}: ncell={prog.ncell} nfacet={prog.nfacet[:dim]} rows={prog.row_rhs.size} steps={steps}")


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        make(n)

/*
 * Oracle harness around the reference HigFlow library (test infrastructure:
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm only).
 *
 * Cases are built by the drop-in host's builder (hfh_build,
 * higflow_b200/host/hf_host.c), the way a HigFlow main program does
 * (higflow/example2d_Newt/ns-example-2d.c:159-230), from legacy text inputs.
 * This file adds what only the checker needs: the reference's own CPU time
 * step (with the CPU Poisson engine of oracle/solver_cpu.c), its fields, its
 * phase timers, CFL and adaptive step, through a small C API for ctypes.
 */
#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "hig-flow-kernel.h"
#include "hig-flow-ic.h"
#include "hig-flow-bc.h"
#include "hig-flow-timestep.h"
#include "hig-flow-step.h"
#include "hig-flow-step-viscoelastic.h"
#include "hig-flow-step-generalized-newtonian.h"
#include "higflow_b200.h"
#include "higflow_b200_higflow.h"

#include "hf_host.h"

/* The case description is the host's (higflow_b200/host/hf_host.h): the
 * oracle builds its cases with the drop-in host's own builder, hfh_build, and
 * adds the reference's CPU step, field access and phase timers. */
typedef hfh_params hfref_params;

typedef struct hfref_case {
    higflow_solver *ns;
    double t_velocity, t_pressure, t_final, t_ve, t_total;
} hfref_case;

extern double hfref_solve_seconds;
extern int hfref_solve_iters;

static void quiet_begin(void) { hfh_quiet_begin(); }
static void quiet_end(void) { hfh_quiet_end(); }

void hfref_set_quiet(int on) { hfh_set_quiet(on); }

static double now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int hfref_dim(void) { return DIM; }

int hfref_create(const char *nameload, const hfref_params *p, hfref_case **out)
{
    hfref_case *C = calloc(1, sizeof *C);
    if (!C) return -1;
    int rc = hfh_build(nameload, p, &C->ns);
    if (rc != 0) {
        free(C);
        return rc;
    }
    *out = C;
    return 0;
}

int hfref_sizes(hfref_case *C, int32_t *ncell, int32_t *nfacet)
{
    higflow_solver *ns = C->ns;
    *ncell = psd_get_local_domain_size(ns->psdp);
    for (int d = 0; d < DIM; d++) nfacet[d] = psfd_get_local_domain_size(ns->psfdu[d]);
    return 0;
}

static distributed_property *field(hfref_case *C, int which, int comp)
{
    higflow_solver *ns = C->ns;
    int i = comp / DIM, j = comp % DIM;
    switch (which) {
    case HF_FIELD_U: return comp < DIM ? ns->dpu[comp] : NULL;
    case HF_FIELD_USTAR: return comp < DIM ? ns->dpustar[comp] : NULL;
    case HF_FIELD_P: return ns->dpp;
    case HF_FIELD_DP: return ns->ddeltap;
    case HF_FIELD_F: return ns->dpF;
    case HF_FIELD_FU: return comp < DIM ? ns->dpFU[comp] : NULL;
    case HF_FIELD_KERNEL: return ns->contr.flowtype == VISCOELASTIC ? ns->ed.ve.dpKernel[i][j] : NULL;
    case HF_FIELD_S: return ns->contr.flowtype == VISCOELASTIC ? ns->ed.ve.dpS[i][j] : NULL;
    case HF_FIELD_DU: return ns->contr.flowtype == VISCOELASTIC ? ns->ed.ve.dpD[i][j] : NULL;
    }
    return NULL;
}

static int field_size(hfref_case *C, int which, int comp)
{
    higflow_solver *ns = C->ns;
    if (which == HF_FIELD_U || which == HF_FIELD_USTAR || which == HF_FIELD_FU)
        return psfd_get_local_domain_size(ns->psfdu[comp]);
    return psd_get_local_domain_size(ns->psdp);
}

int hfref_get_field(hfref_case *C, int32_t which, int32_t comp, double *out, int64_t n)
{
    distributed_property *dp = field(C, which, comp);
    if (!dp || n != field_size(C, which, comp)) return -1;
    for (int64_t k = 0; k < n; k++) out[k] = dp_get_value(dp, (int)k);
    return 0;
}

int hfref_set_field(hfref_case *C, int32_t which, int32_t comp, const double *in, int64_t n)
{
    distributed_property *dp = field(C, which, comp);
    if (!dp || n != field_size(C, which, comp)) return -1;
    for (int64_t k = 0; k < n; k++) dp_set_value(dp, (int)k, in[k]);
    return 0;
}

/* centres of cells (ncell*DIM) or facets normal to d (nfacet[d]*DIM), indexed by local id */
int hfref_centers(hfref_case *C, int32_t facet_dim, double *out)
{
    higflow_solver *ns = C->ns;
    if (facet_dim < 0) {
        sim_domain *sd = psd_get_local_domain(ns->psdp);
        mp_mapper *m = sd_get_domain_mapper(sd);
        higcit_celliterator *it;
        for (it = sd_get_domain_celliterator(sd); !higcit_isfinished(it); higcit_nextcell(it)) {
            hig_cell *c = higcit_getcell(it);
            int id = mp_lookup(m, hig_get_cid(c));
            Point x;
            hig_get_center(c, x);
            for (int k = 0; k < DIM; k++) out[id * DIM + k] = x[k];
        }
        higcit_destroy(it);
    } else {
        sim_facet_domain *sfd = psfd_get_local_domain(ns->psfdu[facet_dim]);
        mp_mapper *m = sfd_get_domain_mapper(sfd);
        higfit_facetiterator *fit;
        for (fit = sfd_get_domain_facetiterator(sfd); !higfit_isfinished(fit); higfit_nextfacet(fit)) {
            hig_facet *f = higfit_getfacet(fit);
            int id = mp_lookup(m, hig_get_fid(f));
            Point x;
            hig_get_facet_center(f, x);
            for (int k = 0; k < DIM; k++) out[id * DIM + k] = x[k];
        }
        higfit_destroy(fit);
    }
    return 0;
}

/* The reference's own step (higflow_solver_step / _viscoelastic), nsteps times,
 * with the time update of the case main loop (ns-example-2d.c:246-248). */
int hfref_step(hfref_case *C, int32_t nsteps, double *seconds)
{
    hfh_select(C->ns);
    higflow_solver *ns = C->ns;
    quiet_begin();
    double t0 = now();
    for (int s = 0; s < nsteps; s++) {
        if (ns->contr.flowtype == VISCOELASTIC) higflow_solver_step_viscoelastic(ns);
        else higflow_solver_step(ns);
        ns->par.t += ns->par.dt;
        ns->par.step++;
    }
    double el = now() - t0;
    quiet_end();
    C->t_total += el;
    if (seconds) *seconds = el;
    return 0;
}

/* The same step with per-phase timers: the sub-steps are called in the order of
 * higflow_solver_step (hig-flow-step.c:1363-1413) and
 * higflow_solver_step_viscoelastic (hig-flow-step-viscoelastic.c:2091-2163).
 * times[0..4] += velocity, pressure (assembly+solve), of which solve,
 * final velocity+pressure, viscoelastic (Du+constitutive+polymeric). */
int hfref_step_phased(hfref_case *C, int32_t nsteps, double *times)
{
    hfh_select(C->ns);
    higflow_solver *ns = C->ns;
    const int ve = ns->contr.flowtype == VISCOELASTIC;
    quiet_begin();
    for (int s = 0; s < nsteps; s++) {
        double a = now();
        if (ve) {
            higflow_compute_velocity_derivative_tensor(ns);
            higflow_explicit_euler_constitutive_equation(ns);
            higflow_compute_polymeric_tensor(ns);
        }
        double b = now();
        higflow_boundary_condition_for_velocity(ns);
        higflow_boundary_condition_for_cell_source_term(ns);
        higflow_boundary_condition_for_facet_source_term(ns);
        higflow_boundary_condition_for_pressure(ns);
        higflow_calculate_source_term(ns);
        higflow_calculate_facet_source_term(ns);
        if (ve) higflow_explicit_euler_intermediate_velocity_viscoelastic(ns, ns->dpu, ns->dpustar);
        else higflow_explicit_euler_intermediate_velocity(ns, ns->dpu, ns->dpustar);
        double c = now();
        double s0 = hfref_solve_seconds;
        higflow_pressure(ns);
        double d = now();
        higflow_final_velocity(ns);
        higflow_final_pressure(ns);
        double e = now();
        ns->par.t += ns->par.dt;
        ns->par.step++;
        times[0] += c - b;
        times[1] += d - c;
        times[2] += hfref_solve_seconds - s0;
        times[3] += e - d;
        times[4] += b - a;
    }
    quiet_end();
    return 0;
}

int hfref_solver_stats(hfref_case *C, int32_t *iters, double *residual)
{
    solver *s = C->ns->slvp;
    *iters = s->SolverIterations;
    *residual = s->SolverResidual;
    return 0;
}

double hfref_time(hfref_case *C) { return C->ns->par.t; }

/* the case's higflow_solver, for the drop-in binding (hf_attach & co.) */
void *hfref_ns(hfref_case *C) { return C->ns; }

/* the case's current time step (ns->par.dt), and the reference's own CFL
 * number and adaptive step on its state (hig-flow-timestep.c:7-40, :115-139;
 * both print through print0f, silenced here like the rest of the harness) */
double hfref_dt(hfref_case *C) { return C->ns->par.dt; }

/* a host-side change of the time step (as a case main loop or a restart makes) */
void hfref_set_dt(hfref_case *C, double dt) { C->ns->par.dt = dt; }

double hfref_cfl(hfref_case *C)
{
    hfh_select(C->ns);
    return higflow_compute_CFL(C->ns);
}

void hfref_adjust_timestep(hfref_case *C)
{
    hfh_select(C->ns);
    higflow_adjust_timestep(C->ns);
}

/* flatten through the binding (hf_flatten) and hand the program to Python */
int hfref_flatten(hfref_case *C, hf_program **out)
{
    hfh_select(C->ns);
    quiet_begin();
    int rc = hf_flatten(C->ns, out);
    quiet_end();
    return rc;
}

void hfref_program_free(hf_program *p) { hf_program_free(p); }

const char *hfref_flatten_error(void) { return hf_flatten_error(); }

void hfref_destroy(hfref_case *C)
{
    if (!C) return;
    hfh_destroy(C->ns);
    free(C);
}

/*
 * Oracle harness around the reference HigFlow library (test infrastructure:
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm only).
 *
 * Builds a case the way a HigFlow main program does
 * (higflow/example2d_Newt/ns-example-2d.c:159-230), but from the legacy text
 * inputs (<name>.domain, <name>.bc, read by higflow_initialize_domain,
 * hig-flow-ic.c:11, and higflow_initialize_boundaries, hig-flow-bc.c:572) and
 * with the controllers filled directly instead of from YAML.  It then exposes
 * the reference's own time step and its fields through a small C API for
 * ctypes.  Boundary and initial values come from the callback tables below,
 * parameterised per boundary id.
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

#define HFREF_MAXBC 16

/* Case description passed from Python (all doubles/ints, no pointers). */
typedef struct hfref_params {
    int32_t flowtype, projtype, convecdiscrtype, secondconvecdiscrtype;
    int32_t ve_model, ve_convecdiscrtype, kernel;  /* kernel: HF_KERNEL_* */
    int32_t nbc;
    double Re, dt, t0;
    double De, beta, kernel_tol, alpha, epsilon, xi;
    /* boundary velocity for bc id b, component d:
     *   bc_u[b][d] + bc_upar[b][d] * (1 - ((x[bc_tdim[b]] - bc_c[b]) / bc_h[b])^2) */
    double bc_u[HFREF_MAXBC][3];
    double bc_upar[HFREF_MAXBC][3];
    int32_t bc_tdim[HFREF_MAXBC];
    double bc_c[HFREF_MAXBC], bc_h[HFREF_MAXBC];
    double bc_p[HFREF_MAXBC];
    double k_init[3][3];        /* initial kernel tensor (get_tensor) */
    int32_t tempdiscrtype;      /* HF_EXPLICIT_EULER / HF_SEMI_IMPLICIT_EULER */
    int32_t pad_;
    double L2_fene, lambda_fene, E_fene;
    int32_t ve_discrtype;       /* HF_VE_EXPLICIT / HF_VE_IMPLICIT */
    int32_t pad2_;
    double alpha_gptt, beta_gptt;
} hfref_params;

typedef struct hfref_case {
    higflow_solver *ns;
    hfref_params par;
    char nameload[1024];
    double t_velocity, t_pressure, t_final, t_ve, t_total;
} hfref_case;

static hfref_case *g_cur;
extern double hfref_solve_seconds;
extern int hfref_solve_iters;

/* ---- callbacks (signatures of higflow_functions, hig-flow-kernel.h:217-234) ---- */
static real cb_get_pressure(Point center, real t) { (void)center; (void)t; return 0.0; }
static real cb_get_velocity(Point center, int dim, real t) { (void)center; (void)dim; (void)t; return 0.0; }
static real cb_get_source_term(Point center, real t) { (void)center; (void)t; return 0.0; }
static real cb_get_facet_source_term(Point center, int dim, real t) { (void)center; (void)dim; (void)t; return 0.0; }
static real cb_get_boundary_pressure(int id, Point center, real t)
{
    (void)center; (void)t;
    if (id < 0 || id >= HFREF_MAXBC) return 0.0;
    return g_cur->par.bc_p[id];
}
static real cb_get_boundary_velocity(int id, Point center, int dim, real t)
{
    (void)t;
    if (id < 0 || id >= HFREF_MAXBC) return 0.0;
    const hfref_params *p = &g_cur->par;
    real v = p->bc_u[id][dim];
    if (p->bc_upar[id][dim] != 0.0) {
        real s = (center[p->bc_tdim[id]] - p->bc_c[id]) / p->bc_h[id];
        v += p->bc_upar[id][dim] * (1.0 - s * s);
    }
    return v;
}
static real cb_get_boundary_source_term(int id, Point center, real t) { (void)id; (void)center; (void)t; return 0.0; }
static real cb_get_boundary_facet_source_term(int id, Point center, int dim, real t) { (void)id; (void)center; (void)dim; (void)t; return 0.0; }

/* kernel-conformation transforms (commented variants in
 * higflow/example2d_Oldroyd/ns-example-2d.c:21-56) */
static real cb_get_tensor(Point center, int i, int j, real t) { (void)center; (void)t; return g_cur->par.k_init[i][j]; }
static real cb_get_kernel(int dim, real lambda, real tol)
{
    (void)dim;
    switch (g_cur->par.kernel) {
    case HF_KERNEL_LOG: return lambda < tol ? log(tol) : log(lambda);
    case HF_KERNEL_SQRT: return lambda < tol ? sqrt(tol) : sqrt(lambda);
    default: return lambda;
    }
}
static real cb_get_kernel_inverse(int dim, real lambda, real tol)
{
    (void)dim; (void)tol;
    switch (g_cur->par.kernel) {
    case HF_KERNEL_LOG: return exp(lambda);
    case HF_KERNEL_SQRT: return lambda * lambda;
    default: return lambda;
    }
}
static real cb_get_kernel_jacobian(int dim, real lambda, real tol)
{
    (void)dim;
    switch (g_cur->par.kernel) {
    case HF_KERNEL_LOG: return lambda < tol ? 1.0 / tol : 1.0 / lambda;
    case HF_KERNEL_SQRT: return lambda < tol ? 0.5 / sqrt(tol) : 0.5 / sqrt(lambda);
    default: return 1.0;
    }
}

static int g_initialized;
static int g_quiet = 1;
static int g_saved_stdout = -1;

static void quiet_begin(void)
{
    if (!g_quiet) return;
    fflush(stdout);
    g_saved_stdout = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
}

static void quiet_end(void)
{
    if (!g_quiet || g_saved_stdout < 0) return;
    fflush(stdout);
    dup2(g_saved_stdout, 1);
    close(g_saved_stdout);
    g_saved_stdout = -1;
}

void hfref_set_quiet(int on) { g_quiet = on; }

static double now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int hfref_dim(void) { return DIM; }

int hfref_create(const char *nameload, const hfref_params *p, hfref_case **out)
{
    if (!g_initialized) {
        int argc = 1;
        static char *argv0[] = {"hfref", NULL};
        char **argv = argv0;
        int myrank, ntasks;
        higflow_initialize(&argc, &argv, &myrank, &ntasks);
        g_initialized = 1;
    }
    hfref_case *C = calloc(1, sizeof *C);
    C->par = *p;
    snprintf(C->nameload, sizeof C->nameload, "%s", nameload);
    g_cur = C;
    quiet_begin();

    higflow_solver *ns = higflow_create();
    memset(ns, 0, sizeof *ns);
    C->ns = ns;
    ns->par.nameload = C->nameload;
    ns->par.namesave = C->nameload;
    ns->par.nameprint = C->nameload;
    ns->par.Re = p->Re;
    ns->par.dt = p->dt;
    ns->par.dt0 = p->dt;
    ns->par.t = p->t0;
    ns->par.step = 0;
    ns->par.initstep = 0;
    ns->par.finalstep = 1 << 30;
    ns->par.ts = 1e30;
    ns->par.tp = 1e30;
    ns->contr.projtype = p->projtype;
    ns->contr.flowtype = p->flowtype;
    ns->contr.eoflow = false;
    ns->contr.tempdiscrtype = p->tempdiscrtype == HF_SEMI_IMPLICIT_EULER ? SEMI_IMPLICIT_EULER
                              : p->tempdiscrtype == HF_SEMI_IMPLICIT_CN ? SEMI_IMPLICIT_CN
                              : p->tempdiscrtype == HF_SEMI_IMPLICIT_BDF2 ? SEMI_IMPLICIT_BDF2
                              : p->tempdiscrtype == HF_EXPLICIT_RK2 ? EXPLICIT_RK2
                              : p->tempdiscrtype == HF_EXPLICIT_RK3 ? EXPLICIT_RK3 : EXPLICIT_EULER;
    ns->contr.spatialdiscrtype = ORDER2;
    ns->contr.convecdiscrtype = p->convecdiscrtype;
    ns->contr.secondconvecdiscrtype = p->secondconvecdiscrtype;
    if (p->flowtype == VISCOELASTIC) {
        ns->ed.ve.contr.model = p->ve_model;
        ns->ed.ve.contr.discrtype = p->ve_discrtype == HF_VE_IMPLICIT ? IMPLICIT : EXPLICIT;
        ns->ed.ve.contr.convecdiscrtype = p->ve_convecdiscrtype;
        ns->ed.ve.par.De = p->De;
        ns->ed.ve.par.beta = p->beta;
        ns->ed.ve.par.kernel_tol = p->kernel_tol;
        ns->ed.ve.par.alpha = p->alpha;
        ns->ed.ve.par.epsilon = p->epsilon;
        ns->ed.ve.par.xi = p->xi;
        ns->ed.ve.par.L2_fene = p->L2_fene;
        ns->ed.ve.par.lambda_fene = p->lambda_fene;
        ns->ed.ve.par.E_fene = p->E_fene;
        ns->ed.ve.par.alpha_gptt = p->alpha_gptt;
        ns->ed.ve.par.beta_gptt = p->beta_gptt;
    }

    higflow_set_external_functions(ns, cb_get_pressure, cb_get_velocity, cb_get_source_term,
                                   cb_get_facet_source_term, cb_get_boundary_pressure,
                                   cb_get_boundary_velocity, cb_get_boundary_source_term,
                                   cb_get_boundary_facet_source_term);
    const int cache = 1, order = 2;
    higflow_create_domain(ns, cache, order);
    if (p->flowtype == VISCOELASTIC)
        higflow_create_domain_viscoelastic(ns, cache, order, cb_get_tensor, cb_get_kernel,
                                           cb_get_kernel_inverse, cb_get_kernel_jacobian);
    higflow_initialize_domain(ns, 1, 0, order);
    higflow_initialize_boundaries(ns);
    higflow_create_distributed_properties(ns);
    higflow_initialize_distributed_properties(ns);
    higflow_create_solver(ns);
    quiet_end();
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
    g_cur = C;
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
    g_cur = C;
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

double hfref_cfl(hfref_case *C)
{
    g_cur = C;
    return higflow_compute_CFL(C->ns);
}

void hfref_adjust_timestep(hfref_case *C)
{
    g_cur = C;
    higflow_adjust_timestep(C->ns);
}

/* flatten through the binding (hf_flatten) and hand the program to Python */
int hfref_flatten(hfref_case *C, hf_program **out)
{
    g_cur = C;
    quiet_begin();
    int rc = hf_flatten(C->ns, out);
    quiet_end();
    return rc;
}

void hfref_program_free(hf_program *p) { hf_program_free(p); }

const char *hfref_flatten_error(void) { return hf_flatten_error(); }

void hfref_destroy(hfref_case *C)
{
    /* higflow_destroy releases everything the case created; the partition
     * graph and trees are leaked by the reference itself and live until exit */
    if (!C) return;
    g_cur = C;
    quiet_begin();
    higflow_destroy(C->ns);
    quiet_end();
    free(C);
}

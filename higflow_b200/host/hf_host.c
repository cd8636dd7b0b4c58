/*
 * HigFlow host of the drop-in (declarations and contract in hf_host.h).
 *
 * hfh_build follows a case main program (higflow/example2d_Newt/
 * ns-example-2d.c:159-230): controllers and parameters are filled directly
 * instead of from YAML, the mesh and boundaries come from the legacy text
 * inputs, and the callbacks below play the part of the case file's functions
 * (signatures of higflow_functions, hig-flow-kernel.h:217-234), parameterised
 * per boundary id by hfh_params.
 */
#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "hig-flow-kernel.h"
#include "hig-flow-ic.h"
#include "hig-flow-bc.h"
#include "hf_host.h"
#include "higflow_b200_higflow.h"

#define HFH_MAXCASES 256

typedef struct hfh_case {
    higflow_solver *ns;
    hfh_params par;
    char nameload[1024];
} hfh_case;

static hfh_case *g_cases[HFH_MAXCASES];
static hfh_case *g_cur;
static char g_err[512];
static int g_initialized;
static int g_quiet = 1;
static int g_saved_stdout = -1;

const char *hfh_error(void) { return g_err; }
int hfh_dim(void) { return DIM; }
void hfh_set_quiet(int on) { g_quiet = on; }

/* nested begin/end pairs: stdout comes back at the outermost end */
static int g_quiet_depth;

void hfh_quiet_begin(void)
{
    if (g_quiet_depth++ > 0 || !g_quiet) return;
    fflush(stdout);
    g_saved_stdout = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
}

void hfh_quiet_end(void)
{
    if (g_quiet_depth > 0 && --g_quiet_depth > 0) return;
    if (g_saved_stdout < 0) return;
    fflush(stdout);
    dup2(g_saved_stdout, 1);
    close(g_saved_stdout);
    g_saved_stdout = -1;
}

/* ---- callbacks ---- */
static real cb_get_pressure(Point center, real t) { (void)center; (void)t; return 0.0; }
static real cb_get_velocity(Point center, int dim, real t) { (void)center; (void)dim; (void)t; return 0.0; }
static real cb_get_source_term(Point center, real t) { (void)center; return g_cur->par.src_t * t; }
static real cb_get_facet_source_term(Point center, int dim, real t) { (void)center; (void)dim; (void)t; return 0.0; }
static real cb_get_boundary_pressure(int id, Point center, real t)
{
    (void)center; (void)t;
    if (id < 0 || id >= HFH_MAXBC) return 0.0;
    return g_cur->par.bc_p[id];
}
static real cb_get_boundary_velocity(int id, Point center, int dim, real t)
{
    (void)t;
    if (id < 0 || id >= HFH_MAXBC) return 0.0;
    const hfh_params *p = &g_cur->par;
    real v = p->bc_u[id][dim];
    if (p->bc_upar[id][dim] != 0.0) {
        real s = (center[p->bc_tdim[id]] - p->bc_c[id]) / p->bc_h[id];
        v += p->bc_upar[id][dim] * (1.0 - s * s);
    }
    return v;
}
static real cb_get_boundary_source_term(int id, Point center, real t) { (void)id; (void)center; (void)t; return 0.0; }
static real cb_get_boundary_facet_source_term(int id, Point center, int dim, real t)
{
    (void)id; (void)center; (void)dim; (void)t;
    return 0.0;
}

/* kernel-conformation transforms (the identity of the shipped case file and
 * its commented log/sqrt variants, higflow/example2d_Oldroyd/ns-example-2d.c:
 * 21-56) */
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

static hfh_case *find(struct higflow_solver *ns)
{
    for (int k = 0; k < HFH_MAXCASES; k++)
        if (g_cases[k] && g_cases[k]->ns == ns) return g_cases[k];
    return NULL;
}

void hfh_select(struct higflow_solver *ns)
{
    hfh_case *c = find(ns);
    if (c) g_cur = c;
}

static int tempdiscr(int32_t t)
{
    switch (t) {
    case HF_SEMI_IMPLICIT_EULER: return SEMI_IMPLICIT_EULER;
    case HF_SEMI_IMPLICIT_CN: return SEMI_IMPLICIT_CN;
    case HF_SEMI_IMPLICIT_BDF2: return SEMI_IMPLICIT_BDF2;
    case HF_EXPLICIT_RK2: return EXPLICIT_RK2;
    case HF_EXPLICIT_RK3: return EXPLICIT_RK3;
    default: return EXPLICIT_EULER;
    }
}

int hfh_build(const char *nameload, const hfh_params *p, struct higflow_solver **ns_out)
{
    int slot = -1;
    for (int k = 0; k < HFH_MAXCASES && slot < 0; k++)
        if (!g_cases[k]) slot = k;
    if (slot < 0) {
        snprintf(g_err, sizeof g_err, "hfh_build: more than %d live cases", HFH_MAXCASES);
        return HF_ERR_INVALID;
    }
    if (p->nbc < 0 || p->nbc > HFH_MAXBC) {
        snprintf(g_err, sizeof g_err, "hfh_build: %d boundaries (at most %d)", p->nbc, HFH_MAXBC);
        return HF_ERR_INVALID;
    }
    if (!g_initialized) {
        int argc = 1;
        static char *argv0[] = {"higflow_b200_host", NULL};
        char **argv = argv0;
        int myrank, ntasks;
        higflow_initialize(&argc, &argv, &myrank, &ntasks);
        g_initialized = 1;
    }
    hfh_case *C = calloc(1, sizeof *C);
    if (!C) {
        snprintf(g_err, sizeof g_err, "hfh_build: out of host memory");
        return HF_ERR_INVALID;
    }
    C->par = *p;
    snprintf(C->nameload, sizeof C->nameload, "%s", nameload);
    g_cases[slot] = C;
    g_cur = C;
    hfh_quiet_begin();

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
    ns->contr.tempdiscrtype = tempdiscr(p->tempdiscrtype);
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
    hfh_quiet_end();
    *ns_out = ns;
    return HF_OK;
}

void hfh_destroy(struct higflow_solver *ns)
{
    /* higflow_destroy releases what the case created; the partition graph and
     * trees are leaked by the reference itself and live until exit */
    for (int k = 0; k < HFH_MAXCASES; k++) {
        if (!g_cases[k] || g_cases[k]->ns != ns) continue;
        g_cur = g_cases[k];
        hfh_quiet_begin();
        higflow_destroy(ns);
        hfh_quiet_end();
        free(g_cases[k]);
        g_cases[k] = NULL;
        g_cur = NULL;
        return;
    }
}

int hfh_record(const char *nameload, const hfh_params *p, hf_program **out)
{
    struct higflow_solver *ns = NULL;
    int rc = hfh_build(nameload, p, &ns);
    if (rc != HF_OK) return rc;
    hfh_select(ns);
    hfh_quiet_begin();
    rc = hf_flatten(ns, out);
    hfh_quiet_end();
    if (rc != HF_OK) snprintf(g_err, sizeof g_err, "hf_flatten: %s", hf_flatten_error());
    hfh_destroy(ns);
    return rc;
}

void hfh_program_free(hf_program *prog) { hf_program_free(prog); }

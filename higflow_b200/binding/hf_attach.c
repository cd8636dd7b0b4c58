/*
 * Step-level drop-in: HigFlow's own solver object (higflow_solver,
 * higflow/src/hig-flow-kernel.h:1142-1194) driven by the GPU engine.
 *
 * Compiled like hf_flatten.c against HigFlow's headers (-DDIM=2 or 3) and
 * linked with libhigflow_b200.so ahead of libhigflow.  A case main loop
 * (e.g. higflow/example2d_Newt/ns-example-2d.c:246, example2d_Oldroyd/
 * ns-example-2d.c:471) keeps calling
 *     higflow_solver_step(ns)  /  higflow_solver_step_viscoelastic(ns)
 * and is linked with -Wl,--wrap=higflow_solver_step and
 * -Wl,--wrap=higflow_solver_step_viscoelastic, so those calls land in the
 * __wrap_ functions below: the first call attaches (flattens the step,
 * uploads program and fields), every call runs one GPU step, and the fields go
 * back into ns->dp*->values whenever the loop is about to print or save (its
 * tests t >= tp, t >= ts after t += dt).
 *
 * Ownership: ns owns the host arrays; the engine owns the device copies,
 * which are authoritative between hf_attach and the next hf_sync_to_host.
 * One host thread per ns (HigTree's stencil code is not reentrant); several ns
 * may be attached, each to its own engine case.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hig-flow-kernel.h"
#include "hig-flow-step.h"
#include "higflow_b200.h"
#include "higflow_b200_higflow.h"

#define HF_MAX_ATTACHED 64

typedef struct hf_binding {
    higflow_solver *ns;
    hf_case *c;
    int ve;
} hf_binding;

static hf_binding g_bind[HF_MAX_ATTACHED];

static hf_binding *find(higflow_solver *ns)
{
    for (int k = 0; k < HF_MAX_ATTACHED; k++)
        if (g_bind[k].ns == ns) return &g_bind[k];
    return NULL;
}

/* the reference's field behind an engine field id (cells or facets, by id) */
static distributed_property *field_of(higflow_solver *ns, int field, int comp)
{
    const int i = comp / DIM, j = comp % DIM;
    const int ve = ns->contr.flowtype == VISCOELASTIC;
    switch (field) {
    case HF_FIELD_U: return ns->dpu[comp];
    case HF_FIELD_USTAR: return ns->dpustar[comp];
    case HF_FIELD_P: return ns->dpp;
    case HF_FIELD_DP: return ns->ddeltap;
    case HF_FIELD_F: return ns->dpF;
    case HF_FIELD_FU: return ns->dpFU[comp];
    case HF_FIELD_KERNEL: return ve ? ns->ed.ve.dpKernel[i][j] : NULL;
    case HF_FIELD_S: return ve ? ns->ed.ve.dpS[i][j] : NULL;
    case HF_FIELD_DU: return ve ? ns->ed.ve.dpD[i][j] : NULL;
    }
    return NULL;
}

static int field_len(higflow_solver *ns, int field, int comp)
{
    if (field == HF_FIELD_U || field == HF_FIELD_USTAR || field == HF_FIELD_FU)
        return psfd_get_local_domain_size(ns->psfdu[comp]);
    return psd_get_local_domain_size(ns->psdp);
}

/* the fields a step reads (state and sources), copied in at attach */
static const int k_in[][2] = {{HF_FIELD_U, DIM}, {HF_FIELD_P, 1}, {HF_FIELD_DP, 1}, {HF_FIELD_F, 1},
                              {HF_FIELD_FU, DIM}, {HF_FIELD_KERNEL, DIM * DIM}, {HF_FIELD_S, DIM * DIM}};
/* the fields a step writes, copied back at sync */
static const int k_out[][2] = {{HF_FIELD_U, DIM}, {HF_FIELD_USTAR, DIM}, {HF_FIELD_P, 1}, {HF_FIELD_DP, 1},
                               {HF_FIELD_KERNEL, DIM * DIM}, {HF_FIELD_S, DIM * DIM}, {HF_FIELD_DU, DIM * DIM}};

static int copy_fields(hf_binding *b, const int (*list)[2], int nlist, int to_device)
{
    higflow_solver *ns = b->ns;
    int rc = HF_OK;
    double *buf = NULL;
    for (int e = 0; e < nlist && rc == HF_OK; e++) {
        const int field = list[e][0];
        if (!b->ve && (field == HF_FIELD_KERNEL || field == HF_FIELD_S || field == HF_FIELD_DU)) continue;
        for (int comp = 0; comp < list[e][1] && rc == HF_OK; comp++) {
            distributed_property *dp = field_of(ns, field, comp);
            if (!dp) continue;
            const int n = field_len(ns, field, comp);
            double *nb = realloc(buf, sizeof(double) * (n > 0 ? n : 1));
            if (!nb) { rc = HF_ERR_INVALID; break; }
            buf = nb;
            if (to_device) {
                for (int k = 0; k < n; k++) buf[k] = dp_get_value(dp, k);
                rc = hf_case_set_field(b->c, field, comp, buf, n);
            } else {
                rc = hf_case_get_field(b->c, field, comp, buf, n);
                if (rc == HF_OK) {
                    for (int k = 0; k < n; k++) dp_set_value(dp, k, buf[k]);
                    dp_sync(dp);
                }
            }
        }
    }
    free(buf);
    return rc;
}

/* The source fields (cell F and facet FU[d]) as the reference computes them
 * at time t, appended to out (grown as needed). */
static int sources_at(higflow_solver *ns, real t, double **out, size_t *len)
{
    const real t0 = ns->par.t;
    ns->par.t = t;
    higflow_calculate_source_term(ns);
    higflow_calculate_facet_source_term(ns);
    ns->par.t = t0;
    size_t n = 0;
    for (int f = 0; f <= DIM; f++) n += f == 0 ? field_len(ns, HF_FIELD_F, 0) : field_len(ns, HF_FIELD_FU, f - 1);
    double *v = realloc(*out, sizeof(double) * (n ? n : 1));
    if (!v) return HF_ERR_INVALID;
    *out = v;
    *len = n;
    size_t at = 0;
    for (int f = 0; f <= DIM; f++) {
        distributed_property *dp = f == 0 ? ns->dpF : ns->dpFU[f - 1];
        const int m = f == 0 ? field_len(ns, HF_FIELD_F, 0) : field_len(ns, HF_FIELD_FU, f - 1);
        for (int k = 0; k < m; k++) v[at++] = dp_get_value(dp, k);
    }
    return HF_OK;
}

/* Refuse source callbacks that depend on time: the sources are evaluated at
 * the case's current time and at two later times (a step and a long span
 * ahead) and must agree bit for bit. */
static int check_sources_fixed(higflow_solver *ns)
{
    double *a = NULL, *b = NULL;
    size_t na = 0, nb = 0;
    const real t = ns->par.t, later[2] = {t + ns->par.dt, t + 1000.0 * ns->par.dt + 1.0};
    int rc = sources_at(ns, t, &a, &na);
    for (int k = 0; k < 2 && rc == HF_OK; k++) {
        rc = sources_at(ns, later[k], &b, &nb);
        if (rc == HF_OK && (nb != na || memcmp(a, b, sizeof(double) * na) != 0)) rc = HF_ERR_UNSUPPORTED;
    }
    free(a);
    free(b);
    return rc;
}

int hf_attach(higflow_solver *ns, const hf_options *opt)
{
    if (!ns) return HF_ERR_INVALID;
    if (find(ns)) return HF_OK;
    hf_binding *b = find(NULL);
    if (!b) return HF_ERR_UNSUPPORTED;
    hf_program *prog = NULL;
    int rc = hf_flatten(ns, &prog);
    if (rc) return rc;
    /* the GPU path keeps the source terms fixed (see below): refuse source
     * callbacks that depend on t before any device work */
    rc = check_sources_fixed(ns);
    if (rc) {
        hf_program_free(prog);
        return rc;
    }
    hf_case *c = NULL;
    rc = hf_case_create(prog, opt, &c);
    hf_program_free(prog);   /* the engine keeps its own copy */
    if (rc) return rc;
    b->ns = ns;
    b->c = c;
    b->ve = ns->contr.flowtype == VISCOELASTIC;
    /* the source terms as the reference's step evaluates them before the
     * velocity stage (hig-flow-step.c:343-606, at ns->par.t, :359); fixed on
     * the GPU path (time-dependent sources were refused above, time-dependent
     * boundary data by hf_flatten) */
    higflow_calculate_source_term(ns);
    higflow_calculate_facet_source_term(ns);
    rc = copy_fields(b, k_in, (int)(sizeof k_in / sizeof k_in[0]), 1);
    if (rc) {
        hf_case_destroy(c);
        memset(b, 0, sizeof *b);
    }
    return rc;
}

int hf_step(higflow_solver *ns)
{
    hf_binding *b = find(ns);
    if (!b) {
        int rc = hf_attach(ns, NULL);
        if (rc) return rc;
        b = find(ns);
    }
    int rc = hf_case_step(b->c, 1);
    hf_stats st;
    if (hf_case_stats(b->c, &st) == HF_OK && ns->slvp) {
        ns->slvp->SolverIterations = st.last_iters;
        ns->slvp->SolverResidual = st.last_residual;
    }
    return rc;
}

int hf_sync_to_host(higflow_solver *ns)
{
    hf_binding *b = find(ns);
    if (!b) return HF_ERR_INVALID;
    return copy_fields(b, k_out, (int)(sizeof k_out / sizeof k_out[0]), 0);
}

/* the other direction, for a case that changed its fields on the host: after
 * higflow_load_properties (a restart from the reference's own checkpoint
 * files, pdomain.c:1358-1385) or any edit of ns->dp*->values between steps.
 * The source fields are copied as they are (the GPU path keeps them fixed);
 * a new pressure also restarts the engine's initial-guess history. */
int hf_sync_to_device(higflow_solver *ns)
{
    hf_binding *b = find(ns);
    if (!b) return HF_ERR_INVALID;
    /* the time step too: a restart or a host edit may have changed it */
    const double dt = ns->par.dt;
    int rc = hf_case_set_timestep(b->c, &dt, 1);
    if (rc) return rc;
    return copy_fields(b, k_in, (int)(sizeof k_in / sizeof k_in[0]), 1);
}

void hf_detach(higflow_solver *ns)
{
    hf_binding *b = find(ns);
    if (!b) return;
    copy_fields(b, k_out, (int)(sizeof k_out / sizeof k_out[0]), 0);
    hf_case_destroy(b->c);
    memset(b, 0, sizeof *b);
}

/* the reference's calling convention: no status, stop on failure
 * (higtree/src/utils.h:46-52 prints and exits) */
void hf_solver_step(higflow_solver *ns)
{
    const int rc = hf_step(ns);
    if (rc) {
        fprintf(stderr, "higflow_b200: step failed (%d): %s%s\n", rc, hf_last_error(),
                rc == HF_ERR_UNSUPPORTED ? hf_flatten_error() : "");
        exit(1);
    }
    /* the case loop prints or saves after t += dt when t >= tp / ts */
    const real t_next = ns->par.t + ns->par.dt;
    if (t_next >= ns->par.tp || t_next >= ns->par.ts) {
        const int rs = hf_sync_to_host(ns);
        if (rs) {
            fprintf(stderr, "higflow_b200: sync to host failed (%d): %s\n", rs, hf_last_error());
            exit(1);
        }
    }
}

/* higflow_adjust_timestep (hig-flow-timestep.c:115-139) on the GPU state:
 * the engine computes the CFL number from its velocity and sets the new dt,
 * which is written back to ns->par.dt as the reference does */
int hf_adjust_timestep(higflow_solver *ns)
{
    hf_binding *b = find(ns);
    if (!b) return HF_ERR_INVALID;
    double cfl = 0.0, dt = 0.0;
    int rc = hf_case_adjust_timestep(b->c, &cfl, &dt, 1);
    if (rc == HF_OK) ns->par.dt = dt;
    return rc;
}

/* targets of -Wl,--wrap=higflow_solver_step[_viscoelastic] */
void __wrap_higflow_solver_step(higflow_solver *ns) { hf_solver_step(ns); }
void __wrap_higflow_solver_step_viscoelastic(higflow_solver *ns) { hf_solver_step(ns); }
/* target of -Wl,--wrap=higflow_adjust_timestep: the GPU state's CFL; an
 * unattached case keeps the reference's own routine (weak: links that wrap
 * only the step functions do not define the __real_ alias) */
extern void __real_higflow_adjust_timestep(higflow_solver *ns) __attribute__((weak));
void __wrap_higflow_adjust_timestep(higflow_solver *ns)
{
    if (!find(ns)) {
        if (__real_higflow_adjust_timestep) __real_higflow_adjust_timestep(ns);
        return;
    }
    const int rc = hf_adjust_timestep(ns);
    if (rc) {
        fprintf(stderr, "higflow_b200: adaptive time step failed (%d): %s\n", rc, hf_last_error());
        exit(1);
    }
}

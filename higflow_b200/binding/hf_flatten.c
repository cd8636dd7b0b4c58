/*
 * Step-program flattener: the HigFlow-side half of the drop-in boundary.
 *
 * Compiled against HigFlow's own headers (with -DDIM=2 or 3, like libhigflow)
 * and linked into the host program ahead of libhigflow.  At attach time it
 * walks the reference's meshes once and asks HigTree's stencil builder
 * (sd_get_stencil / sfd_get_stencil, higtree/src/domain.c:1434, :1604) for
 * every query one time step makes, at exactly the points the reference
 * computes them, and stores the answers as a flat hf_program
 * (include/higflow_b200.h).  The ids, weights and boundary terms are therefore
 * HigTree's own, never re-derived.
 *
 * Query sequences restated here (point arithmetic written as in the
 * reference so the floating-point query points are identical):
 *   velocity stage   higflow_computational_cell   hig-flow-discret.c:86-259
 *                    + _viscoelastic              hig-flow-discret.c:541-569
 *   divergence       higflow_pressure             hig-flow-step.c:58-80
 *   Poisson rows     higflow_pressure             hig-flow-step.c:81-120
 *   pressure pin     remove_pressure_singularity  hig-flow-step.c:14-45
 *   cell stage       velocity-derivative tensor   hig-flow-step-generalized-newtonian.c:14-97
 *                    explicit constitutive step   hig-flow-step-viscoelastic.c:352-544
 *                    cell CUBISTA convection      hig-flow-step.c:1185-1358
 *
 * Every query is made twice and the second answer recorded: the first call
 * fills HigTree's point-keyed interpolation cache (domain.c:560-670), and the
 * second returns the cached form that every later reference step uses.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hig-flow-kernel.h"
#include "higflow_b200.h"
#include "higflow_b200_higflow.h"

/* reason of the last non-zero status, for hf_flatten_error() */
static char g_err[256];
#define REASON(code, msg) (snprintf(g_err, sizeof g_err, "%s", (msg)), (code))

const char *hf_flatten_error(void) { return g_err; }

/* ------------------------------------------------------------------ */
/* growable arrays                                                     */
/* ------------------------------------------------------------------ */
typedef struct { void *p; size_t n, cap, esz; } vec;

static int vec_push(vec *v, const void *e)
{
    if (v->n == v->cap) {
        size_t nc = v->cap ? v->cap * 2 : 1024;
        void *np = realloc(v->p, nc * v->esz);
        if (!np) return -1;
        v->p = np;
        v->cap = nc;
    }
    memcpy((char *)v->p + v->n * v->esz, e, v->esz);
    v->n++;
    return 0;
}

/* ------------------------------------------------------------------ */
/* general-row table with content deduplication                        */
/* ------------------------------------------------------------------ */
typedef struct {
    vec ptr;   /* int64 */
    vec col;   /* int32 */
    vec w;     /* double */
    vec rhs;   /* double */
    int64_t *hkeys;   /* hash slot -> row + 1 (0 = empty) */
    uint64_t *hvals;
    size_t hcap, hcount;
    int err;
} rowtab;

static uint64_t mix(uint64_t h, uint64_t x)
{
    h ^= x + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    return h;
}

static uint64_t dbits(double d)
{
    uint64_t u;
    memcpy(&u, &d, sizeof u);
    return u;
}

static uint64_t row_hash(int n, const int *ids, const double *w, double rhs)
{
    uint64_t h = 1469598103934665603ULL ^ (uint64_t)n;
    h = mix(h, dbits(rhs));
    for (int k = 0; k < n; k++) {
        h = mix(h, (uint64_t)(uint32_t)ids[k]);
        h = mix(h, dbits(w[k]));
    }
    return h;
}

static int row_equal(rowtab *t, int64_t r, int n, const int *ids, const double *w, double rhs)
{
    const int64_t *ptr = t->ptr.p;
    if (ptr[r + 1] - ptr[r] != n) return 0;
    if (dbits(((double *)t->rhs.p)[r]) != dbits(rhs)) return 0;
    const int32_t *col = (const int32_t *)t->col.p + ptr[r];
    const double *ww = (const double *)t->w.p + ptr[r];
    for (int k = 0; k < n; k++)
        if (col[k] != ids[k] || dbits(ww[k]) != dbits(w[k])) return 0;
    return 1;
}

static int rowtab_grow(rowtab *t)
{
    size_t nc = t->hcap ? t->hcap * 2 : 1 << 16;
    int64_t *nk = calloc(nc, sizeof *nk);
    uint64_t *nv = calloc(nc, sizeof *nv);
    if (!nk || !nv) { free(nk); free(nv); return -1; }
    for (size_t i = 0; i < t->hcap; i++) {
        if (!t->hkeys[i]) continue;
        size_t s = t->hvals[i] & (nc - 1);
        while (nk[s]) s = (s + 1) & (nc - 1);
        nk[s] = t->hkeys[i];
        nv[s] = t->hvals[i];
    }
    free(t->hkeys);
    free(t->hvals);
    t->hkeys = nk;
    t->hvals = nv;
    t->hcap = nc;
    return 0;
}

/* returns the row index (>= 0) of this content, inserting it if new */
static int64_t rowtab_insert(rowtab *t, int n, const int *ids, const double *w, double rhs)
{
    if ((t->hcount + 1) * 2 > t->hcap && rowtab_grow(t)) { t->err = 1; return -1; }
    uint64_t h = row_hash(n, ids, w, rhs);
    size_t s = h & (t->hcap - 1);
    while (t->hkeys[s]) {
        if (t->hvals[s] == h && row_equal(t, t->hkeys[s] - 1, n, ids, w, rhs)) return t->hkeys[s] - 1;
        s = (s + 1) & (t->hcap - 1);
    }
    int64_t r = (int64_t)t->rhs.n;
    if (t->ptr.n == 0) {
        int64_t z = 0;
        if (vec_push(&t->ptr, &z)) { t->err = 1; return -1; }
    }
    for (int k = 0; k < n; k++) {
        int32_t c = ids[k];
        if (vec_push(&t->col, &c) || vec_push(&t->w, &w[k])) { t->err = 1; return -1; }
    }
    int64_t end = (int64_t)t->col.n;
    if (vec_push(&t->ptr, &end) || vec_push(&t->rhs, &rhs)) { t->err = 1; return -1; }
    t->hkeys[s] = r + 1;
    t->hvals[s] = h;
    t->hcount++;
    return r;
}

/* ------------------------------------------------------------------ */
/* flattening context                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
    higflow_solver *ns;
    sim_stencil *stn;
    rowtab rows;
    vec deltas;      /* double[DIM] per entry */
    int err;
} flat;

static int32_t record(flat *F)
{
    sim_stencil *stn = F->stn;
    int n = stn_get_numelems(stn);
    double rhs = stn_get_rhs(stn);
    int *ids = stn_get_ids(stn);
    double *vals = stn_get_vals(stn);
    if (n == 1 && vals[0] == 1.0 && rhs == 0.0 && ids[0] >= 0) return ids[0];
    int64_t r = rowtab_insert(&F->rows, n, ids, vals, rhs);
    if (r < 0 || r > INT32_MAX - 1) { F->err = HF_ERR_INVALID; return 0; }
    return (int32_t)(-(r + 1));
}

/* query on a facet domain, weight 1 (compute_facet_value_at_point, hig-flow-eval.c:44) */
static int32_t qf(flat *F, sim_facet_domain *sfd, Point center, Point p)
{
    stn_reset(F->stn);
    sfd_get_stencil(sfd, center, p, 1.0, F->stn);
    stn_reset(F->stn);
    sfd_get_stencil(sfd, center, p, 1.0, F->stn);
    return record(F);
}

/* query on a cell domain, weight 1 (compute_value_at_point, hig-flow-eval.c:421) */
static int32_t qc(flat *F, sim_domain *sd, Point center, Point p)
{
    stn_reset(F->stn);
    sd_get_stencil(sd, center, p, 1.0, F->stn);
    stn_reset(F->stn);
    sd_get_stencil(sd, center, p, 1.0, F->stn);
    return record(F);
}

static uint16_t delta_index(flat *F, const Point d)
{
    double *tab = F->deltas.p;
    for (size_t i = 0; i < F->deltas.n; i++) {
        int same = 1;
        for (int k = 0; k < DIM; k++)
            if (dbits(tab[i * DIM + k]) != dbits(d[k])) { same = 0; break; }
        if (same) return (uint16_t)i;
    }
    if (F->deltas.n >= 65535) { F->err = HF_ERR_UNSUPPORTED; return 0; }
    /* the vec holds DIM doubles per entry */
    double e[DIM];
    for (int k = 0; k < DIM; k++) e[k] = d[k];
    if (vec_push(&F->deltas, e)) F->err = HF_ERR_INVALID;
    return (uint16_t)(F->deltas.n - 1);
}

/* ------------------------------------------------------------------ */
/* configuration checks                                                */
/* ------------------------------------------------------------------ */
static int detect_kernel(higflow_solver *ns, int32_t *kind)
{
    real tol = ns->ed.ve.par.kernel_tol;
    const real xs[3] = {0.37, 1.0, 2.9};
    int ident = 1, logk = 1, sqrtk = 1;
    for (int i = 0; i < 3; i++) {
        real x = xs[i];
        real inv = ns->ed.ve.get_kernel_inverse(0, x, tol);
        real jac = ns->ed.ve.get_kernel_jacobian(0, x, tol);
        if (!(inv == x && jac == 1.0)) ident = 0;
        if (!(inv == exp(x) && jac == (x < tol ? 1.0 / tol : 1.0 / x))) logk = 0;
        if (!(inv == x * x && jac == (x < tol ? 0.5 / sqrt(tol) : 0.5 / sqrt(x)))) sqrtk = 0;
    }
    if (ident) *kind = HF_KERNEL_IDENTITY;
    else if (logk) *kind = HF_KERNEL_LOG;
    else if (sqrtk) *kind = HF_KERNEL_SQRT;
    else return HF_ERR_UNSUPPORTED;
    return HF_OK;
}

static int check_bcs_fixed(sim_domain *sd)
{
    for (int t = 0; t < 2; t++) {
        bc_type bt = t == 0 ? DIRICHLET : NEUMANN;
        int nb = sd_get_num_bcs(sd, bt);
        for (int i = 0; i < nb; i++)
            if (sb_get_valuetype(sd_get_bc(sd, bt, i)) == timedependent) return HF_ERR_UNSUPPORTED;
    }
    return HF_OK;
}

/* ------------------------------------------------------------------ */
/* main entry                                                          */
/* ------------------------------------------------------------------ */
static void flat_free(flat *F)
{
    free(F->rows.ptr.p); free(F->rows.col.p); free(F->rows.w.p); free(F->rows.rhs.p);
    free(F->rows.hkeys); free(F->rows.hvals);
    free(F->deltas.p);
}

int hf_flatten(higflow_solver *ns, hf_program **out)
{
    *out = NULL;
    g_err[0] = 0;
    if (ns->contr.spatialdiscrtype != ORDER2) return REASON(HF_ERR_UNSUPPORTED, "spatial discretisation is not second order");
    if (ns->contr.tempdiscrtype != EXPLICIT_EULER && ns->contr.tempdiscrtype != EXPLICIT_RK2 &&
        ns->contr.tempdiscrtype != EXPLICIT_RK3 && ns->contr.tempdiscrtype != SEMI_IMPLICIT_EULER &&
        ns->contr.tempdiscrtype != SEMI_IMPLICIT_CN && ns->contr.tempdiscrtype != SEMI_IMPLICIT_BDF2)
        return REASON(HF_ERR_UNSUPPORTED, "unknown time discretisation");
    if (ns->contr.flowtype != NEWTONIAN && ns->contr.flowtype != VISCOELASTIC) return REASON(HF_ERR_UNSUPPORTED, "flow type is neither Newtonian nor viscoelastic");
    if (ns->contr.eoflow) return REASON(HF_ERR_UNSUPPORTED, "electro-osmotic flow");
    const int ve = ns->contr.flowtype == VISCOELASTIC;
    int32_t kernel = HF_KERNEL_IDENTITY;
    if (ve) {
        if (ns->ed.ve.contr.discrtype != EXPLICIT && ns->ed.ve.contr.discrtype != IMPLICIT)
            return REASON(HF_ERR_UNSUPPORTED, "constitutive step neither explicit nor implicit Euler");
        /* FENE-P is left out: the reference's polymeric tensor reads xi without
         * assigning it for this model (hig-flow-step-viscoelastic.c:285-292),
         * so its stress has no defined value to reproduce */
        if (ns->ed.ve.contr.model == FENE_P)
            return REASON(HF_ERR_UNSUPPORTED, "FENE-P (the reference's stress for it reads an unassigned xi)");
        if (ns->ed.ve.contr.model != OLDROYD_B && ns->ed.ve.contr.model != GIESEKUS &&
            ns->ed.ve.contr.model != LPTT && ns->ed.ve.contr.model != GPTT && ns->ed.ve.contr.model != E_FENE)
            return REASON(HF_ERR_UNSUPPORTED, "viscoelastic model other than Oldroyd-B, Giesekus, LPTT, GPTT, e-FENE");
        /* the Mittag-Leffler evaluation takes 0 < alpha <= 5 and beta <= 5
         * (hig-flow-mittag-leffler.c:143-153 reports the others as errors) */
        if (ns->ed.ve.contr.model == GPTT &&
            !(ns->ed.ve.par.alpha_gptt > 0.0 && ns->ed.ve.par.alpha_gptt <= 5.0 && ns->ed.ve.par.beta_gptt <= 5.0))
            return REASON(HF_ERR_INVALID, "GPTT needs 0 < alpha_gptt <= 5 and beta_gptt <= 5");
        if (detect_kernel(ns, &kernel)) return REASON(HF_ERR_UNSUPPORTED, "kernel transform callbacks are not identity, log or sqrt");
    }

    sim_domain *sdp = psd_get_local_domain(ns->psdp);
    sim_facet_domain *sfdu[DIM];
    for (int d = 0; d < DIM; d++) sfdu[d] = psfd_get_local_domain(ns->psfdu[d]);
    /* Velocity and pressure boundary values must be fixed (they are folded into
     * the recorded rows).  The source-term domains always carry "timedependent"
     * boundaries (hig-flow-bc.c:497, :535); the program samples the source
     * fields and their boundary values once, at attach, so time-dependent
     * source callbacks are outside this path. */
    if (check_bcs_fixed(sdp)) return REASON(HF_ERR_UNSUPPORTED, "time-dependent pressure boundary condition");
    for (int d = 0; d < DIM; d++)
        if (check_bcs_fixed(sfdu[d]->cdom)) return REASON(HF_ERR_UNSUPPORTED, "time-dependent velocity boundary condition");
    sim_domain *sded = ve ? ns->ed.sdED : NULL;

    hf_program *P = calloc(1, sizeof *P);
    if (!P) return HF_ERR_INVALID;
    flat F;
    memset(&F, 0, sizeof F);
    F.ns = ns;
    F.stn = stn_create();
    F.rows.ptr.esz = sizeof(int64_t);
    F.rows.col.esz = sizeof(int32_t);
    F.rows.w.esz = sizeof(double);
    F.rows.rhs.esz = sizeof(double);
    F.deltas.esz = sizeof(double) * DIM;

    hf_params *par = &P->par;
    par->dim = DIM;
    par->flowtype = ns->contr.flowtype;
    par->projtype = ns->contr.projtype;
    par->convecdiscrtype = ns->contr.convecdiscrtype;
    par->secondconvecdiscrtype = ns->contr.secondconvecdiscrtype;
    par->Re = ns->par.Re;
    par->dt = ns->par.dt;
    /* the semi-implicit velocity system (hig-flow-step.c:788-883) is assembled
     * by the engine from the recorded UL/UR stencils of every direction: the
     * same sfd_get_stencil queries at fcenter -/+ fdelta[dim2], here with
     * weight 1 and there with weight -dt/(Re fdelta[dim2]^2) */
    par->tempdiscrtype = ns->contr.tempdiscrtype == SEMI_IMPLICIT_EULER ? HF_SEMI_IMPLICIT_EULER
                         : ns->contr.tempdiscrtype == SEMI_IMPLICIT_CN ? HF_SEMI_IMPLICIT_CN
                         : ns->contr.tempdiscrtype == SEMI_IMPLICIT_BDF2 ? HF_SEMI_IMPLICIT_BDF2
                         : ns->contr.tempdiscrtype == EXPLICIT_RK2 ? HF_EXPLICIT_RK2
                         : ns->contr.tempdiscrtype == EXPLICIT_RK3 ? HF_EXPLICIT_RK3 : HF_EXPLICIT_EULER;
    if (ve) {
        par->ve_model = ns->ed.ve.contr.model;
        par->ve_convecdiscrtype = ns->ed.ve.contr.convecdiscrtype;
        par->kernel = kernel;
        par->De = ns->ed.ve.par.De;
        par->beta = ns->ed.ve.par.beta;
        par->kernel_tol = ns->ed.ve.par.kernel_tol;
        par->alpha = ns->ed.ve.par.alpha;
        par->epsilon = ns->ed.ve.par.epsilon;
        par->xi = ns->ed.ve.par.xi;
        par->L2_fene = ns->ed.ve.par.L2_fene;
        par->lambda_fene = ns->ed.ve.par.lambda_fene;
        par->E_fene = ns->ed.ve.par.E_fene;
        par->alpha_gptt = ns->ed.ve.par.alpha_gptt;
        par->beta_gptt = ns->ed.ve.par.beta_gptt;
        par->gamma_gptt = tgamma(ns->ed.ve.par.beta_gptt);
        par->ve_discrtype = ns->ed.ve.contr.discrtype == IMPLICIT ? HF_VE_IMPLICIT : HF_VE_EXPLICIT;
    }

    const int ncell = psd_get_local_domain_size(ns->psdp);
    P->ncell = ncell;
    int rc = HF_OK;

    /* ---- cells: ids, deltas, gid == lid check ---- */
    mp_mapper *mp = sd_get_domain_mapper(sdp);
    uint16_t *cdel = calloc((size_t)ncell, sizeof *cdel);
    int32_t *div = calloc((size_t)HF_P_NSLOT(DIM) * ncell, sizeof *div);
    const int cns = ve ? HF_C_NSLOT(DIM) : 0;
    int32_t *cslots = ve ? calloc((size_t)cns * ncell, sizeof *cslots) : NULL;
    uint32_t *cflags = ve ? calloc((size_t)ncell, sizeof *cflags) : NULL;
    vec pptr = {0}, pcol = {0}, pval = {0};
    pptr.esz = sizeof(int64_t); pcol.esz = sizeof(int32_t); pval.esz = sizeof(double);
    double *brhs = calloc((size_t)ncell, sizeof *brhs);
    int64_t *rowstart = calloc((size_t)ncell + 1, sizeof *rowstart);
    int32_t *rowlen = calloc((size_t)ncell, sizeof *rowlen);
    if (!cdel || !div || !brhs || !rowstart || !rowlen || (ve && (!cslots || !cflags))) { rc = HF_ERR_INVALID; goto fail; }

    /* pressure pin (remove_pressure_singularity, hig-flow-step.c:14-45) */
    P->pin_row = -1;
    if (ns->contr.desingpressure == true) {
        hig_cell *c = sd_get_higtree(sdp, 0);
        Point ccenter, ccenter2;
        hig_get_center(c, ccenter);
        hig_cell *c2 = hig_get_cell_with_point(c, ccenter);
        int clid = mp_lookup(mp, hig_get_cid(c2));
        hig_get_center(c2, ccenter2);
        P->pin_row = psd_lid_to_gid(ns->psdp, clid);
        P->pin_value = ns->func.get_pressure(ccenter2, ns->par.t + ns->par.dt);
    }

    {
        /* Poisson rows are stored temporarily per gid then compacted */
        vec tcol = {0}, tval = {0};
        tcol.esz = sizeof(int32_t); tval.esz = sizeof(double);
        higcit_celliterator *it;
        for (it = sd_get_domain_celliterator(sdp); !higcit_isfinished(it); higcit_nextcell(it)) {
            hig_cell *c = higcit_getcell(it);
            int clid = mp_lookup(mp, hig_get_cid(c));
            int cgid = psd_get_global_id(ns->psdp, c);
            if (clid != cgid || clid < 0 || clid >= ncell) { rc = REASON(HF_ERR_UNSUPPORTED, "cell global ids differ from local ids"); break; }
            Point ccenter, cdelta;
            hig_get_center(c, ccenter);
            hig_get_delta(c, cdelta);
            cdel[clid] = delta_index(&F, cdelta);

            /* divergence queries: compute_facet_u_left/right(sfdu[dim], ccenter, cdelta, dim, 0.5) */
            for (int dim = 0; dim < DIM; dim++) {
                Point p;
                POINT_ASSIGN(p, ccenter);
                p[dim] = ccenter[dim] - 0.5 * cdelta[dim];
                div[(size_t)HF_P_UL(dim) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
                POINT_ASSIGN(p, ccenter);
                p[dim] = ccenter[dim] + 0.5 * cdelta[dim];
                div[(size_t)HF_P_UR(dim) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
            }

            /* Poisson row: boundary part of the rhs only (the divergence part is added per
             * step).  Built twice so interpolated neighbours come from the warm cache. */
            for (int pass = 0; pass < 2; pass++) {
                stn_reset(F.stn);
                stn_set_rhs(F.stn, 0.0);
                real alpha = 0.0;
                for (int dim = 0; dim < DIM; dim++) {
                    real w = 1.0 / (cdelta[dim] * cdelta[dim]);
                    alpha -= 2.0 * w;
                    Point p;
                    POINT_ASSIGN(p, ccenter);
                    p[dim] = ccenter[dim] + cdelta[dim];
                    sd_get_stencil(sdp, ccenter, p, w, F.stn);
                    p[dim] = ccenter[dim] - cdelta[dim];
                    sd_get_stencil(sdp, ccenter, p, w, F.stn);
                }
                sd_get_stencil(sdp, ccenter, ccenter, alpha, F.stn);
            }
            int *ids = psd_stn_get_gids(ns->psdp, F.stn);
            real *vals = stn_get_vals(F.stn);
            int nel = stn_get_numelems(F.stn);
            brhs[cgid] = stn_get_rhs(F.stn);
            rowstart[cgid] = (int64_t)tcol.n;
            rowlen[cgid] = nel;
            for (int k = 0; k < nel; k++) {
                int32_t cc = ids[k];
                double vv = vals[k];
                if (vec_push(&tcol, &cc) || vec_push(&tval, &vv)) { rc = HF_ERR_INVALID; break; }
            }

            /* viscoelastic cell-stage queries */
            if (ve && rc == HF_OK) {
                int elid = mp_lookup(sd_get_domain_mapper(sded), hig_get_cid(c));
                if (elid != clid) { rc = REASON(HF_ERR_UNSUPPORTED, "tensor-domain cell ids differ from pressure ids"); break; }
                uint32_t fl = 0;
                cslots[(size_t)HF_C_SELF * ncell + clid] = qc(&F, sded, ccenter, ccenter);
                for (int dim = 0; dim < DIM; dim++) {
                    int b = HF_C_BLK0 + HF_C_NB * dim;
                    Point p;
                    POINT_ASSIGN(p, ccenter);
                    p[dim] = ccenter[dim] - 0.5 * cdelta[dim];
                    cslots[(size_t)(b + HF_C_UVL) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
                    POINT_ASSIGN(p, ccenter);
                    p[dim] = ccenter[dim] + 0.5 * cdelta[dim];
                    cslots[(size_t)(b + HF_C_UVR) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
                    const real al[4] = {1.0, 1.0, 2.0, 2.0};
                    const int sg[4] = {-1, 1, -1, 1};
                    for (int k = 0; k < 4; k++) {
                        POINT_ASSIGN(p, ccenter);
                        if (sg[k] < 0) p[dim] = ccenter[dim] - al[k] * cdelta[dim];
                        else p[dim] = ccenter[dim] + al[k] * cdelta[dim];
                        if (sd_get_cell_with_point(sded, p) != NULL) fl |= 1u << (4 * dim + k);
                        cslots[(size_t)(b + HF_C_KL + k) * ncell + clid] = qc(&F, sded, ccenter, p);
                    }
                }
                int q = HF_C_BLK0 + HF_C_NB * DIM;
                for (int dim = 0; dim < DIM; dim++) {
                    for (int dim2 = 0; dim2 < DIM; dim2++) {
                        if (dim2 == dim) continue;
                        const real a = 1.0;
                        Point p;
                        /* compute_facet_u_4_left: valuerr, valuell */
                        POINT_ASSIGN(p, ccenter);
                        p[dim] = ccenter[dim] + 0.5 * a * cdelta[dim];
                        p[dim2] = ccenter[dim2] - a * cdelta[dim2];
                        cslots[(size_t)(q + 0) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
                        POINT_ASSIGN(p, ccenter);
                        p[dim] = ccenter[dim] - 0.5 * a * cdelta[dim];
                        p[dim2] = ccenter[dim2] - a * cdelta[dim2];
                        cslots[(size_t)(q + 1) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
                        /* compute_facet_u_4_right: valuerr, valuell */
                        POINT_ASSIGN(p, ccenter);
                        p[dim] = ccenter[dim] + 0.5 * a * cdelta[dim];
                        p[dim2] = ccenter[dim2] + a * cdelta[dim2];
                        cslots[(size_t)(q + 2) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
                        POINT_ASSIGN(p, ccenter);
                        p[dim] = ccenter[dim] - 0.5 * a * cdelta[dim];
                        p[dim2] = ccenter[dim2] + a * cdelta[dim2];
                        cslots[(size_t)(q + 3) * ncell + clid] = qf(&F, sfdu[dim], ccenter, p);
                        q += HF_C_NQ;
                    }
                }
                cflags[clid] = fl;
            }
            if (F.err) { rc = F.err; break; }
        }
        higcit_destroy(it);
        if (rc == HF_OK) {
            /* compact the Poisson rows in gid order; the pinned row is left empty */
            int64_t z = 0;
            vec_push(&pptr, &z);
            for (int r = 0; r < ncell && rc == HF_OK; r++) {
                if (r != P->pin_row) {
                    for (int k = 0; k < rowlen[r]; k++) {
                        if (vec_push(&pcol, (int32_t *)tcol.p + rowstart[r] + k) ||
                            vec_push(&pval, (double *)tval.p + rowstart[r] + k)) rc = HF_ERR_INVALID;
                    }
                }
                int64_t e = (int64_t)pcol.n;
                vec_push(&pptr, &e);
            }
        }
        free(tcol.p);
        free(tval.p);
        if (rc) goto fail;
    }

    /* ---- velocity stage per facet direction ---- */
    const int vns = ve ? HF_V_NSLOT_VE(DIM) : HF_V_NSLOT_NEWT(DIM);
    P->vel_nslot = vns;
    for (int dim = 0; dim < DIM; dim++) {
        int nf = psfd_get_local_domain_size(ns->psfdu[dim]);
        P->nfacet[dim] = nf;
        int32_t *vs = calloc((size_t)vns * (nf ? nf : 1), sizeof *vs);
        uint32_t *vf = calloc((size_t)(nf ? nf : 1), sizeof *vf);
        uint16_t *vd = calloc((size_t)(nf ? nf : 1), sizeof *vd);
        P->vel_slots[dim] = vs;
        P->vel_flags[dim] = vf;
        P->vel_delta[dim] = vd;
        if (!vs || !vf || !vd) { rc = HF_ERR_INVALID; goto fail; }
        mp_mapper *mu = sfd_get_domain_mapper(sfdu[dim]);
        mp_mapper *mF = sfd_get_domain_mapper(ns->sfdF[dim]);
        higfit_facetiterator *fit;
        for (fit = sfd_get_domain_facetiterator(sfdu[dim]); !higfit_isfinished(fit); higfit_nextfacet(fit)) {
            hig_facet *f = higfit_getfacet(fit);
            int flid = mp_lookup(mu, hig_get_fid(f));
            if (flid < 0 || flid >= nf || mp_lookup(mF, hig_get_fid(f)) != flid) { rc = REASON(HF_ERR_UNSUPPORTED, "source-facet ids differ from velocity-facet ids"); break; }
            Point fcenter, fdelta;
            hig_get_facet_center(f, fcenter);
            hig_get_facet_delta(f, fdelta);
            vd[flid] = delta_index(&F, fdelta);
            uint32_t fl = 0;
#define VS(slot) vs[(size_t)(slot) * nf + flid]
            VS(HF_V_FU) = qf(&F, ns->sfdF[dim], fcenter, fcenter);
            Point p;
            POINT_ASSIGN(p, fcenter);
            p[dim] = fcenter[dim] - 0.5 * fdelta[dim];
            VS(HF_V_PL) = qc(&F, sdp, fcenter, p);
            POINT_ASSIGN(p, fcenter);
            p[dim] = fcenter[dim] + 0.5 * fdelta[dim];
            VS(HF_V_PR) = qc(&F, sdp, fcenter, p);
            POINT_ASSIGN(p, fcenter);
            p[dim] = fcenter[dim] - 0.5 * fdelta[dim];
            VS(HF_V_FL) = qc(&F, ns->sdF, fcenter, p);
            POINT_ASSIGN(p, fcenter);
            p[dim] = fcenter[dim] + 0.5 * fdelta[dim];
            VS(HF_V_FR) = qc(&F, ns->sdF, fcenter, p);
            for (int dim2 = 0; dim2 < DIM; dim2++) {
                int b = HF_V_BLK0 + HF_V_NB * dim2;
                if (dim2 != dim) {
                    /* compute_facet_u_2(sfdu[dim2], fcenter, fdelta, dim, dim2, 1.0) */
                    const real a = 1.0;
                    POINT_ASSIGN(p, fcenter);
                    p[dim] = fcenter[dim] + 0.5 * a * fdelta[dim];
                    p[dim2] = fcenter[dim2] + 0.5 * a * fdelta[dim2];
                    VS(b + HF_V_V4 + 0) = qf(&F, sfdu[dim2], fcenter, p);
                    p[dim] = fcenter[dim] + 0.5 * a * fdelta[dim];
                    p[dim2] = fcenter[dim2] - 0.5 * a * fdelta[dim2];
                    VS(b + HF_V_V4 + 1) = qf(&F, sfdu[dim2], fcenter, p);
                    p[dim] = fcenter[dim] - 0.5 * a * fdelta[dim];
                    p[dim2] = fcenter[dim2] + 0.5 * a * fdelta[dim2];
                    VS(b + HF_V_V4 + 2) = qf(&F, sfdu[dim2], fcenter, p);
                    p[dim] = fcenter[dim] - 0.5 * a * fdelta[dim];
                    p[dim2] = fcenter[dim2] - 0.5 * a * fdelta[dim2];
                    VS(b + HF_V_V4 + 3) = qf(&F, sfdu[dim2], fcenter, p);
                }
                /* compute_facet_u_left/right(sfdu[dim], fcenter, fdelta, dim2, alpha) */
                const real al[4] = {1.0, 1.0, 2.0, 2.0};
                const int sg[4] = {-1, 1, -1, 1};
                for (int k = 0; k < 4; k++) {
                    hig_facet ff;
                    POINT_ASSIGN(p, fcenter);
                    if (sg[k] < 0) p[dim2] = fcenter[dim2] - al[k] * fdelta[dim2];
                    else p[dim2] = fcenter[dim2] + al[k] * fdelta[dim2];
                    if (sfd_get_facet_with_point(sfdu[dim], p, &ff)) fl |= 1u << (4 * dim2 + k);
                    VS(b + HF_V_UL + k) = qf(&F, sfdu[dim], fcenter, p);
                }
                /* CUBISTA face velocities: compute_facet_u_right/left(sfdu[dim2], ..., dim2, 0.5) */
                POINT_ASSIGN(p, fcenter);
                p[dim2] = fcenter[dim2] + 0.5 * fdelta[dim2];
                VS(b + HF_V_VCR) = qf(&F, sfdu[dim2], fcenter, p);
                POINT_ASSIGN(p, fcenter);
                p[dim2] = fcenter[dim2] - 0.5 * fdelta[dim2];
                VS(b + HF_V_VCL) = qf(&F, sfdu[dim2], fcenter, p);
            }
            if (ve) {
                for (int dim2 = 0; dim2 < DIM; dim2++) {
                    int b = HF_V_NSLOT_NEWT(DIM) + HF_V_NS * dim2;
                    if (dim2 == dim) {
                        POINT_ASSIGN(p, fcenter);
                        p[dim2] = fcenter[dim2] - 0.5 * fdelta[dim2];
                        VS(b + 0) = qc(&F, sded, fcenter, p);
                        POINT_ASSIGN(p, fcenter);
                        p[dim2] = fcenter[dim2] + 0.5 * fdelta[dim2];
                        VS(b + 2) = qc(&F, sded, fcenter, p);
                        VS(b + 1) = VS(b + 0);
                        VS(b + 3) = VS(b + 2);
                    } else {
                        const real a = 1.0;
                        /* compute_center_p_left_2(sdED, fcenter, fdelta, dim, dim2, 1.0) */
                        POINT_ASSIGN(p, fcenter);
                        p[dim2] = fcenter[dim2] - a * fdelta[dim2];
                        p[dim] = fcenter[dim] - 0.5 * a * fdelta[dim];
                        VS(b + 0) = qc(&F, sded, fcenter, p);
                        p[dim2] = fcenter[dim2] - a * fdelta[dim2];
                        p[dim] = fcenter[dim] + 0.5 * a * fdelta[dim];
                        VS(b + 1) = qc(&F, sded, fcenter, p);
                        /* compute_center_p_right_2 */
                        POINT_ASSIGN(p, fcenter);
                        p[dim2] = fcenter[dim2] + a * fdelta[dim2];
                        p[dim] = fcenter[dim] - 0.5 * a * fdelta[dim];
                        VS(b + 2) = qc(&F, sded, fcenter, p);
                        p[dim2] = fcenter[dim2] + a * fdelta[dim2];
                        p[dim] = fcenter[dim] + 0.5 * a * fdelta[dim];
                        VS(b + 3) = qc(&F, sded, fcenter, p);
                    }
                }
            }
#undef VS
            vf[flid] = fl;
            if (F.err) { rc = F.err; break; }
        }
        higfit_destroy(fit);
        if (rc) goto fail;
    }

    if (F.rows.err) { rc = HF_ERR_INVALID; goto fail; }
    if (F.rows.ptr.n == 0) {
        int64_t z = 0;
        vec_push(&F.rows.ptr, &z);
    }
    /* one template per recorded row, base 0 */
    P->nrows = (int64_t)F.rows.rhs.n;
    P->ntmpl = P->nrows;
    P->nnz = (int64_t)F.rows.col.n;
    {
        int32_t *tm = malloc(sizeof(int32_t) * (size_t)(P->nrows ? P->nrows : 1));
        int32_t *bs = calloc((size_t)(P->nrows ? P->nrows : 1), sizeof(int32_t));
        if (!tm || !bs) { free(tm); free(bs); rc = HF_ERR_INVALID; goto fail; }
        for (int64_t r = 0; r < P->nrows; r++) tm[r] = (int32_t)r;
        P->row_tmpl = tm;
        P->row_base = bs;
    }
    P->tmpl_ptr = F.rows.ptr.p;
    P->tmpl_col = F.rows.col.p;
    P->tmpl_w = F.rows.w.p;
    P->row_rhs = F.rows.rhs.p;
    F.rows.ptr.p = F.rows.col.p = F.rows.w.p = F.rows.rhs.p = NULL;
    P->ndelta = (int32_t)F.deltas.n;
    P->delta = F.deltas.p;
    F.deltas.p = NULL;
    P->div_slots = div;
    P->cell_delta = cdel;
    P->pnnz = (int64_t)pcol.n;
    P->p_ptr = pptr.p;
    P->p_col = pcol.p;
    P->p_val = pval.p;
    P->p_brhs = brhs;
    P->cell_nslot = cns;
    P->cell_slots = cslots;
    P->cell_flags = cflags;
    free(rowstart);
    free(rowlen);
    flat_free(&F);
    stn_destroy(F.stn);
    *out = P;
    return HF_OK;

fail:
    free(cdel); free(div); free(cslots); free(cflags); free(brhs); free(rowstart); free(rowlen);
    free(pptr.p); free(pcol.p); free(pval.p);
    for (int d = 0; d < DIM; d++) {
        free((void *)P->vel_slots[d]); free((void *)P->vel_flags[d]); free((void *)P->vel_delta[d]);
    }
    free(P);
    flat_free(&F);
    stn_destroy(F.stn);
    return rc ? rc : HF_ERR_INVALID;
}

void hf_program_free(hf_program *P)
{
    if (!P) return;
    free((void *)P->delta);
    free((void *)P->row_tmpl); free((void *)P->row_base); free((void *)P->row_rhs);
    free((void *)P->tmpl_ptr); free((void *)P->tmpl_col); free((void *)P->tmpl_w);
    for (int d = 0; d < 3; d++) {
        free((void *)P->vel_slots[d]); free((void *)P->vel_flags[d]); free((void *)P->vel_delta[d]);
    }
    free((void *)P->div_slots); free((void *)P->cell_delta);
    free((void *)P->p_ptr); free((void *)P->p_col); free((void *)P->p_val); free((void *)P->p_brhs);
    free((void *)P->cell_slots); free((void *)P->cell_flags);
    free(P);
}

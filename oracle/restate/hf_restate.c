/*
 * CPU restatement of HigFlow's time step (explicit or semi-implicit Euler
 * velocity) over a flattened step program (test infrastructure: the oracle the GPU engine is checked against;
 * never linked into the product).
 *
 * Each function follows the reference routine cited beside it, statement by
 * statement, in plain FP64 with the reference's evaluation order; stencil
 * queries read the recorded slots instead of calling HigTree
 * (include/higflow_b200.h documents the slot layouts).  Its own agreement with
 * the reference's stepping (oracle/_ref) is checked by tests/test_oracle.py.
 *
 * Poisson: the system the reference hands to its solver plugin (rows of
 * higflow_pressure, hig-flow-step.c:48-131, identity row at the pinned cell,
 * solver.c:142-150) is solved here by BiCGStab with Jacobi scaling to the
 * caller's relative tolerance, starting from the previous solution as the
 * reference's engine does (solver-petsc.c:386-399).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "higflow_b200.h"

#define EPSMACH 1.0e-12
#define FLT_EQ(x, y) (fabs((x) - (y)) < EPSMACH)   /* higtree/src/utils.h:40 */

typedef struct hfr_fields {
    double *u[3], *us[3], *p, *dp, *F, *FU[3];
    double *K[9], *S[9], *Du[9];
} hfr_fields;

/* value of one recorded query (dp_interpolate_from_stencil, pdomain.c:1026-1053) */
static double q(const hf_program *P, int32_t code, const double *f)
{
    if (code >= 0) return f[code];
    int64_t r = -(int64_t)code - 1;
    int64_t t = P->row_tmpl[r];
    const double *fb = f + P->row_base[r];
    double res = 0.0;
    res += -P->row_rhs[r];
    for (int64_t k = P->tmpl_ptr[t]; k < P->tmpl_ptr[t + 1]; k++) res += fb[P->tmpl_col[k]] * P->tmpl_w[k];
    return res;
}

/* ------------------------------------------------------------------ */
/* velocity stage: higflow_computational_cell (hig-flow-discret.c:86-259),  */
/* terms (hig-flow-terms.c), explicit Euler (hig-flow-step.c:613-660,       */
/* hig-flow-step-viscoelastic.c:931-980)                                    */
/* ------------------------------------------------------------------ */
/* ebr: BDF2 only, receives the bracket (source - pressure [+ tensor] -
 * convection) of every facet for the second solve */
static void velocity_stage_e(const hf_program *P, hfr_fields *F, int d, double *ebr)
{
    const int D = P->par.dim;
    const int nf = P->nfacet[d];
    const int ns = P->vel_nslot;
    const int ve = P->par.flowtype == HF_VISCOELASTIC;
    const double a = 1.7500, b = 0.3750, c = 0.7500, dd = 0.1250, e = 0.2500;
    for (int f = 0; f < nf; f++) {
        const int32_t *sl = P->vel_slots[d];
#define SL(s) sl[(size_t)(s) * nf + f]
        const double *fd = P->delta + (size_t)P->vel_delta[d][f] * D;
        const uint32_t fl = P->vel_flags[d][f];
        int convec = P->par.convecdiscrtype;
        double conv1 = 0.0, conv2 = 0.0;
        double ufacet = F->u[d][f];
        double Fs = q(P, SL(HF_V_FU), F->FU[d]);
        double pl = q(P, SL(HF_V_PL), F->p);
        double pr = q(P, SL(HF_V_PR), F->p);
        double dpdx = (pr - pl) / (2.0 * 0.5 * fd[d]);
        double Fl = q(P, SL(HF_V_FL), F->F);
        double Fr = q(P, SL(HF_V_FR), F->F);
        Fs += (Fr + Fl) / 2.0;
        double v[3], dudxc[3], dudxr[3], dudxl[3], dudxrr[3] = {0}, dudxll[3] = {0}, du2dx2[3], vc[3] = {0};
        for (int d2 = 0; d2 < D; d2++) {
            const int B = HF_V_BLK0 + HF_V_NB * d2;
            if (d2 == d) {
                v[d2] = ufacet;
            } else {
                double vrr = q(P, SL(B + HF_V_V4 + 0), F->u[d2]);
                double vlr = q(P, SL(B + HF_V_V4 + 1), F->u[d2]);
                double vrl = q(P, SL(B + HF_V_V4 + 2), F->u[d2]);
                double vll = q(P, SL(B + HF_V_V4 + 3), F->u[d2]);
                v[d2] = 0.25 * (vll + vlr + vrl + vrr);
            }
            double ul = q(P, SL(B + HF_V_UL), F->u[d]);
            int infl = (fl >> (4 * d2 + 0)) & 1;
            if (infl == 0 && convec == HF_SECOND_ORDER) convec = HF_FIRST_ORDER;
            double ur = q(P, SL(B + HF_V_UR), F->u[d]);
            int infr = (fl >> (4 * d2 + 1)) & 1;
            if (infr == 0 && convec == HF_SECOND_ORDER) convec = HF_FIRST_ORDER;
            dudxc[d2] = (ur - ul) / (2.0 * 1.0 * fd[d2]);
            dudxr[d2] = (ur - ufacet) / (1.0 * fd[d2]);
            dudxl[d2] = (ufacet - ul) / (1.0 * fd[d2]);
            double urr = q(P, SL(B + HF_V_URR), F->u[d]);
            int infrr = (fl >> (4 * d2 + 3)) & 1;
            double ull = q(P, SL(B + HF_V_ULL), F->u[d]);
            int infll = (fl >> (4 * d2 + 2)) & 1;
            if (convec == HF_SECOND_ORDER) {
                if (P->par.secondconvecdiscrtype == HF_QUICK) {
                    dudxrr[d2] = (urr - ur) / (1.0 * fd[d2]);
                    dudxll[d2] = (ul - ull) / (1.0 * fd[d2]);
                } else if (P->par.secondconvecdiscrtype == HF_CUBISTA) {
                    if (infl == 0) convec = HF_FIRST_ORDER;
                    if (infr == 0) convec = HF_FIRST_ORDER;
                    double vcr = q(P, SL(B + HF_V_VCR), F->u[d2]);
                    if (vcr > 0.0) {
                        if (FLT_EQ(ur, ul)) {
                            conv1 = vcr * ufacet;
                        } else {
                            double fi = (ufacet - ul) / (ur - ul);
                            if ((fi <= 0.0) || (fi >= 1.0)) {
                                conv1 = vcr * ufacet;
                            } else {
                                if (fi < b) conv1 = vcr * (a * ufacet - c * ul);
                                if ((fi >= b) && (fi <= c)) conv1 = vcr * (c * ufacet + b * ur - dd * ul);
                                if (fi > c) conv1 = vcr * (e * ufacet + c * ur);
                            }
                        }
                    } else {
                        if (FLT_EQ(ufacet, urr)) {
                            conv1 = vcr * ur;
                        } else {
                            double fi = (ur - urr) / (ufacet - urr);
                            if ((fi <= 0.0) || (fi >= 1.0)) {
                                conv1 = vcr * ur;
                            } else {
                                if (fi < b) conv1 = infrr == 1 ? vcr * (a * ur - c * urr) : vcr * ur;
                                if ((fi >= b) && (fi <= c)) conv1 = infrr == 1 ? vcr * (c * ur + b * ufacet - dd * urr) : vcr * ur;
                                if (fi > c) conv1 = vcr * (c * ufacet + e * ur);
                            }
                        }
                    }
                    double vcl = q(P, SL(B + HF_V_VCL), F->u[d2]);
                    if (vcl > 0.0) {
                        if (FLT_EQ(ufacet, ull)) {
                            conv2 = vcl * ul;
                        } else {
                            double fi = (ul - ull) / (ufacet - ull);
                            if ((fi <= 0.0) || (fi >= 1.0)) {
                                conv2 = vcl * ul;
                            } else {
                                if (fi < b) conv2 = infll == 1 ? vcl * (a * ul - c * ull) : vcl * ul;
                                if ((fi >= b) && (fi <= c)) conv2 = infll == 1 ? vcl * (b * ufacet + c * ul - dd * ull) : vcl * ul;
                                if (fi > c) conv2 = vcl * (c * ufacet + e * ul);
                            }
                        }
                    } else {
                        if (FLT_EQ(ul, ur)) {
                            conv2 = vcl * ufacet;
                        } else {
                            double fi = (ufacet - ur) / (ul - ur);
                            if ((fi <= 0.0) || (fi >= 1.0)) {
                                conv2 = vcl * ufacet;
                            } else {
                                if (fi < b) conv2 = vcl * (a * ufacet - c * ur);
                                if ((fi >= b) && (fi <= c)) conv2 = vcl * (b * ul + c * ufacet - dd * ur);
                                if (fi > c) conv2 = vcl * (c * ul + e * ufacet);
                            }
                        }
                    }
                    vc[d2] = ((conv1 - conv2) / fd[d]);
                }
            }
            du2dx2[d2] = (ul - 2.0 * ufacet + ur) / (fd[d2] * fd[d2] * 1.0 * 1.0);
        }
        double dSdx[3] = {0};
        if (ve) {
            for (int d2 = 0; d2 < D; d2++) {
                const int B = HF_V_NSLOT_NEWT(D) + HF_V_NS * d2;
                const double *Sf = F->S[d * D + d2];
                if (d2 == d) {
                    double Sl = q(P, SL(B + 0), Sf);
                    double Sr = q(P, SL(B + 2), Sf);
                    dSdx[d2] = (Sr - Sl) / (2.0 * 0.5 * fd[d2]);
                } else {
                    double l1 = q(P, SL(B + 0), Sf), l2 = q(P, SL(B + 1), Sf);
                    double Sl = 0.5 * (l1 + l2);
                    double r1 = q(P, SL(B + 2), Sf), r2 = q(P, SL(B + 3), Sf);
                    double Sr = 0.5 * (r1 + r2);
                    dSdx[d2] = (Sr - Sl) / (2.0 * 1.0 * fd[d2]);
                }
            }
        }
#undef SL
        /* hig-flow-terms.c */
        double pterm = P->par.projtype == HF_INCREMENTAL ? dpdx : 0.0;
        double conv = 0.0;
        switch (convec) {
        case HF_CENTRAL:
            for (int d2 = 0; d2 < D; d2++) conv += v[d2] * dudxc[d2];
            break;
        case HF_FIRST_ORDER:
            for (int d2 = 0; d2 < D; d2++) {
                conv += 0.5 * (v[d2] + fabs(v[d2])) * dudxl[d2];
                conv += 0.5 * (v[d2] - fabs(v[d2])) * dudxr[d2];
            }
            break;
        case HF_SECOND_ORDER:
            if (P->par.secondconvecdiscrtype == HF_CUBISTA) {
                for (int d2 = 0; d2 < D; d2++) conv += vc[d2];
            } else if (P->par.secondconvecdiscrtype == HF_QUICK) {
                for (int d2 = 0; d2 < D; d2++) {
                    conv += (v[d2] + fabs(v[d2])) * 0.1875 * dudxl[d2];
                    conv += (v[d2] + fabs(v[d2])) * 0.3750 * dudxr[d2];
                    conv -= (v[d2] + fabs(v[d2])) * 0.0625 * dudxrr[d2];
                    conv += (v[d2] - fabs(v[d2])) * 0.3750 * dudxl[d2];
                    conv += (v[d2] - fabs(v[d2])) * 0.1875 * dudxr[d2];
                    conv -= (v[d2] - fabs(v[d2])) * 0.0625 * dudxll[d2];
                }
            } else {
                for (int d2 = 0; d2 < D; d2++) {
                    conv += 0.5 * (v[d2] + fabs(v[d2])) * dudxl[d2];
                    conv += 0.5 * (v[d2] - fabs(v[d2])) * dudxr[d2];
                    if (v[d2] > 0.0) {
                        if (fabs(dudxl[d2]) > 1.0e-8) conv += 0.5 * v[d2] * fd[d2] * du2dx2[d2] / dudxl[d2];
                    } else {
                        if (fabs(dudxr[d2]) > 1.0e-8) conv -= 0.5 * v[d2] * fd[d2] * du2dx2[d2] / dudxr[d2];
                    }
                }
            }
            break;
        }
        double diff = 0.0;
        for (int d2 = 0; d2 < D; d2++) diff += du2dx2[d2];
        diff /= P->par.Re;
        double rhs = 0.0;
        if (!ve) {
            rhs -= pterm;
            rhs -= conv;
            rhs += diff;
            rhs += Fs;
        } else {
            double tens = 0.0;
            for (int d2 = 0; d2 < D; d2++) tens += dSdx[d2];
            rhs += Fs;
            rhs -= pterm;
            rhs += tens;
            rhs -= conv;
            rhs += diff;
        }
        if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_BDF2) {
            /* higflow_semi_implicit_bdf2_intermediate_velocity, first solve
             * (hig-flow-step.c:1021-1033; viscoelastic
             * hig-flow-step-viscoelastic.c:1349-1363) */
            double br = 0.0;
            br += Fs;
            br -= pterm;
            if (ve) {
                double tens = 0.0;
                for (int d2 = 0; d2 < D; d2++) tens += dSdx[d2];
                br += tens;
            }
            br -= conv;
            ebr[f] = br;
            double r = br;
            r *= 0.5 * P->par.dt;
            r += 0.25 * P->par.dt * diff;
            r += ufacet;
            F->us[d][f] = r;
            continue;
        }
        if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_EULER || P->par.tempdiscrtype == HF_SEMI_IMPLICIT_CN) {
            /* higflow_semi_implicit_euler_intermediate_velocity
             * (hig-flow-step.c:812-829; viscoelastic
             * hig-flow-step-viscoelastic.c:1136-1147): the right-hand side
             * without diffusion; Crank-Nicolson (hig-flow-step.c:908-917)
             * keeps half of it; the system is solved by sie_solve */
            double r = 0.0;
            if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_CN) r += 0.5 * diff;
            r += Fs;
            r -= pterm;
            if (ve) {
                double tens = 0.0;
                for (int d2 = 0; d2 < D; d2++) tens += dSdx[d2];
                r += tens;
            }
            r -= conv;
            r *= P->par.dt;
            r += ufacet;
            F->us[d][f] = r;
            continue;
        }
        F->us[d][f] = ufacet + P->par.dt * rhs;
    }
}

/* ------------------------------------------------------------------ */
/* semi-implicit Euler: the velocity system of direction d              */
/* (hig-flow-step.c:830-883): row f = alpha u_f + sum_d2 w_d2 (S(f +    */
/* delta_d2) + S(f - delta_d2)), w_d2 = -dt/(Re delta_d2^2), alpha = 1 - */
/* 2 sum w_d2; S(point) = the recorded UR/UL stencils (sfd_get_stencil  */
/* at fcenter +/- fdelta[d2], here scaled by w_d2); their boundary terms */
/* (w times the row's rhs) join the right-hand side held in us[d].      */
/* Solved by BiCGStab with Jacobi scaling from u.                       */
/* ------------------------------------------------------------------ */
static void velocity_stage(const hf_program *P, hfr_fields *F, int d) { velocity_stage_e(P, F, d, NULL); }

typedef struct csr { int n; int64_t *ptr; int32_t *col; double *val; } csr;

static double dot(int n, const double *a, const double *b);

static void csr_spmv(const csr *A, const double *x, double *y)
{
    for (int i = 0; i < A->n; i++) {
        double s = 0.0;
        for (int64_t k = A->ptr[i]; k < A->ptr[i + 1]; k++) s += A->val[k] * x[A->col[k]];
        y[i] = s;
    }
}

static int csr_bicgstab(const csr *A, const double *bvec, double *x, double rtol)
{
    const int n = A->n;
    double *mem = malloc(sizeof(double) * (size_t)n * 9);
    double *r = mem, *rh = r + n, *p = rh + n, *v = p + n, *s = v + n, *t = s + n, *ph = t + n,
           *sh = ph + n, *dinv = sh + n;
    for (int i = 0; i < n; i++) {
        double dg = 0.0;
        for (int64_t k = A->ptr[i]; k < A->ptr[i + 1]; k++)
            if (A->col[k] == i) dg += A->val[k];
        dinv[i] = dg != 0.0 ? 1.0 / dg : 1.0;
    }
    csr_spmv(A, x, r);
    for (int i = 0; i < n; i++) r[i] = bvec[i] - r[i];
    const double bn = sqrt(dot(n, bvec, bvec));
    const double tol = rtol * (bn > 0 ? bn : 1.0);
    double rn = sqrt(dot(n, r, r));
    memcpy(rh, r, sizeof(double) * (size_t)n);
    memset(p, 0, sizeof(double) * (size_t)n);
    memset(v, 0, sizeof(double) * (size_t)n);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int it = 0, restarts = 0;
    while (rn > tol && it < 200000) {
        const double rho1 = dot(n, rh, r);
        if (rho1 == 0.0 || omega == 0.0) {
            if (++restarts > 100) break;
            csr_spmv(A, x, r);
            for (int i = 0; i < n; i++) r[i] = bvec[i] - r[i];
            memcpy(rh, r, sizeof(double) * (size_t)n);
            memset(p, 0, sizeof(double) * (size_t)n);
            memset(v, 0, sizeof(double) * (size_t)n);
            rho = alpha = omega = 1.0;
            continue;
        }
        const double beta = (rho1 / rho) * (alpha / omega);
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        for (int i = 0; i < n; i++) ph[i] = dinv[i] * p[i];
        csr_spmv(A, ph, v);
        alpha = rho1 / dot(n, rh, v);
        for (int i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
        for (int i = 0; i < n; i++) sh[i] = dinv[i] * s[i];
        csr_spmv(A, sh, t);
        const double tt = dot(n, t, t);
        omega = tt > 0.0 ? dot(n, t, s) / tt : 0.0;
        for (int i = 0; i < n; i++) {
            x[i] += alpha * ph[i] + omega * sh[i];
            r[i] = s[i] - omega * t[i];
        }
        rho = rho1;
        rn = sqrt(dot(n, r, r));
        it++;
        if (it % 50 == 0) {
            csr_spmv(A, x, r);
            for (int i = 0; i < n; i++) r[i] = bvec[i] - r[i];
            rn = sqrt(dot(n, r, r));
        }
    }
    free(mem);
    return rn <= tol ? 0 : HF_ERR_NOT_CONVERGED;
}

static void row_add(int32_t *cols, double *vals, int *len, int32_t c, double v)
{
    for (int k = 0; k < *len; k++)
        if (cols[k] == c) { vals[k] += v; return; }
    cols[*len] = c;
    vals[*len] = v;
    (*len)++;
}

/* stage: 0 for Euler and Crank-Nicolson and BDF2's first solve, 1 for BDF2's
 * second (hig-flow-step.c:1129); the right-hand side comes in x (us[d]) and
 * the solution leaves there, from the initial guess x0 */
static int sie_solve_x(const hf_program *P, int d, int stage, double *x, const double *x0, double rtol)
{
    const int D = P->par.dim, nf = P->nfacet[d];
    const double dt = P->par.dt, Re = P->par.Re;
    /* entries per row: the centre plus 2D stencils of at most maxlen entries */
    int64_t maxlen = 1;
    for (int64_t t = 0; t < P->ntmpl; t++) {
        const int64_t l = P->tmpl_ptr[t + 1] - P->tmpl_ptr[t];
        if (l > maxlen) maxlen = l;
    }
    const int cap = (int)(1 + 2 * D * maxlen);
    csr A;
    A.n = nf;
    A.ptr = malloc(sizeof(int64_t) * (size_t)(nf + 1));
    A.col = malloc(sizeof(int32_t) * (size_t)nf * cap);
    A.val = malloc(sizeof(double) * (size_t)nf * cap);
    double *bvec = malloc(sizeof(double) * (size_t)nf);
    int32_t *rc = malloc(sizeof(int32_t) * cap);
    double *rv = malloc(sizeof(double) * cap);
    int64_t nz = 0;
    A.ptr[0] = 0;
    for (int f = 0; f < nf; f++) {
        const double *fd = P->delta + (size_t)P->vel_delta[d][f] * D;
        double alpha = 0.0, b = x[f];
        int len = 0;
        for (int d2 = 0; d2 < D; d2++) {
            double w = -dt / (Re * fd[d2] * fd[d2]);
            if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_CN) w = -0.5 * dt / (Re * fd[d2] * fd[d2]);
            if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_BDF2)
                w = stage == 0 ? -0.25 * dt / (Re * fd[d2] * fd[d2]) : -1.0 / 3.0 * dt / (Re * fd[d2] * fd[d2]);
            alpha -= 2.0 * w;
            const int sides[2] = {HF_V_UR, HF_V_UL};
            for (int k = 0; k < 2; k++) {
                const int32_t code = P->vel_slots[d][(size_t)(HF_V_BLK0 + HF_V_NB * d2 + sides[k]) * nf + f];
                if (code >= 0) { row_add(rc, rv, &len, code, w); continue; }
                const int64_t r = -(int64_t)code - 1;
                const int64_t t = P->row_tmpl[r];
                for (int64_t e = P->tmpl_ptr[t]; e < P->tmpl_ptr[t + 1]; e++)
                    row_add(rc, rv, &len, (int32_t)(P->row_base[r] + P->tmpl_col[e]), w * P->tmpl_w[e]);
                b += w * P->row_rhs[r];
            }
        }
        alpha = 1.0 + alpha;
        row_add(rc, rv, &len, f, alpha);
        memcpy(A.col + nz, rc, sizeof(int32_t) * len);
        memcpy(A.val + nz, rv, sizeof(double) * len);
        nz += len;
        A.ptr[f + 1] = nz;
        bvec[f] = b;
    }
    memcpy(x, x0, sizeof(double) * (size_t)nf);
    const int status = csr_bicgstab(&A, bvec, x, rtol);
    free(A.ptr); free(A.col); free(A.val); free(bvec); free(rc); free(rv);
    return status;
}

static int sie_solve(const hf_program *P, hfr_fields *F, int d, double rtol)
{
    return sie_solve_x(P, d, 0, F->us[d], F->u[d], rtol);
}

/* BDF2 (hig-flow-step.c:992-1179; viscoelastic
 * hig-flow-step-viscoelastic.c:1320-1513): every direction's first solve
 * into uaux, then the second with right-hand side bracket * dt/3 +
 * (4 uaux - u)/3 (hig-flow-step.c:1119-1120) into u* */
static int bdf2_velocity(const hf_program *P, hfr_fields *F, double rtol)
{
    const int D = P->par.dim;
    double *ebr[3] = {0}, *ua[3] = {0};
    int rc = 0;
    for (int d = 0; d < D; d++) {
        ebr[d] = malloc(sizeof(double) * (size_t)P->nfacet[d]);
        ua[d] = malloc(sizeof(double) * (size_t)P->nfacet[d]);
        velocity_stage_e(P, F, d, ebr[d]);
    }
    for (int d = 0; d < D && rc == 0; d++) {
        memcpy(ua[d], F->us[d], sizeof(double) * (size_t)P->nfacet[d]);
        rc = sie_solve_x(P, d, 0, ua[d], F->u[d], rtol);
    }
    for (int d = 0; d < D && rc == 0; d++) {
        for (int f = 0; f < P->nfacet[d]; f++) {
            double r = ebr[d][f];
            r *= 1.0 / 3.0 * P->par.dt;
            r += (4.0 * ua[d][f] - F->u[d][f]) / 3.0;
            F->us[d][f] = r;
        }
        rc = sie_solve_x(P, d, 1, F->us[d], ua[d], rtol);
    }
    for (int d = 0; d < D; d++) { free(ebr[d]); free(ua[d]); }
    return rc;
}

/* ------------------------------------------------------------------ */
/* Poisson: higflow_pressure (hig-flow-step.c:48-131)                 */
/* ------------------------------------------------------------------ */
static void spmv(const hf_program *P, const double *x, double *y)
{
    for (int r = 0; r < P->ncell; r++) {
        if (r == P->pin_row) { y[r] = x[r]; continue; }
        double s = 0.0;
        for (int64_t k = P->p_ptr[r]; k < P->p_ptr[r + 1]; k++) s += P->p_val[k] * x[P->p_col[k]];
        y[r] = s;
    }
}

static double dot(int n, const double *a, const double *b)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

static int poisson(const hf_program *P, const double *bvec, double *x, double rtol, int *iters)
{
    const int n = P->ncell;
    double *mem = malloc(sizeof(double) * (size_t)n * 9);
    double *r = mem, *rh = r + n, *p = rh + n, *v = p + n, *s = v + n, *t = s + n, *ph = t + n,
           *sh = ph + n, *dinv = sh + n;
    for (int i = 0; i < n; i++) {
        double dg = 0.0;
        if (i == P->pin_row) dg = 1.0;
        else
            for (int64_t k = P->p_ptr[i]; k < P->p_ptr[i + 1]; k++)
                if (P->p_col[k] == i) dg += P->p_val[k];
        dinv[i] = dg != 0.0 ? 1.0 / dg : 1.0;
    }
    spmv(P, x, r);
    for (int i = 0; i < n; i++) r[i] = bvec[i] - r[i];
    double bn = sqrt(dot(n, bvec, bvec));
    double tol = rtol * (bn > 0 ? bn : 1.0);
    double rn = sqrt(dot(n, r, r));
    memcpy(rh, r, sizeof(double) * (size_t)n);
    memset(p, 0, sizeof(double) * (size_t)n);
    memset(v, 0, sizeof(double) * (size_t)n);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int it = 0, restarts = 0;
    while (rn > tol && it < 200000) {
        double rho1 = dot(n, rh, r);
        if (rho1 == 0.0 || omega == 0.0) {
            if (++restarts > 100) break;
            spmv(P, x, r);
            for (int i = 0; i < n; i++) r[i] = bvec[i] - r[i];
            memcpy(rh, r, sizeof(double) * (size_t)n);
            memset(p, 0, sizeof(double) * (size_t)n);
            memset(v, 0, sizeof(double) * (size_t)n);
            rho = alpha = omega = 1.0;
            continue;
        }
        double beta = (rho1 / rho) * (alpha / omega);
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        for (int i = 0; i < n; i++) ph[i] = dinv[i] * p[i];
        spmv(P, ph, v);
        alpha = rho1 / dot(n, rh, v);
        for (int i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
        for (int i = 0; i < n; i++) sh[i] = dinv[i] * s[i];
        spmv(P, sh, t);
        double tt = dot(n, t, t);
        omega = tt > 0.0 ? dot(n, t, s) / tt : 0.0;
        for (int i = 0; i < n; i++) {
            x[i] += alpha * ph[i] + omega * sh[i];
            r[i] = s[i] - omega * t[i];
        }
        rho = rho1;
        rn = sqrt(dot(n, r, r));
        it++;
        if (it % 50 == 0) {   /* refresh the true residual */
            spmv(P, x, r);
            for (int i = 0; i < n; i++) r[i] = bvec[i] - r[i];
            rn = sqrt(dot(n, r, r));
        }
    }
    if (iters) *iters = it;
    free(mem);
    return rn <= tol ? 0 : HF_ERR_NOT_CONVERGED;
}

static int pressure_stage(const hf_program *P, hfr_fields *F, double rtol, int *iters)
{
    const int D = P->par.dim, n = P->ncell;
    double *bvec = malloc(sizeof(double) * (size_t)n);
    for (int cc = 0; cc < n; cc++) {
        const double *cd = P->delta + (size_t)P->cell_delta[cc] * D;
        double sumdudx = 0.0;
        for (int dim = 0; dim < D; dim++) {
            double ustarl = q(P, P->div_slots[(size_t)HF_P_UL(dim) * n + cc], F->us[dim]);
            double ustarr = q(P, P->div_slots[(size_t)HF_P_UR(dim) * n + cc], F->us[dim]);
            double dudx = (ustarr - ustarl) / (2.0 * 0.5 * cd[dim]);
            sumdudx += dudx;
        }
        bvec[cc] = sumdudx / P->par.dt + P->p_brhs[cc];
    }
    double *x = P->par.projtype == HF_INCREMENTAL ? F->dp : F->p;
    if (P->pin_row >= 0) {
        bvec[P->pin_row] = P->par.projtype == HF_INCREMENTAL ? P->pin_value - F->p[P->pin_row] : P->pin_value;
    }
    int rc = poisson(P, bvec, x, rtol, iters);
    free(bvec);
    return rc;
}

/* final velocity and pressure (hig-flow-step.c:242-340) */
static void final_stage(const hf_program *P, hfr_fields *F)
{
    const int D = P->par.dim;
    const double *pp = P->par.projtype == HF_INCREMENTAL ? F->dp : F->p;
    for (int d = 0; d < D; d++) {
        const int nf = P->nfacet[d];
        for (int f = 0; f < nf; f++) {
            const double *fd = P->delta + (size_t)P->vel_delta[d][f] * D;
            double pl = q(P, P->vel_slots[d][(size_t)HF_V_PL * nf + f], pp);
            double pr = q(P, P->vel_slots[d][(size_t)HF_V_PR * nf + f], pp);
            double dpdx = (pr - pl) / (2.0 * 0.5 * fd[d]);
            F->u[d][f] = F->us[d][f] - P->par.dt * dpdx;
        }
    }
    if (P->par.projtype == HF_INCREMENTAL)
        for (int c = 0; c < P->ncell; c++) F->p[c] = F->p[c] + F->dp[c];
}

/* ------------------------------------------------------------------ */
/* viscoelastic cell stage                                             */
/* ------------------------------------------------------------------ */
/* hig_flow_jacobi, hig-flow-step-viscoelastic.c:1517-1600 */
static void jacobi(int D, double A[3][3], double d[3], double V[3][3])
{
    double bb[3], z[3];
    const int NMAX = 500;
    for (int ip = 0; ip < D; ip++) {
        for (int iq = 0; iq < D; iq++) V[ip][iq] = 0.0;
        V[ip][ip] = 1.0;
        bb[ip] = A[ip][ip];
        d[ip] = bb[ip];
        z[ip] = 0.0;
    }
    for (int i = 1; i <= NMAX; i++) {
        double tresh, sm = 0.0;
        for (int ip = 0; ip < D - 1; ip++)
            for (int iq = ip + 1; iq < D; iq++) sm += fabs(A[ip][iq]);
        if (sm == 0.0) return;
        if (i < 4) tresh = 0.2 * sm / (D * D);
        else tresh = 0.0;
        for (int ip = 0; ip < D - 1; ip++)
            for (int iq = ip + 1; iq < D; iq++) {
                double g = 100.0 * fabs(A[ip][iq]);
                if ((i > 4) && (fabs(d[ip]) + g == fabs(d[ip])) && (fabs(d[iq]) + g == fabs(d[iq]))) {
                    A[ip][iq] = 0.0;
                } else if (fabs(A[ip][iq]) > tresh) {
                    double t, theta;
                    double h = d[iq] - d[ip];
                    if (fabs(h) + g == fabs(h)) {
                        t = A[ip][iq] / h;
                    } else {
                        theta = 0.5 * h / A[ip][iq];
                        t = 1.0 / (fabs(theta) + sqrt(1.0 + theta * theta));
                        if (theta < 0.0) t = -t;
                    }
                    double c = 1.0 / sqrt(1.0 + t * t);
                    double s = t * c;
                    double tau = s / (1.0 + c);
                    h = t * A[ip][iq];
                    z[ip] = z[ip] - h;
                    z[iq] = z[iq] + h;
                    d[ip] = d[ip] - h;
                    d[iq] = d[iq] + h;
                    A[ip][iq] = 0.0;
                    for (int j = 0; j <= ip - 1; j++) {
                        g = A[j][ip]; h = A[j][iq];
                        A[j][ip] = g - s * (h + g * tau);
                        A[j][iq] = h + s * (g - h * tau);
                    }
                    for (int j = ip + 1; j <= iq - 1; j++) {
                        g = A[ip][j]; h = A[j][iq];
                        A[ip][j] = g - s * (h + g * tau);
                        A[j][iq] = h + s * (g - h * tau);
                    }
                    for (int j = iq + 1; j < D; j++) {
                        g = A[ip][j]; h = A[iq][j];
                        A[ip][j] = g - s * (h + g * tau);
                        A[iq][j] = h + s * (g - h * tau);
                    }
                    for (int j = 0; j < D; j++) {
                        g = V[j][ip]; h = V[j][iq];
                        V[j][ip] = g - s * (h + g * tau);
                        V[j][iq] = h + s * (g - h * tau);
                    }
                }
            }
        for (int ip = 0; ip < D; ip++) {
            bb[ip] = bb[ip] + z[ip];
            d[ip] = bb[ip];
            z[ip] = 0.0;
        }
    }
}

/* R^t A R (hig_flow_matrix_product, :1603) */
static void mprod(int D, double A[3][3], double R[3][3], double B[3][3])
{
    for (int i = 0; i < D; i++)
        for (int j = 0; j < D; j++) {
            B[i][j] = 0.0;
            for (int k = 0; k < D; k++)
                for (int l = 0; l < D; l++) B[i][j] += R[k][i] * A[k][l] * R[l][j];
        }
}

/* R A R^t (hig_flow_matrix_transpose_product, :1617) */
static void mtprod(int D, double A[3][3], double R[3][3], double B[3][3])
{
    for (int i = 0; i < D; i++)
        for (int j = 0; j < D; j++) {
            B[i][j] = 0.0;
            for (int k = 0; k < D; k++)
                for (int l = 0; l < D; l++) B[i][j] += R[i][k] * A[k][l] * R[j][l];
        }
}

static double kinv(int kind, double l)
{
    if (kind == HF_KERNEL_LOG) return exp(l);
    if (kind == HF_KERNEL_SQRT) return l * l;
    return l;
}

static double kjac(int kind, double l, double tol)
{
    if (kind == HF_KERNEL_LOG) return l < tol ? 1.0 / tol : 1.0 / l;
    if (kind == HF_KERNEL_SQRT) return l < tol ? 0.5 / sqrt(tol) : 0.5 / sqrt(l);
    return 1.0;
}

/* hig_flow_convective_cell_term_cubista (hig-flow-step.c:1185-1358) */
static double cubista_cell(double kl, double kr, double kll, double krr, int incell_l, int incell_r,
                           int incell_ll, int incell_rr, double vl, double vr, double kc, double cdelta)
{
    const double a = 1.7500, b = 0.3750, c = 0.7500, d = 0.1250, e = 0.2500;
    double vbar, fi, conv1 = 0.0, conv2 = 0.0;
    vbar = vr;
    if (vbar > 0.0) {
        if (FLT_EQ(kr, kl)) {
            conv1 = vbar * kc;
        } else {
            fi = (kc - kl) / (kr - kl);
            if ((fi <= 0.0) || (fi >= 1.0)) {
                conv1 = vbar * kc;
            } else {
                if (fi < b) conv1 = incell_l == 1 ? vbar * (a * kc - c * kl) : vbar * kc;
                if ((fi >= b) && (fi <= c))
                    conv1 = ((incell_l == 1) && (incell_r == 1)) ? vbar * (c * kc + b * kr - d * kl) : vbar * kc;
                if (fi > c) conv1 = incell_r == 1 ? vbar * (e * kc + c * kr) : vbar * kc;
            }
        }
    } else {
        if ((incell_r == 1) && (incell_rr == 1)) {
            if (FLT_EQ(kc, krr)) {
                conv1 = vbar * kr;
            } else {
                fi = (kr - krr) / (kc - krr);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv1 = vbar * kr;
                } else {
                    if (fi < b) conv1 = vbar * (a * kr - c * krr);
                    if ((fi >= b) && (fi <= c)) conv1 = vbar * (c * kr + b * kc - d * krr);
                    if (fi > c) conv1 = vbar * (c * kc + e * kr);
                }
            }
        } else if ((incell_r == 1) && (incell_rr == 0)) {
            if (FLT_EQ(kc, krr)) {
                conv1 = vbar * kr;
            } else {
                fi = (kr - krr) / (kc - krr);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv1 = vbar * kr;
                } else {
                    if (fi <= c) conv1 = vbar * kr;
                    if (fi > c) conv1 = vbar * (c * kc + e * kr);
                }
            }
        } else {
            vbar = vr;
            conv1 = vbar * kc;
            vbar = vl;
            if (vbar > 0.0) conv2 = vbar * kl;
            else conv2 = vbar * kc;
            return ((conv1 - conv2) / cdelta);
        }
    }
    vbar = vl;
    if (vbar > 0.0) {
        if ((incell_l == 1) && (incell_ll == 1)) {
            if (FLT_EQ(kc, kll)) {
                conv2 = vbar * kl;
            } else {
                fi = (kl - kll) / (kc - kll);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv2 = vbar * kl;
                } else {
                    if (fi < b) conv2 = vbar * (a * kl - c * kll);
                    if ((fi >= b) && (fi <= c)) conv2 = vbar * (b * kc + c * kl - d * kll);
                    if (fi > c) conv2 = vbar * (c * kc + e * kl);
                }
            }
        } else if ((incell_l == 1) && (incell_ll == 0)) {
            if (FLT_EQ(kc, kll)) {
                conv2 = vbar * kl;
            } else {
                fi = (kl - kll) / (kc - kll);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv2 = vbar * kl;
                } else {
                    if (fi <= c) conv2 = vbar * kl;
                    if (fi > c) conv2 = vbar * (c * kc + e * kl);
                }
            }
        } else {
            vbar = vr;
            if (vbar > 0.0) conv1 = vbar * kc;
            else conv1 = vbar * kr;
            vbar = vl;
            conv2 = vbar * kc;
            return ((conv1 - conv2) / cdelta);
        }
    } else {
        if (FLT_EQ(kl, kr)) {
            conv2 = vbar * kc;
        } else {
            fi = (kc - kr) / (kl - kr);
            if ((fi <= 0.0) || (fi >= 1.0)) {
                conv2 = vbar * kc;
            } else {
                if (fi < b) conv2 = incell_r == 1 ? vbar * (a * kc - c * kr) : vbar * kc;
                if ((fi >= b) && (fi <= c))
                    conv2 = ((incell_l == 1) && (incell_r == 1)) ? vbar * (c * kc + b * kl - d * kr) : vbar * kc;
                if (fi > c) conv2 = incell_l == 1 ? vbar * (e * kc + c * kl) : vbar * kc;
            }
        }
    }
    return ((conv1 - conv2) / cdelta);
}

/* velocity-derivative tensor (hig-flow-step-generalized-newtonian.c:14-97) */
static void du_stage(const hf_program *P, hfr_fields *F)
{
    const int D = P->par.dim, n = P->ncell, ns = P->cell_nslot;
    (void)ns;
    for (int cc = 0; cc < n; cc++) {
#define CS(s) P->cell_slots[(size_t)(s) * n + cc]
        const double *cd = P->delta + (size_t)P->cell_delta[cc] * D;
        int qb = HF_C_BLK0 + HF_C_NB * D;
        for (int dim = 0; dim < D; dim++) {
            const int B = HF_C_BLK0 + HF_C_NB * dim;
            for (int dim2 = 0; dim2 < D; dim2++) {
                double ul, ur;
                if (dim == dim2) {
                    ul = q(P, CS(B + HF_C_UVL), F->u[dim]);
                    ur = q(P, CS(B + HF_C_UVR), F->u[dim]);
                } else {
                    int pair = 0;
                    for (int a = 0; a < D; a++)
                        for (int bq = 0; bq < D; bq++) {
                            if (bq == a) continue;
                            if (a == dim && bq == dim2) goto found;
                            pair++;
                        }
                found:;
                    int Q = qb + HF_C_NQ * pair;
                    double vrr = q(P, CS(Q + 0), F->u[dim]);
                    double vr = q(P, CS(B + HF_C_UVR), F->u[dim]);
                    double vl = q(P, CS(B + HF_C_UVL), F->u[dim]);
                    double vll = q(P, CS(Q + 1), F->u[dim]);
                    ul = 0.25 * (vll + vl + vr + vrr);
                    vrr = q(P, CS(Q + 2), F->u[dim]);
                    vr = q(P, CS(B + HF_C_UVR), F->u[dim]);
                    vl = q(P, CS(B + HF_C_UVL), F->u[dim]);
                    vll = q(P, CS(Q + 3), F->u[dim]);
                    ur = 0.25 * (vll + vl + vr + vrr);
                }
                F->Du[dim * D + dim2][cc] = (ur - ul) / (2.0 * 0.5 * cd[dim2]);
            }
        }
#undef CS
    }
}

/* ------------------------------------------------------------------ */
/* Mittag-Leffler function E_{alpha,beta}(z), the GPTT model's         */
/* generalised exponential (hig_flow_calculate_m_gptt,                 */
/* hig-flow-step-viscoelastic.c:1771-1830, evaluated by mlfv,          */
/* hig-flow-mittag-leffler.c:117-366).  The algorithm is the published */
/* one of Gorenflo, Loutchko and Luchko (Fract. Calc. Appl. Anal. 5,   */
/* 2002): the power series near the origin, the integral               */
/* representation (a ray integral of K and an arc integral of P, each  */
/* by a six-level Romberg rule) in the middle, the asymptotic series   */
/* far out for alpha <= 1, and for alpha > 1 the reduction to smaller  */
/* alpha (roots of z).  rho = 10^-fi is the accuracy the region bounds */
/* and the Romberg order derive from (the reference passes fi = 6).    */
/* Powers of z are taken in polar form, |z|^p e^{i p arg z}, as the    */
/* reference does.  Only the real part enters the model; the imaginary */
/* part of the asymptotic leading term is the true one here (the       */
/* reference's sine there has the wrong sign, :287-288, :317-318,      */
/* which never reaches a real part).                                   */
/* ------------------------------------------------------------------ */
typedef struct hfr_cx { double re, im; } hfr_cx;

static hfr_cx cx_make(double re, double im) { hfr_cx z = {re, im}; return z; }
static hfr_cx cx_polar(double r, double t) { return cx_make(r * cos(t), r * sin(t)); }
static hfr_cx cx_add(hfr_cx a, hfr_cx b) { return cx_make(a.re + b.re, a.im + b.im); }
static hfr_cx cx_scale(hfr_cx a, double s) { return cx_make(s * a.re, s * a.im); }
static hfr_cx cx_div(hfr_cx a, hfr_cx b)
{
    const double d = b.re * b.re + b.im * b.im;
    return cx_make((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}

typedef struct ml_ctx { double a, b, eps; hfr_cx z; } ml_ctx;

/* the ray integrand K(r) = r^((1-b)/a) e^(-r^(1/a)) / (pi a)
 *   * (r sin(pi (1-b)) - z sin(pi (1-b+a))) / (r^2 - 2 r z cos(pi a) + z^2) */
static hfr_cx ml_ray(const ml_ctx *c, double r)
{
    const double a = c->a, b = c->b;
    const double A = pow(r, (1.0 - b) / a) * exp(-pow(r, 1.0 / a)) / (M_PI * a);
    const double s1 = r * sin(M_PI * (1.0 - b)), s2 = sin(M_PI * (1.0 - b + a));
    const double e = 2.0 * r * cos(M_PI * a);
    const hfr_cx z = c->z;
    const hfr_cx num = cx_make(s1 - s2 * z.re, -s2 * z.im);
    const hfr_cx den = cx_make(r * r - e * z.re + (z.re * z.re - z.im * z.im), -e * z.im + 2.0 * z.re * z.im);
    return cx_scale(cx_div(num, den), A);
}

/* the arc integrand P(phi) on |zeta| = eps:
 *   eps^(1+(1-b)/a) e^(eps^(1/a) cos(phi/a)) e^(i w) / (2 pi a (eps e^(i phi) - z)),
 *   w = eps^(1/a) sin(phi/a) + phi (1 + (1-b)/a) */
static hfr_cx ml_arc(const ml_ctx *c, double phi)
{
    const double a = c->a, b = c->b, eps = c->eps;
    const double p = 1.0 + (1.0 - b) / a, er = pow(eps, 1.0 / a);
    const double A = pow(eps, p) * exp(er * cos(phi / a)) / (2.0 * M_PI * a);
    const double w = er * sin(phi / a) + phi * p;
    const hfr_cx den = cx_make(eps * cos(phi) - c->z.re, eps * sin(phi) - c->z.im);
    return cx_div(cx_polar(A, w), den);
}

/* Romberg's rule with n levels (trapezoid sums of 1, 2, 4, ... panels,
 * Richardson-extrapolated); the ray integral always takes six levels, the
 * arc integral fi (rombint, hig-flow-mittag-leffler.c:53-56) */
static hfr_cx ml_romberg(hfr_cx (*f)(const ml_ctx *, double), const ml_ctx *c, double lo, double hi, int n)
{
    if (f == ml_ray) n = 6;
    if (n > 8) n = 8;   /* the reference's table holds eight levels (:46-50) */
    if (n < 1) n = 1;
    hfr_cx prev[16], cur[16];
    double h = hi - lo;
    const hfr_cx fa = f(c, lo), fb = f(c, hi);
    prev[0] = cx_make(h * (fa.re + fb.re) / 2.0, h * (fa.im + fb.im) / 2.0);
    int npts = 1;
    for (int i = 1; i < n; i++) {
        hfr_cx s = cx_make(0.0, 0.0);
        for (int j = 1; j <= npts; j++) s = cx_add(s, f(c, lo + h * (j - 0.5)));
        cur[0] = cx_make((prev[0].re + h * s.re) / 2.0, (prev[0].im + h * s.im) / 2.0);
        double q = 1.0;
        for (int k = 1; k <= i; k++) {
            q *= 4.0;
            cur[k] = cx_make((q * cur[k - 1].re - prev[k - 1].re) / (q - 1.0),
                             (q * cur[k - 1].im - prev[k - 1].im) / (q - 1.0));
        }
        for (int k = 0; k <= i; k++) prev[k] = cur[k];
        npts *= 2;
        h /= 2.0;
    }
    return prev[n - 1];
}

/* z^((1-b)/a) e^(z^(1/a)) / a, the leading term of the integral and
 * asymptotic forms */
static hfr_cx ml_lead(double a, double b, double az, double th)
{
    const double ra = pow(az, 1.0 / a);
    const double mag = (pow(az, (1.0 - b) / a) / a) * exp(ra * cos(th / a));
    return cx_polar(mag, th * (1.0 - b) / a + ra * sin(th / a));
}

static hfr_cx ml_eval(double a, double b, hfr_cx z, int fi)
{
    const double az = sqrt(z.re * z.re + z.im * z.im);
    const double th = atan2(z.im, z.re), ath = fabs(th);
    const double rho = pow(10.0, -fi);
    const int series = (a < 1.0 && az <= 1.0) ||
                       (1.0 <= a && a < 2.0 && az <= floor(20.0 / pow(2.1 - a, 5.5 - 2.0 * a))) ||
                       (a >= 2.0 && az <= 50.0);
    if (series) {
        /* sum z^k / Gamma(a k + b) from the first k with a k + b > 0, two
         * terms at a time, until the sum stops changing */
        int k = 0;
        while (a * k + b <= 0.0) k++;
        hfr_cx s = cx_make(pow(az, k) * cos(th * k) / tgamma(a * k + b), pow(az, k) * sin(th * k) / tgamma(a * k + b));
        for (int it = 0; it < 100000; it++) {
            const hfr_cx old = s;
            for (int t = 0; t < 2; t++) {
                k++;
                const double g = tgamma(a * k + b), pk = pow(az, k);
                s = cx_make(s.re + pk * cos(th * k) / g, s.im + pk * sin(th * k) / g);
            }
            if (s.re == old.re && s.im == old.im) break;
        }
        return s;
    }
    if (a <= 1.0 && az <= floor(5.0 * a + 10.0)) {
        const double r0 = fmax(fmax(1.0, 2.0 * az), pow(-2.0 * log(rho * M_PI / 6.0), a));
        ml_ctx c = {a, b, 0.0, z};
        const double pa = M_PI * a;
        if (ath > pa && fabs(ath - pa) > rho) {
            if (b <= 1.0) return ml_romberg(ml_ray, &c, 0.0, r0, fi);
            c.eps = 1.0;
            return cx_add(ml_romberg(ml_ray, &c, c.eps, r0, fi), ml_romberg(ml_arc, &c, -pa, pa, fi));
        }
        if (ath < pa && fabs(ath - pa) > rho) {
            if (b <= 1.0) return cx_add(ml_romberg(ml_ray, &c, 0.0, r0, fi), ml_lead(a, b, az, th));
            c.eps = az / 2.0;
            const hfr_cx arc = ml_romberg(ml_arc, &c, -pa, pa, fi);
            return cx_add(cx_add(arc, ml_romberg(ml_ray, &c, c.eps, r0, fi)), ml_lead(a, b, az, th));
        }
        c.eps = az + 0.5;
        return cx_add(ml_romberg(ml_ray, &c, c.eps, r0, fi), ml_romberg(ml_arc, &c, -pa, pa, fi));
    }
    if (a <= 1.0) {
        /* asymptotic: the leading term inside the sector, minus
         * sum_k z^-k / Gamma(b - a k) (terms with b - a k an integer skipped) */
        hfr_cx s = cx_make(0.0, 0.0);
        if (ath < (M_PI * a / 2.0 + fmin(M_PI, M_PI * a)) / 2.0) s = ml_lead(a, b, az, th);
        for (int k = 1; k <= floor(fi / log10(az)); k++) {
            const double g = b - a * k;
            if (ceil(g) == floor(g)) continue;
            const double pk = pow(az, -k);
            s = cx_make(s.re - pk * cos(th * k) / tgamma(g), s.im - (-(pk * sin(th * k))) / tgamma(g));
        }
        return s;
    }
    if (a >= 2.0) {
        /* E_{a,b}(z) = 1/(m+1) sum_h E_{a/(m+1),b}(z^(1/(m+1)) e^(2 pi i h/(m+1))) */
        const int m = (int)floor(a / 2.0);
        hfr_cx s = cx_make(0.0, 0.0);
        for (int h = 0; h <= m; h++) {
            const double r = pow(az, 1.0 / (m + 1.0));
            s = cx_add(s, ml_eval(a / (m + 1), b, cx_polar(r, (2.0 * M_PI * h + th) / (m + 1.0)), fi));
        }
        return cx_scale(s, 1.0 / (m + 1.0));
    }
    /* 1 < a < 2: E_{a,b}(z) = (E_{a/2,b}(sqrt z) + E_{a/2,b}(-sqrt z)) / 2 */
    const double r = sqrt(az);
    const hfr_cx z1 = cx_make(r * cos(th / 2.0), r * sin(th / 2.0));
    const hfr_cx e1 = ml_eval(a / 2.0, b, z1, fi), e2 = ml_eval(a / 2.0, b, cx_make(-z1.re, -z1.im), fi);
    return cx_make((e1.re + e2.re) / 2.0, (e1.im + e2.im) / 2.0);
}

/* the GPTT factor Gamma(beta_g) E_{alpha_g,beta_g}(eps Re De tr(S) / (1 - beta)) */
static double gptt_factor(const hf_params *pr, double trS)
{
    const hfr_cx z = cx_make(pr->epsilon * pr->Re * pr->De * trS / (1.0 - pr->beta), 0.0);
    return ml_eval(pr->alpha_gptt, pr->beta_gptt, z, 6).re;
}

/* the evaluation alone, for the tests of the device form */
void hfr_mittag_leffler(double alpha, double beta, double zr, double zi, int fi, double *out)
{
    const hfr_cx e = ml_eval(alpha, beta, cx_make(zr, zi), fi);
    out[0] = e.re;
    out[1] = e.im;
}

/* implicit Euler constitutive step of one cell (higflow_implicit_euler_
 * constitutive_equation, hig-flow-step-viscoelastic.c:841-877): right-hand
 * side for every (i, j), the Kronecker system of hig_flow_kernel_system_matrix
 * (:1964-1989), Gauss elimination with partial pivoting
 * (hig_flow_solve_system_constitutive_equation, :1912-1953) */
static void implicit_cell(const hf_program *P, hfr_fields *F, const hf_params *pr, int cc, uint32_t fl,
                          const double *cd, const double *vl, const double *vr, const double *uc,
                          double K[3][3], double RHS[3][3], double Om[3][3], double **knew)
{
    const int D = P->par.dim, n = D * D, nc = P->ncell;
    const double dt = pr->dt;
    double b[9], w[9][10];
    for (int i = 0; i < D; i++)
        for (int j = 0; j < D; j++) {
            const double *Kf = F->K[i * D + j];
            double rhs = 0.0;
            for (int dim = 0; dim < D; dim++) {
                const int B = HF_C_BLK0 + HF_C_NB * dim;
                int il = (fl >> (4 * dim + 0)) & 1, ir = (fl >> (4 * dim + 1)) & 1;
                int ill = (fl >> (4 * dim + 2)) & 1, irr = (fl >> (4 * dim + 3)) & 1;
                double kl = q(P, P->cell_slots[(size_t)(B + HF_C_KL) * nc + cc], Kf);
                double kr = q(P, P->cell_slots[(size_t)(B + HF_C_KR) * nc + cc], Kf);
                if (pr->ve_convecdiscrtype == HF_CELL_CUBISTA) {
                    double kll = q(P, P->cell_slots[(size_t)(B + HF_C_KLL) * nc + cc], Kf);
                    double krr = q(P, P->cell_slots[(size_t)(B + HF_C_KRR) * nc + cc], Kf);
                    rhs -= cubista_cell(kl, kr, kll, krr, il, ir, ill, irr, vl[dim], vr[dim], K[i][j], cd[dim]);
                } else {
                    double dk;
                    if ((il == 1) && (ir == 1)) dk = (kr - kl) / (2.0 * 1.0 * cd[dim]);
                    else if (ir == 1) dk = (kr - K[i][j]) / (1.0 * cd[dim]);
                    else dk = (K[i][j] - kl) / (1.0 * cd[dim]);
                    rhs -= uc[dim] * dk;
                }
            }
            rhs += RHS[i][j];
            rhs *= dt;
            rhs += K[i][j];
            b[i * D + j] = rhs;
        }
    double I[3][3];
    for (int i = 0; i < D; i++)
        for (int j = 0; j < D; j++) I[i][j] = i == j ? 1.0 : 0.0;
    for (int i = 0; i < D; i++)
        for (int j = i; j < D; j++)
            for (int k = 0; k < D; k++)
                for (int l = 0; l < D; l++) {
                    if (i == j) {
                        w[i * D + k][j * D + l] = I[k][l] - dt * Om[k][l] - dt * Om[i][i] * I[k][l];
                    } else {
                        w[i * D + k][j * D + l] = dt * Om[j][i] * I[k][l];
                        w[j * D + l][i * D + k] = -dt * Om[j][i] * I[k][l];
                    }
                }
    for (int j = 0; j < n; j++) w[j][n] = b[j];
    for (int k = 0; k < n - 1; k++) {
        double mx = fabs(w[k][k]);
        int l = k;
        for (int i = k + 1; i < n; i++)
            if (fabs(w[i][k]) > mx) { mx = fabs(w[i][k]); l = i; }
        if (l != k)
            for (int j = k; j <= n; j++) { const double aux = w[k][j]; w[k][j] = w[l][j]; w[l][j] = aux; }
        for (int i = k + 1; i < n; i++) {
            const double s = w[i][k] / w[k][k];
            w[i][k] = 0;
            for (int j = k + 1; j <= n; j++) w[i][j] -= s * w[k][j];
        }
    }
    b[n - 1] = w[n - 1][n] / w[n - 1][n - 1];
    for (int i = n - 2; i >= 0; i--) {
        double s = 0;
        for (int j = i + 1; j < n; j++) s += w[i][j] * b[j];
        b[i] = (w[i][n] - s) / w[i][i];
    }
    for (int i = 0; i < D; i++)
        for (int j = i; j < D; j++) {
            knew[i * D + j][cc] = b[i * D + j];
            if (i != j) knew[j * D + i][cc] = b[i * D + j];
        }
}

/* explicit constitutive step (hig-flow-step-viscoelastic.c:352-544); the new
 * kernel goes to knew[] (the reference stores it in dpS, then copies) */
static void constitutive_stage(const hf_program *P, hfr_fields *F, double **knew)
{
    const int D = P->par.dim, n = P->ncell;
    const hf_params *pr = &P->par;
    const double Re = pr->Re, De = pr->De, tol = pr->kernel_tol, small = EPSMACH;
    for (int cc = 0; cc < n; cc++) {
#define CS(s) P->cell_slots[(size_t)(s) * n + cc]
        const double *cd = P->delta + (size_t)P->cell_delta[cc] * D;
        const uint32_t fl = P->cell_flags[cc];
        double Du[3][3], S[3][3], K[3][3], KC[3][3];
        double trS = 0.0;
        for (int i = 0; i < D; i++) {
            for (int j = 0; j < D; j++) {
                Du[i][j] = q(P, CS(HF_C_SELF), F->Du[i * D + j]);
                S[i][j] = q(P, CS(HF_C_SELF), F->S[i * D + j]);
                K[i][j] = q(P, CS(HF_C_SELF), F->K[i * D + j]);
                KC[i][j] = K[i][j];
            }
            trS += S[i][i];
        }
        double R[3][3], Kl[3], lam[3];
        jacobi(D, KC, Kl, R);
        for (int dim = 0; dim < D; dim++) lam[dim] = kinv(pr->kernel, Kl[dim]);
        double Mt[3][3], M[3][3];
        for (int i = 0; i < D; i++)
            for (int j = 0; j < D; j++) {
                Mt[i][j] = Du[i][j];
                if (pr->ve_model == HF_LPTT || pr->ve_model == HF_GPTT) Mt[i][j] -= pr->xi * 0.5 * (Du[i][j] + Du[j][i]);
            }
        mprod(D, Mt, R, M);
        /* hig_flow_calculate_omega (:1667) */
        double Oa[3][3], Om[3][3];
        for (int i = 0; i < D - 1; i++) {
            for (int j = i + 1; j < D; j++) {
                Oa[i][j] = (M[i][j] * lam[j] + M[j][i] * lam[i]) / (lam[j] - lam[i] + small);
                Oa[j][i] = -Oa[i][j];
            }
            Oa[i][i] = 0.0;
        }
        Oa[D - 1][D - 1] = 0.0;
        mtprod(D, Oa, R, Om);
        double jl[3];
        for (int i = 0; i < D; i++) jl[i] = kjac(pr->kernel, lam[i], tol);
        /* hig_flow_calculate_b (:1683) */
        double Ba[3][3], BB[3][3];
        for (int i = 0; i < D; i++) {
            for (int j = i + 1; j < D; j++) { Ba[i][j] = 0.0; Ba[j][i] = 0.0; }
            Ba[i][i] = M[i][i] * lam[i] * jl[i];
        }
        mtprod(D, Ba, R, BB);
        /* model terms (:1710-1770) */
        double Ma[3][3], MM[3][3];
        /* e-FENE (:1855-1876): trace of the eigenvalues */
        double trA = 0.0, fA = 0.0;
        for (int i = 0; i < D; i++) trA += lam[i];
        if (pr->ve_model == HF_E_FENE) {
            const double b = pr->L2_fene, lf = pr->lambda_fene, E = pr->E_fene;
            fA = b / (b - trA) - E * sqrt(b) * exp(-sqrt(trA) / lf) * (1.0 / (trA * lf) + 1 / (trA * sqrt(trA)));
        }
        /* GPTT (:1771-1830): Gamma(beta_g) E_{alpha_g,beta_g}(eps Re De tr S / (1 - beta)) */
        const double mlv = pr->ve_model == HF_GPTT ? gptt_factor(pr, trS) : 0.0;
        for (int i = 0; i < D; i++) {
            for (int j = i + 1; j < D; j++) { Ma[i][j] = 0.0; Ma[j][i] = 0.0; }
            if (pr->ve_model == HF_GIESEKUS) {
                double aux = 1.0 - lam[i];
                Ma[i][i] = (aux - pr->alpha * aux * aux) * jl[i];
            } else if (pr->ve_model == HF_LPTT) {
                Ma[i][i] = (1.0 - lam[i]) * (1.0 + (pr->epsilon * Re * De * trS) / (1.0 - pr->beta)) * jl[i];
            } else if (pr->ve_model == HF_GPTT) {
                Ma[i][i] = (1.0 - lam[i]) * pr->gamma_gptt * mlv * jl[i];
            } else if (pr->ve_model == HF_E_FENE) {
                Ma[i][i] = (1.0 - fA * lam[i]) * jl[i];
            } else {
                Ma[i][i] = (1.0 - lam[i]) * jl[i];
            }
        }
        mtprod(D, Ma, R, MM);
        /* hig_flow_kernel_rhs (:1631) */
        double OK[3][3], KO[3][3], RHS[3][3];
        for (int i = 0; i < D; i++)
            for (int j = 0; j < D; j++) {
                OK[i][j] = 0.0;
                KO[i][j] = 0.0;
                for (int k = 0; k < D; k++) {
                    OK[i][j] += Om[i][k] * K[k][j];
                    KO[i][j] += K[i][k] * Om[k][j];
                }
            }
        const int implicit = pr->ve_discrtype == HF_VE_IMPLICIT;
        for (int i = 0; i < D; i++)
            for (int j = 0; j < D; j++)
                RHS[i][j] = implicit ? 2.0 * BB[i][j] + MM[i][j] / De   /* hig_flow_implicit_kernel_rhs (:1956) */
                                     : OK[i][j] - KO[i][j] + 2.0 * BB[i][j] + MM[i][j] / De;
        /* hig_flow_velocity_at_center_cell (:1879) */
        double uc[3], vl[3], vr[3];
        for (int dim = 0; dim < D; dim++) {
            const int B = HF_C_BLK0 + HF_C_NB * dim;
            vl[dim] = q(P, CS(B + HF_C_UVL), F->u[dim]);
            vr[dim] = q(P, CS(B + HF_C_UVR), F->u[dim]);
            uc[dim] = 0.5 * (vl[dim] + vr[dim]);
        }
        if (implicit) {
            implicit_cell(P, F, pr, cc, fl, cd, vl, vr, uc, K, RHS, Om, knew);
            continue;
        }
        for (int i = 0; i < D; i++) {
            for (int j = i; j < D; j++) {
                const double *Kf = F->K[i * D + j];
                double rhs = 0.0;
                for (int dim = 0; dim < D; dim++) {
                    const int B = HF_C_BLK0 + HF_C_NB * dim;
                    int il = (fl >> (4 * dim + 0)) & 1, ir = (fl >> (4 * dim + 1)) & 1;
                    int ill = (fl >> (4 * dim + 2)) & 1, irr = (fl >> (4 * dim + 3)) & 1;
                    double kl = q(P, CS(B + HF_C_KL), Kf);
                    double kr = q(P, CS(B + HF_C_KR), Kf);
                    if (pr->ve_convecdiscrtype == HF_CELL_CUBISTA) {
                        double kll = q(P, CS(B + HF_C_KLL), Kf);
                        double krr = q(P, CS(B + HF_C_KRR), Kf);
                        rhs -= cubista_cell(kl, kr, kll, krr, il, ir, ill, irr, vl[dim], vr[dim], K[i][j], cd[dim]);
                    } else {
                        double dk;
                        if ((il == 1) && (ir == 1)) dk = (kr - kl) / (2.0 * 1.0 * cd[dim]);
                        else if (ir == 1) dk = (kr - K[i][j]) / (1.0 * cd[dim]);
                        else dk = (K[i][j] - kl) / (1.0 * cd[dim]);
                        rhs -= uc[dim] * dk;
                    }
                }
                rhs += RHS[i][j];
                double kernel = K[i][j] + pr->dt * rhs;
                knew[i * D + j][cc] = kernel;
                if (i != j) knew[j * D + i][cc] = kernel;
            }
        }
#undef CS
    }
}

/* polymeric tensor (hig-flow-step-viscoelastic.c:212-347) */
static void polymeric_stage(const hf_program *P, hfr_fields *F)
{
    const int D = P->par.dim, n = P->ncell;
    const hf_params *pr = &P->par;
    const double Re = pr->Re, De = pr->De, beta = pr->beta;
    for (int cc = 0; cc < n; cc++) {
        int32_t self = P->cell_slots[(size_t)HF_C_SELF * n + cc];
        double Du[3][3], K[3][3];
        for (int i = 0; i < D; i++)
            for (int j = 0; j < D; j++) {
                Du[i][j] = q(P, self, F->Du[i * D + j]);
                K[i][j] = q(P, self, F->K[i * D + j]);
            }
        double R[3][3], lam[3], B[3][3], A[3][3];
        jacobi(D, K, lam, R);
        for (int i = 0; i < D; i++) {
            for (int j = i + 1; j < D; j++) { B[i][j] = 0.0; B[j][i] = 0.0; }
            B[i][i] = kinv(pr->kernel, lam[i]);
        }
        mtprod(D, B, R, A);
        /* the model switch of :274-309: LPTT and GPTT set xi; e-FENE computes its fA
         * there but falls through to the default (fA = a = 1, xi = 0) */
        double fA = 1.0, a = 1.0, xi = 0.0;
        if (pr->ve_model == HF_LPTT || pr->ve_model == HF_GPTT) xi = pr->xi;
        for (int i = 0; i < D; i++) {
            for (int j = 0; j < D; j++)
                F->S[i * D + j][cc] = (1.0 - beta) * (fA * A[i][j]) / (Re * De * (1.0 - xi)) - (1.0 - beta) * Du[i][j] / Re;
            F->S[i * D + i][cc] += -a * (1.0 - beta) / (Re * De * (1.0 - xi));
        }
    }
}

/* explicit Runge-Kutta velocity (higflow_explicit_runge_kutta_{2,3}_
 * intermediate_velocity, hig-flow-step.c:666-784), stage by stage: each
 * explicit Euler stage writes its output field, but its computational cell
 * reads ns->dpu (hig-flow-step.c:639), so every stage's input is u */
static void rk_stage(const hf_program *P, hfr_fields *F)
{
    const int D = P->par.dim;
    double *ua[3] = {0};
    for (int d = 0; d < D; d++) ua[d] = malloc(sizeof(double) * (size_t)P->nfacet[d]);
    hfr_fields F1 = *F;
    for (int d = 0; d < D; d++) F1.us[d] = ua[d];
    for (int d = 0; d < D; d++) velocity_stage(P, &F1, d);   /* dpuaux = E(u) */
    for (int d = 0; d < D; d++) velocity_stage(P, F, d);     /* dpustar = E(u) (input dpuaux unread) */
    if (P->par.tempdiscrtype == HF_EXPLICIT_RK2) {
        for (int d = 0; d < D; d++)
            for (int f = 0; f < P->nfacet[d]; f++) F->us[d][f] = 0.5 * (F->u[d][f] + F->us[d][f]);
    } else {
        for (int d = 0; d < D; d++)
            for (int f = 0; f < P->nfacet[d]; f++) ua[d][f] = 0.75 * F->u[d][f] + 0.25 * F->us[d][f];
        for (int d = 0; d < D; d++) velocity_stage(P, F, d);     /* dpustar = E(u) */
        for (int d = 0; d < D; d++)
            for (int f = 0; f < P->nfacet[d]; f++) F->us[d][f] = F->u[d][f] / 3.0 + 2.0 * F->us[d][f] / 3.0;
    }
    for (int d = 0; d < D; d++) free(ua[d]);
}

/* one or more full time steps; returns 0 or a negative HF_ERR_* code */
int hfr_step(const hf_program *P, hfr_fields *F, int nsteps, double rtol, int *iters)
{
    const int D = P->par.dim;
    const int ve = P->par.flowtype == HF_VISCOELASTIC;
    double *knew[9] = {0};
    if (ve)
        for (int k = 0; k < D * D; k++) knew[k] = malloc(sizeof(double) * (size_t)P->ncell);
    int rc = 0;
    for (int s = 0; s < nsteps && rc == 0; s++) {
        if (ve) {
            du_stage(P, F);
            constitutive_stage(P, F, knew);
            for (int k = 0; k < D * D; k++) memcpy(F->K[k], knew[k], sizeof(double) * (size_t)P->ncell);
            polymeric_stage(P, F);
        }
        if (P->par.tempdiscrtype == HF_EXPLICIT_RK2 || P->par.tempdiscrtype == HF_EXPLICIT_RK3) rk_stage(P, F);
        else if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_BDF2) rc = bdf2_velocity(P, F, rtol);
        else
            for (int d = 0; d < D; d++) velocity_stage(P, F, d);
        if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_EULER || P->par.tempdiscrtype == HF_SEMI_IMPLICIT_CN)
            for (int d = 0; d < D && rc == 0; d++) rc = sie_solve(P, F, d, rtol);
        if (rc) break;
        rc = pressure_stage(P, F, rtol, iters);
        final_stage(P, F);
    }
    if (ve)
        for (int k = 0; k < D * D; k++) free(knew[k]);
    return rc;
}

/* individual stages, for stage-by-stage parity tests */
void hfr_velocity(const hf_program *P, hfr_fields *F)
{
    if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_BDF2) {
        bdf2_velocity(P, F, 1e-14);
        return;
    }
    for (int d = 0; d < P->par.dim; d++) velocity_stage(P, F, d);
    if (P->par.tempdiscrtype == HF_SEMI_IMPLICIT_EULER || P->par.tempdiscrtype == HF_SEMI_IMPLICIT_CN)
        for (int d = 0; d < P->par.dim; d++) sie_solve(P, F, d, 1e-14);
}

int hfr_pressure(const hf_program *P, hfr_fields *F, double rtol, int *iters)
{
    return pressure_stage(P, F, rtol, iters);
}

void hfr_final(const hf_program *P, hfr_fields *F) { final_stage(P, F); }

void hfr_ve_cell(const hf_program *P, hfr_fields *F)
{
    const int D = P->par.dim;
    double *knew[9] = {0};
    for (int k = 0; k < D * D; k++) knew[k] = malloc(sizeof(double) * (size_t)P->ncell);
    du_stage(P, F);
    constitutive_stage(P, F, knew);
    for (int k = 0; k < D * D; k++) {
        memcpy(F->K[k], knew[k], sizeof(double) * (size_t)P->ncell);
        free(knew[k]);
    }
    polymeric_stage(P, F);
}

/* divergence right-hand side only (for the Poisson-engine tests) */
void hfr_divergence_rhs(const hf_program *P, hfr_fields *F, double *bvec)
{
    const int D = P->par.dim, n = P->ncell;
    for (int cc = 0; cc < n; cc++) {
        const double *cd = P->delta + (size_t)P->cell_delta[cc] * D;
        double sumdudx = 0.0;
        for (int dim = 0; dim < D; dim++) {
            double ustarl = q(P, P->div_slots[(size_t)HF_P_UL(dim) * n + cc], F->us[dim]);
            double ustarr = q(P, P->div_slots[(size_t)HF_P_UR(dim) * n + cc], F->us[dim]);
            sumdudx += (ustarr - ustarl) / (2.0 * 0.5 * cd[dim]);
        }
        bvec[cc] = sumdudx / P->par.dt + P->p_brhs[cc];
    }
    if (P->pin_row >= 0)
        bvec[P->pin_row] = P->par.projtype == HF_INCREMENTAL ? P->pin_value - F->p[P->pin_row] : P->pin_value;
}

/* CFL number (higflow_compute_CFL, hig-flow-timestep.c:7-40): dt times the
 * largest over cells of sum_d |(u_l + u_r)/2| / (the face area normal to d),
 * u_l, u_r the face velocities from the divergence's own queries on u */
double hfr_cfl(const hf_program *P, hfr_fields *F)
{
    const int D = P->par.dim, n = P->ncell;
    double maxu_dx_norm = 0.0;
    for (int cc = 0; cc < n; cc++) {
        const double *cd = P->delta + (size_t)P->cell_delta[cc] * D;
        double u_dx_norm = 0.0;
        for (int dim = 0; dim < D; dim++) {
            const double ul = q(P, P->div_slots[(size_t)HF_P_UL(dim) * n + cc], F->u[dim]);
            const double ur = q(P, P->div_slots[(size_t)HF_P_UR(dim) * n + cc], F->u[dim]);
            const double u = (ul + ur) / 2.0;
            double facet_area = 1.0;
            for (int dim2 = 0; dim2 < D; dim2++)
                if (dim2 != dim) facet_area *= cd[dim2];
            u_dx_norm += fabs(u) / facet_area;
        }
        if (u_dx_norm > maxu_dx_norm) maxu_dx_norm = u_dx_norm;
    }
    return maxu_dx_norm * P->par.dt;
}

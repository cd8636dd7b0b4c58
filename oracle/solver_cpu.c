/*
 * CPU linear-solver engine for the oracle build (test infrastructure).
 *
 * PETSc 3.14 is not available here, so this file provides the engine that
 * higtree/src/solver.c:slv_create() selects by default (_slv_create_petsc) and
 * implements the _solver_vtable contract of higtree/src/solver.h:42-60:
 * rows are (re)set with set_Ai every step, b with set_bi/add_bi, the initial
 * guess is the previous solution (solver-petsc.c:386-399 uses a nonzero
 * initial guess), and solve() runs BiCGStab with an ILU(0) preconditioner
 * (the reference's command line is -ksp_type bcgs -pc_type bjacobi, i.e.
 * ILU(0) on the single block of one rank), stopping on the unpreconditioned
 * residual ||b - A x|| <= max(rtol*||b||, atol) as PETSc does.
 *
 * Tolerances: rtol = atol = 1e-10 (higflow/example2d_Newt/Makefile:76) unless
 * HF_ORACLE_RTOL is set; the parity tests set it tighter so the oracle's
 * fields carry no solver error at the 1e-10 comparison level.
 *
 * The engine also keeps the last assembled system so the harness can compare
 * it with the flattened Poisson rows.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "solver.h"

typedef struct cpu_solver {
    solver base;
    int first;
    int n;
    int *rlen;
    int **rcol;
    double **rval;
    double *b;
    double *x;
    /* assembled CSR (rows sorted by column) */
    int *ptr;
    int *col;
    double *val;
    int *diag;
    double *ilu;
    int csr_valid;
} cpu_solver;

/* last system solved and solve-time accounting, for the harness */
cpu_solver *hfref_last_pressure_solver = NULL;
double hfref_solve_seconds = 0.0;
int hfref_solve_iters = 0;

#include <time.h>
static double wall(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static cpu_solver *C(struct solver *s) { return (cpu_solver *)s; }

static void cs_set_maxnonzeros(struct solver *s) { (void)s; }

static void cs_set_Ai(struct solver *s, int i, int numjs, const int *j, const real *v)
{
    cpu_solver *c = C(s);
    int r = i - c->first;
    if (r < 0 || r >= c->n) { fprintf(stderr, "solver_cpu: row %d out of range\n", i); abort(); }
    free(c->rcol[r]);
    free(c->rval[r]);
    c->rcol[r] = malloc(sizeof(int) * (size_t)(numjs > 0 ? numjs : 1));
    c->rval[r] = malloc(sizeof(double) * (size_t)(numjs > 0 ? numjs : 1));
    /* duplicate columns in one call are summed (ADD semantics inside a row set) */
    int m = 0;
    for (int k = 0; k < numjs; k++) {
        int jj = j[k] - c->first;
        int found = -1;
        for (int q = 0; q < m; q++) if (c->rcol[r][q] == jj) { found = q; break; }
        if (found >= 0) c->rval[r][found] += v[k];
        else { c->rcol[r][m] = jj; c->rval[r][m] = v[k]; m++; }
    }
    c->rlen[r] = m;
    c->csr_valid = 0;
}

static void cs_set_bi(struct solver *s, int i, real v) { C(s)->b[i - C(s)->first] = v; }
static void cs_add_bi(struct solver *s, int i, real v) { C(s)->b[i - C(s)->first] += v; }
static void cs_set_xi(struct solver *s, int i, real v) { C(s)->x[i - C(s)->first] = v; }
static void cs_set_x(struct solver *s, const real *x) { memcpy(C(s)->x, x, sizeof(double) * (size_t)C(s)->n); }
static real cs_get_xi(struct solver *s, int i) { return C(s)->x[i - C(s)->first]; }
static void cs_get_x(struct solver *s, real *x) { memcpy(x, C(s)->x, sizeof(double) * (size_t)C(s)->n); }
static void cs_get_x_scatter(struct solver *s, int size, const int *idx, real *x)
{
    for (int k = 0; k < size; k++) x[k] = C(s)->x[idx[k] - C(s)->first];
}

static int cmp_pair(const void *a, const void *b)
{
    const int *x = a, *y = b;
    return (x[0] > y[0]) - (x[0] < y[0]);
}

static void build_csr(cpu_solver *c)
{
    if (c->csr_valid) return;
    free(c->ptr); free(c->col); free(c->val); free(c->diag); free(c->ilu);
    int n = c->n;
    c->ptr = malloc(sizeof(int) * (size_t)(n + 1));
    c->ptr[0] = 0;
    for (int r = 0; r < n; r++) c->ptr[r + 1] = c->ptr[r] + c->rlen[r];
    int nnz = c->ptr[n];
    c->col = malloc(sizeof(int) * (size_t)(nnz ? nnz : 1));
    c->val = malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
    c->diag = malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int r = 0; r < n; r++) {
        int m = c->rlen[r];
        int (*pairs)[2] = malloc(sizeof(int[2]) * (size_t)(m ? m : 1));
        for (int k = 0; k < m; k++) { pairs[k][0] = c->rcol[r][k]; pairs[k][1] = k; }
        qsort(pairs, (size_t)m, sizeof(int[2]), cmp_pair);
        c->diag[r] = -1;
        for (int k = 0; k < m; k++) {
            int p = c->ptr[r] + k;
            c->col[p] = pairs[k][0];
            c->val[p] = c->rval[r][pairs[k][1]];
            if (pairs[k][0] == r) c->diag[r] = p;
        }
        free(pairs);
    }
    /* ILU(0) factorisation, IKJ variant on the sparsity pattern of A */
    c->ilu = malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
    memcpy(c->ilu, c->val, sizeof(double) * (size_t)nnz);
    int *pos = malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int r = 0; r < n; r++) pos[r] = -1;
    for (int i = 0; i < n; i++) {
        for (int p = c->ptr[i]; p < c->ptr[i + 1]; p++) pos[c->col[p]] = p;
        for (int p = c->ptr[i]; p < c->ptr[i + 1] && c->col[p] < i; p++) {
            int k = c->col[p];
            double dk = c->diag[k] >= 0 ? c->ilu[c->diag[k]] : 0.0;
            if (dk == 0.0) continue;
            double lik = c->ilu[p] / dk;
            c->ilu[p] = lik;
            for (int q = c->diag[k] + 1; q < c->ptr[k + 1]; q++) {
                int jpos = pos[c->col[q]];
                if (jpos >= 0) c->ilu[jpos] -= lik * c->ilu[q];
            }
        }
        for (int p = c->ptr[i]; p < c->ptr[i + 1]; p++) pos[c->col[p]] = -1;
    }
    free(pos);
    c->csr_valid = 1;
}

static void spmv(const cpu_solver *c, const double *x, double *y)
{
    for (int r = 0; r < c->n; r++) {
        double s = 0.0;
        for (int p = c->ptr[r]; p < c->ptr[r + 1]; p++) s += c->val[p] * x[c->col[p]];
        y[r] = s;
    }
}

static void ilu_apply(const cpu_solver *c, const double *r, double *z)
{
    int n = c->n;
    for (int i = 0; i < n; i++) {
        double s = r[i];
        for (int p = c->ptr[i]; p < c->ptr[i + 1] && c->col[p] < i; p++) s -= c->ilu[p] * z[c->col[p]];
        z[i] = s;
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = z[i];
        int d = c->diag[i];
        for (int p = (d >= 0 ? d + 1 : c->ptr[i]); p < c->ptr[i + 1]; p++)
            if (c->col[p] > i) s -= c->ilu[p] * z[c->col[p]];
        z[i] = (d >= 0 && c->ilu[d] != 0.0) ? s / c->ilu[d] : s;
    }
}

static double dot(int n, const double *a, const double *b)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

static void cs_assemble_matrix(struct solver *s) { build_csr(C(s)); }
static void cs_assemble_rhs(struct solver *s) { (void)s; }
static void cs_assemble_output(struct solver *s) { (void)s; }

static void cs_solve(struct solver *s)
{
    cpu_solver *c = C(s);
    double t_start = wall();
    build_csr(c);
    hfref_last_pressure_solver = c;
    int n = c->n;
    double rtol = s->relative_tolerance, atol = s->absolute_tolerance;
    const char *env = getenv("HF_ORACLE_RTOL");
    if (env) { rtol = atof(env); atol = rtol * 1e-6; }
    double *r = malloc(sizeof(double) * (size_t)n * 8);
    double *rh = r + n, *p = rh + n, *v = p + n, *sv = v + n, *t = sv + n, *ph = t + n, *shat = ph + n;
    spmv(c, c->x, r);
    for (int i = 0; i < n; i++) r[i] = c->b[i] - r[i];
    double bn = sqrt(dot(n, c->b, c->b));
    double tol = fmax(rtol * bn, atol);
    double rn = sqrt(dot(n, r, r));
    int it = 0;
    int maxit = s->MaxIteration > 0 ? s->MaxIteration : 100000;
    if (maxit < 100000) maxit = 100000;
    memcpy(rh, r, sizeof(double) * (size_t)n);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    memset(v, 0, sizeof(double) * (size_t)n);
    memset(p, 0, sizeof(double) * (size_t)n);
    int restarts = 0;
    while (rn > tol && it < maxit) {
        double rho1 = dot(n, rh, r);
        if (rho1 == 0.0 || omega == 0.0) {
            /* breakdown: restart from the current iterate */
            if (++restarts > 50) break;
            spmv(c, c->x, r);
            for (int i = 0; i < n; i++) r[i] = c->b[i] - r[i];
            memcpy(rh, r, sizeof(double) * (size_t)n);
            rho = alpha = omega = 1.0;
            memset(v, 0, sizeof(double) * (size_t)n);
            memset(p, 0, sizeof(double) * (size_t)n);
            continue;
        }
        double beta = (rho1 / rho) * (alpha / omega);
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        ilu_apply(c, p, ph);
        spmv(c, ph, v);
        alpha = rho1 / dot(n, rh, v);
        for (int i = 0; i < n; i++) sv[i] = r[i] - alpha * v[i];
        ilu_apply(c, sv, shat);
        spmv(c, shat, t);
        double tt = dot(n, t, t);
        omega = tt > 0.0 ? dot(n, t, sv) / tt : 0.0;
        for (int i = 0; i < n; i++) {
            c->x[i] += alpha * ph[i] + omega * shat[i];
            r[i] = sv[i] - omega * t[i];
        }
        rho = rho1;
        rn = sqrt(dot(n, r, r));
        it++;
    }
    /* report the true residual */
    spmv(c, c->x, r);
    for (int i = 0; i < n; i++) r[i] = c->b[i] - r[i];
    rn = sqrt(dot(n, r, r));
    s->SolverIterations = it;
    s->SolverResidual = bn > 0 ? rn / bn : rn;
    s->converged = rn <= tol * 10.0;
    free(r);
    hfref_solve_iters = it;
    hfref_solve_seconds += wall() - t_start;
}

static void cs_destroy(struct solver *s)
{
    cpu_solver *c = C(s);
    if (hfref_last_pressure_solver == c) hfref_last_pressure_solver = NULL;
    for (int r = 0; r < c->n; r++) { free(c->rcol[r]); free(c->rval[r]); }
    free(c->rlen); free(c->rcol); free(c->rval); free(c->b); free(c->x);
    free(c->ptr); free(c->col); free(c->val); free(c->diag); free(c->ilu);
}

static const _solver_vtable cpu_vtable = {
    .set_maxnonzeros = cs_set_maxnonzeros,
    .set_Ai = cs_set_Ai,
    .set_bi = cs_set_bi,
    .add_bi = cs_add_bi,
    .set_xi = cs_set_xi,
    .set_x = cs_set_x,
    .get_xi = cs_get_xi,
    .get_x = cs_get_x,
    .get_x_scatter = cs_get_x_scatter,
    .assemble_matrix = cs_assemble_matrix,
    .assemble_rhs = cs_assemble_rhs,
    .assemble_output = cs_assemble_output,
    .solve = cs_solve,
    .destroy = cs_destroy,
};

solver *_slv_create_petsc(int first_gid, int size)
{
    cpu_solver *c = calloc(1, sizeof *c);
    c->base.vtable = &cpu_vtable;
    c->base.MaxIteration = 100000;
    c->base.relative_tolerance = 1e-10;
    c->base.absolute_tolerance = 1e-10;
    c->first = first_gid;
    c->n = size;
    c->rlen = calloc((size_t)(size ? size : 1), sizeof(int));
    c->rcol = calloc((size_t)(size ? size : 1), sizeof(int *));
    c->rval = calloc((size_t)(size ? size : 1), sizeof(double *));
    c->b = calloc((size_t)(size ? size : 1), sizeof(double));
    c->x = calloc((size_t)(size ? size : 1), sizeof(double));
    return &c->base;
}

static solver *unavailable(const char *name)
{
    fprintf(stderr, "oracle build: solver engine %s is not available\n", name);
    abort();
    return NULL;
}

solver *_slv_create_hollow_setup_petsc(int first_gid, int size) { (void)first_gid; (void)size; return unavailable("hollow"); }
solver *_slv_create_hypre(int ilower, int iupper) { (void)ilower; (void)iupper; return unavailable("hypre"); }
solver *_slv_create_debug_write(size_t start, size_t size) { (void)start; (void)size; return unavailable("debug-write"); }

/* harness access to the last assembled pressure system */
int hfref_last_system(int *n, int *nnz)
{
    cpu_solver *c = hfref_last_pressure_solver;
    if (!c) return -1;
    *n = c->n;
    *nnz = c->ptr[c->n];
    return 0;
}

int hfref_last_system_copy(int *ptr, int *col, double *val, double *b)
{
    cpu_solver *c = hfref_last_pressure_solver;
    if (!c) return -1;
    memcpy(ptr, c->ptr, sizeof(int) * (size_t)(c->n + 1));
    memcpy(col, c->col, sizeof(int) * (size_t)c->ptr[c->n]);
    memcpy(val, c->val, sizeof(double) * (size_t)c->ptr[c->n]);
    memcpy(b, c->b, sizeof(double) * (size_t)c->n);
    return 0;
}

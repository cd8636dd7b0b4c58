/*
 * The GPU solver engine as HigTree's solver plugin: the hf_slv_* entry points
 * of libhigflow_b200 (one per _solver_vtable slot, higtree/src/solver.h:42-60)
 * behind the engine constructor that slv_create selects by default
 * (_slv_create_petsc, higtree/src/solver.c:239-331), so every Poisson solve the
 * host's own HigFlow code makes runs on the B200.  The device side is created
 * on the first slot call that needs it: a host that only records step
 * programs never touches the GPU.
 */
#include <stdio.h>
#include <stdlib.h>

#include "solver.h"
#include "higflow_b200.h"

typedef struct solver_b200 {
    solver base;
    int first;
    int size;
    hf_slv *s;
} solver_b200;

static void die(const char *what)
{
    fprintf(stderr, "b200 solver engine: %s: %s\n", what, hf_last_error());
    exit(1);   /* the reference's convention on errors (utils.h:46-52) */
}

static hf_slv *S(solver *cs)
{
    solver_b200 *b = (solver_b200 *)cs;
    if (!b->s) {
        if (hf_slv_create(b->first, b->size, &b->s) != HF_OK) die("create");
        if (hf_slv_set_maxnonzeros(b->s, cs->MaxNonZeros) != HF_OK) die("set_maxnonzeros");
    }
    return b->s;
}

static void b_set_maxnonzeros(solver *cs)
{
    solver_b200 *b = (solver_b200 *)cs;
    if (b->s && hf_slv_set_maxnonzeros(b->s, cs->MaxNonZeros) != HF_OK) die("set_maxnonzeros");
}
static void b_set_Ai(solver *cs, int i, int n, const int *j, const real *v)
{
    if (hf_slv_set_Ai(S(cs), i, n, j, v) != HF_OK) die("set_Ai");
}
static void b_set_bi(solver *cs, int i, real v) { if (hf_slv_set_bi(S(cs), i, v) != HF_OK) die("set_bi"); }
static void b_add_bi(solver *cs, int i, real v) { if (hf_slv_add_bi(S(cs), i, v) != HF_OK) die("add_bi"); }
static void b_set_xi(solver *cs, int i, real v) { if (hf_slv_set_xi(S(cs), i, v) != HF_OK) die("set_xi"); }
static void b_set_x(solver *cs, const real *x) { if (hf_slv_set_x(S(cs), x) != HF_OK) die("set_x"); }
static real b_get_xi(solver *cs, int i)
{
    double v = 0.0;
    if (hf_slv_get_xi(S(cs), i, &v) != HF_OK) die("get_xi");
    return v;
}
static void b_get_x(solver *cs, real *x) { if (hf_slv_get_x(S(cs), x) != HF_OK) die("get_x"); }
static void b_get_x_scatter(solver *cs, int n, const int *idx, real *x)
{
    if (hf_slv_get_x_scatter(S(cs), n, idx, x) != HF_OK) die("get_x_scatter");
}
static void b_assemble_matrix(solver *cs) { if (hf_slv_assemble_matrix(S(cs)) != HF_OK) die("assemble_matrix"); }
static void b_assemble_rhs(solver *cs) { if (hf_slv_assemble_rhs(S(cs)) != HF_OK) die("assemble_rhs"); }
static void b_assemble_output(solver *cs) { if (hf_slv_assemble_output(S(cs)) != HF_OK) die("assemble_output"); }
static void b_solve(solver *cs)
{
    hf_slv *s = S(cs);
    if (hf_slv_set_tolerances(s, cs->relative_tolerance, cs->absolute_tolerance, cs->MaxIteration) != HF_OK)
        die("set_tolerances");
    const int rc = hf_slv_solve(s);
    int32_t it = 0, conv = 0;
    double res = 0.0;
    hf_slv_result(s, &it, &res, &conv);
    cs->SolverIterations = it;
    cs->SolverResidual = res;
    cs->converged = conv != 0;
    /* PETSc reports divergence through the converged flag and carries on */
    if (rc != HF_OK && rc != HF_ERR_NOT_CONVERGED) die("solve");
}
/* slv_destroy frees the solver struct itself after this (solver.c:228-237) */
static void b_destroy(solver *cs)
{
    solver_b200 *b = (solver_b200 *)cs;
    if (b->s) hf_slv_destroy(b->s);
    b->s = NULL;
}

static const _solver_vtable b200_vtable = {
    b_set_maxnonzeros, b_set_Ai, b_set_bi, b_add_bi, b_set_xi, b_set_x, b_get_xi, b_get_x, b_get_x_scatter,
    b_assemble_matrix, b_assemble_rhs, b_assemble_output, b_solve, b_destroy};

solver *_slv_create_petsc(int first_gid, int size)
{
    solver_b200 *b = calloc(1, sizeof *b);
    if (!b) die("out of host memory");
    b->base.vtable = &b200_vtable;
    /* HigFlow sets its own tolerances before solving (-ksp_rtol/-ksp_atol
     * 1e-10 in the shipped cases, higflow/example2d_Newt/Makefile:76) */
    b->base.MaxIteration = 100000;
    b->base.relative_tolerance = 1e-10;
    b->base.absolute_tolerance = 1e-10;
    b->first = first_gid;
    b->size = size;
    return &b->base;
}

static solver *unavailable(const char *name)
{
    fprintf(stderr, "b200 host build: solver engine %s is not available (the B200 engine replaces PETSc)\n", name);
    exit(1);
    return NULL;
}

solver *_slv_create_hollow_setup_petsc(int first_gid, int size) { (void)first_gid; (void)size; return unavailable("hollow"); }
solver *_slv_create_hypre(int ilower, int iupper) { (void)ilower; (void)iupper; return unavailable("hypre"); }
solver *_slv_create_debug_write(size_t start, size_t size) { (void)start; (void)size; return unavailable("debug-write"); }

/*
 * higflow_b200 — C ABI of the B200 (sm_100a) engine for HigFlow's per-time-step
 * hot path: explicit intermediate velocity, kernel-conformation constitutive
 * update, pressure-Poisson projection.
 *
 * Two layers are exposed, both with plain pointers and sizes only:
 *
 *  1. The step engine (hf_case_*): consumes a flattened "step program" — every
 *     stencil query one reference time step makes, recorded once from HigTree's
 *     own stencil builder — and runs whole time steps on the GPU with the fields
 *     resident in HBM.  It replaces, per step,
 *        higflow_solver_step               higflow/src/hig-flow-step.c:1363-1413
 *        higflow_solver_step_viscoelastic  higflow/src/hig-flow-step-viscoelastic.c:2091-2163
 *     for the configurations listed under hf_params.
 *
 *  2. The linear-solver engine (hf_slv_*): a GPU implementation of HigTree's
 *     solver plugin, one entry point per slot of _solver_vtable
 *     (higtree/src/solver.h:42-60), for callers that keep assembling the
 *     Poisson system on the host (solver.c:38-202 call sites).
 *
 * Every function returns an int status: 0 on success, a negative HF_ERR_* code
 * otherwise (the reference has no status returns; it exits, utils.h:46-52).
 * No entry point falls back to the CPU: without a usable CUDA device the
 * create calls return HF_ERR_NO_DEVICE.
 */
#ifndef HIGFLOW_B200_H
#define HIGFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes                                                        */
/* ------------------------------------------------------------------ */
#define HF_OK                  0
#define HF_ERR_INVALID        -1  /* malformed program / argument            */
#define HF_ERR_UNSUPPORTED    -2  /* configuration outside the GPU path       */
#define HF_ERR_NOT_CONVERGED  -3  /* Poisson solve hit its iteration limit    */
#define HF_ERR_NAN            -4  /* NaN/Inf detected in a field or residual  */
#define HF_ERR_OOM_BUDGET     -5  /* request exceeds the HBM budget           */
#define HF_ERR_CUDA           -6  /* CUDA runtime error                       */
#define HF_ERR_NO_DEVICE      -7  /* no CUDA device / extension unusable      */
#define HF_ERR_TIMEOUT        -8  /* a bounded device-side wait gave up       */

/* ------------------------------------------------------------------ */
/* enumerations mirroring the reference's controllers                 */
/* (higflow/src/hig-flow-kernel.h:27-31, 152-193, 295-313)             */
/* ------------------------------------------------------------------ */
enum { HF_NEWTONIAN = 0, HF_VISCOELASTIC = 3 };                 /* flow_type      */
enum { HF_NON_INCREMENTAL = 0, HF_INCREMENTAL = 1 };            /* projection     */
enum { HF_CENTRAL = 0, HF_FIRST_ORDER = 1, HF_SECOND_ORDER = 2 };/* convecdiscr   */
enum { HF_MCU = 0, HF_CUBISTA = 1, HF_QUICK = 2 };              /* second order   */
enum { HF_OLDROYD_B = 0, HF_GIESEKUS = 1, HF_LPTT = 2,           /* VE model       */
       HF_GPTT = 3, HF_FENE_P = 4, HF_E_FENE = 5 };
enum { HF_CELL_CENTRAL = 0, HF_CELL_CUBISTA = 1 };              /* VE convection  */
/* constitutive step (hig-flow-kernel.h:305-308): explicit Euler, or the
 * implicit form that solves (I - dt (Omega x I - I x Omega)) K = K + dt (-conv
 * + 2B + M/De) per cell (hig-flow-step-viscoelastic.c:720-926) */
enum { HF_VE_EXPLICIT = 0, HF_VE_IMPLICIT = 1 };
enum { HF_KERNEL_IDENTITY = 0, HF_KERNEL_LOG = 1, HF_KERNEL_SQRT = 2 };
/* intermediate velocity (hig-flow-kernel.h:169-176): explicit Euler; the
 * explicit Runge-Kutta forms chain Euler stages E (RK2: u* = (u + E(E(u)))/2;
 * RK3: v = E(u), w = 3u/4 + E(v)/4, u* = u/3 + 2 E(w)/3; hig-flow-step.c:
 * 666-784); the semi-implicit form solves (I - dt/Re Lap_h) u* = u + dt
 * (sources - grad p - conv [+ div S]) per direction (hig-flow-step.c:788-883,
 * hig-flow-step-viscoelastic.c:1108-1210) */
enum { HF_EXPLICIT_EULER = 0, HF_EXPLICIT_RK2 = 1, HF_EXPLICIT_RK3 = 2, HF_SEMI_IMPLICIT_EULER = 3,
       HF_SEMI_IMPLICIT_CN = 4,     /* Crank-Nicolson: weights -dt/(2 Re delta^2), half the diffusion explicit */
       HF_SEMI_IMPLICIT_BDF2 = 5 }; /* two solves: weights -dt/(4 Re delta^2), then -dt/(3 Re delta^2) */

/* precision forms */
enum {
    HF_PREC_FP64 = 0,   /* plain: every gather, update and Poisson iterate in FP64 */
    HF_PREC_MIXED = 1   /* velocity-stage stencil rows with FP32 weights
                           (FP64 field values and sums), FP32 CUBISTA
                           convection; the Poisson solve as FP32 AMG-CG
                           sweeps (operator, vectors, V-cycle in FP32) inside
                           FP64 iterative refinement: after each sweep the
                           FP64 unknown takes the correction and the FP64
                           residual is updated with the FP64 operator, to the
                           plain form's residual test; eigensystem, kernel
                           transform and the velocity/pressure/conformation
                           time updates stay FP64 */
};

/* Poisson preconditioner (CG path) */
enum {
    HF_PRECOND_AUTO = 0,    /* smoothed-aggregation AMG V-cycle                 */
    HF_PRECOND_JACOBI = 1,  /* diagonal scaling                                  */
    HF_PRECOND_AMG = 2
};

/* Poisson solver choice */
enum {
    HF_POISSON_AUTO = 0,    /* CG when the reduced matrix is symmetric, else BiCGStab */
    HF_POISSON_CG = 1,
    HF_POISSON_BICGSTAB = 2
};

/* ------------------------------------------------------------------ */
/* step-program slot layouts                                           */
/*                                                                     */
/* A slot holds one recorded stencil query as an int32 code:           */
/*   code >= 0 : the query is a centre hit with weight 1 and no        */
/*               boundary term; its value is field[code]               */
/*   code <  0 : general query r = -code-1; its value is               */
/*               -rhs[r] + sum_k w[k]*field[base[r] + col[k]] over the */
/*               entries k of template tmpl[r], accumulated in that    */
/*               order (pdomain.c:1026-1053).  A recorded program has  */
/*               one template per row and base 0; rows that are        */
/*               translates of each other on a uniform grid share one  */
/*               template and differ only in base.                     */
/* Which field a slot reads is fixed by its position (listed below).   */
/* Slot arrays are slot-major: slots[s * nelem + e].                   */
/* ------------------------------------------------------------------ */

/* Velocity stage, one element per facet normal to d
 * (higflow_computational_cell, higflow/src/hig-flow-discret.c:86-259;
 *  higflow_computational_cell_viscoelastic, :541-569). */
#define HF_V_FU   0   /* facet source FU[d] at the facet centre (sfdF[d])         */
#define HF_V_PL   1   /* p at centre - 0.5*delta_d (sdp); reused for dp in the    */
#define HF_V_PR   2   /*   final velocity (hig-flow-step.c:242-308)               */
#define HF_V_FL   3   /* cell source F at centre -/+ 0.5*delta_d (sdF)           */
#define HF_V_FR   4
#define HF_V_BLK0 5   /* first per-direction block                                */
#define HF_V_NB   10  /* slots per direction d2:                                  */
#define HF_V_V4   0   /*   +0..3 u[d2] at (+,+),(+,-),(-,+),(-,-) half-deltas in  */
                      /*         (d, d2)  (compute_facet_u_2, hig-flow-eval.c:65) */
#define HF_V_UL   4   /*   +4 u[d] at centre - 1*delta_d2                         */
#define HF_V_UR   5   /*   +5 u[d] at centre + 1*delta_d2                         */
#define HF_V_ULL  6   /*   +6 u[d] at centre - 2*delta_d2                         */
#define HF_V_URR  7   /*   +7 u[d] at centre + 2*delta_d2                         */
#define HF_V_VCR  8   /*   +8 u[d2] at centre + 0.5*delta_d2 (CUBISTA v1bar)      */
#define HF_V_VCL  9   /*   +9 u[d2] at centre - 0.5*delta_d2 (CUBISTA v2bar)      */
#define HF_V_NSLOT_NEWT(D) (HF_V_BLK0 + HF_V_NB * (D))
/* viscoelastic extension, per direction d2, on S[d][d2] (sdED):
 *   +0 SL_A  +1 SL_B  +2 SR_A  +3 SR_B
 *   d2 == d : SL_A = centre - 0.5*delta_d, SR_A = centre + 0.5*delta_d
 *   d2 != d : compute_center_p_left_2 / _right_2 (hig-flow-eval.c:454-487):
 *             SL_A/SL_B at d2 - delta_d2 with d -/+ 0.5*delta_d,
 *             SR_A/SR_B at d2 + delta_d2 with d -/+ 0.5*delta_d            */
#define HF_V_NS   4
#define HF_V_NSLOT_VE(D) (HF_V_NSLOT_NEWT(D) + HF_V_NS * (D))
/* velocity-stage flag bits: for direction d2, bit 4*d2+k is the infacet
 * flag of UL, UR, ULL, URR (k = 0..3) (sfd_get_facet_with_point)          */

/* Divergence stage, one element per cell: u*[d] at centre -/+ 0.5*delta_d
 * (higflow_pressure, hig-flow-step.c:58-80). */
#define HF_P_UL(d) (2 * (d))
#define HF_P_UR(d) (2 * (d) + 1)
#define HF_P_NSLOT(D) (2 * (D))

/* Viscoelastic cell stage, one element per cell
 * (higflow_compute_velocity_derivative_tensor, hig-flow-step-generalized-
 *  newtonian.c:14-97; higflow_explicit_euler_constitutive_equation,
 *  hig-flow-step-viscoelastic.c:352-544; higflow_compute_polymeric_tensor,
 *  :212-347; hig_flow_convective_cell_term_cubista, hig-flow-step.c:1185). */
#define HF_C_SELF 0   /* Du, S, Kernel at the cell centre (sdED)                  */
#define HF_C_BLK0 1
#define HF_C_NB   6   /* per direction d:                                         */
#define HF_C_UVL  0   /*   +0 u[d] at centre - 0.5*delta_d                        */
#define HF_C_UVR  1   /*   +1 u[d] at centre + 0.5*delta_d                        */
#define HF_C_KL   2   /*   +2 Kernel at centre - delta_d   (sdED)                 */
#define HF_C_KR   3   /*   +3 Kernel at centre + delta_d                          */
#define HF_C_KLL  4   /*   +4 Kernel at centre - 2*delta_d                        */
#define HF_C_KRR  5   /*   +5 Kernel at centre + 2*delta_d                        */
/* then, for each ordered pair (d, d2), d2 != d, in row-major order, 4 slots on
 * u[d] for the corner values of compute_facet_u_4_left/_right
 * (hig-flow-eval.c:95-195):
 *   +0 (d + 0.5, d2 - 1)  +1 (d - 0.5, d2 - 1)  +2 (d + 0.5, d2 + 1)  +3 (d - 0.5, d2 + 1)
 * (in units of delta); the (d -/+ 0.5, d2) values are UVL/UVR.              */
#define HF_C_NQ   4
#define HF_C_NSLOT(D) (HF_C_BLK0 + HF_C_NB * (D) + HF_C_NQ * (D) * ((D) - 1))
/* cell-stage flag bits: for direction d, bit 4*d+k is the incell flag of
 * KL, KR, KLL, KRR (k = 0..3) (sd_get_cell_with_point != NULL)             */

/* field identifiers for hf_case_set_field / hf_case_get_field */
enum {
    HF_FIELD_U = 0,       /* comp = d: facet velocity u[d]                   */
    HF_FIELD_USTAR = 1,   /* comp = d: intermediate velocity u*[d]           */
    HF_FIELD_P = 2,       /* cell pressure                                   */
    HF_FIELD_DP = 3,      /* cell pressure increment (incremental projection)*/
    HF_FIELD_F = 4,       /* cell source term                                */
    HF_FIELD_FU = 5,      /* comp = d: facet source term                     */
    HF_FIELD_KERNEL = 6,  /* comp = i*D+j: kernel tensor                      */
    HF_FIELD_S = 7,       /* comp = i*D+j: polymeric tensor                  */
    HF_FIELD_DU = 8       /* comp = i*D+j: velocity-gradient tensor          */
};

/* physical and numerical parameters (hig-flow-kernel.h:108-214, 425-457) */
typedef struct hf_params {
    int32_t dim;                  /* 2 or 3                                  */
    int32_t flowtype;             /* HF_NEWTONIAN / HF_VISCOELASTIC          */
    int32_t projtype;             /* HF_INCREMENTAL / HF_NON_INCREMENTAL     */
    int32_t convecdiscrtype;      /* HF_CENTRAL / HF_FIRST_ORDER / HF_SECOND_ORDER */
    int32_t secondconvecdiscrtype;/* HF_MCU / HF_CUBISTA / HF_QUICK          */
    int32_t ve_model;             /* HF_OLDROYD_B / HF_GIESEKUS / HF_LPTT    */
    int32_t ve_convecdiscrtype;   /* HF_CELL_CENTRAL / HF_CELL_CUBISTA       */
    int32_t kernel;               /* HF_KERNEL_*                             */
    double Re, dt;
    double De, beta, kernel_tol, alpha, epsilon, xi;
    int32_t tempdiscrtype;        /* HF_EXPLICIT_EULER / _RK2 / _RK3 / HF_SEMI_IMPLICIT_EULER / _CN / _BDF2 */
    int32_t pad_;
    double L2_fene, lambda_fene, E_fene;   /* e-FENE (ve_parameters, hig-flow-kernel.h:443-445) */
    int32_t ve_discrtype;         /* HF_VE_EXPLICIT / HF_VE_IMPLICIT (constitutive step) */
    int32_t pad2_;
    /* GPTT (ve_parameters, hig-flow-kernel.h:439-441): the Mittag-Leffler
     * E_{alpha,beta} parameters and gamma = Gamma(beta_gptt), which the
     * reference recomputes with tgamma every constitutive step
     * (hig-flow-step-viscoelastic.c:359-362) */
    double alpha_gptt, beta_gptt, gamma_gptt;
} hf_params;

/* A flattened step program (host memory, read-only for the engine). */
typedef struct hf_program {
    hf_params par;
    int32_t ncell;                 /* leaf cells (pressure unknowns)           */
    int32_t nfacet[3];             /* interior facets normal to each direction */

    /* distinct cell/facet deltas; elements store an index into these tables */
    int32_t ndelta;
    const double *delta;           /* ndelta * dim                             */

    /* general stencil rows: template, base offset and boundary term per row */
    int64_t nrows;
    const int32_t *row_tmpl;       /* nrows: template index                    */
    const int32_t *row_base;       /* nrows: added to every template column    */
    const double  *row_rhs;        /* nrows                                    */
    /* stencil templates (CSR of ids and weights), deduplicated by content */
    int64_t ntmpl;
    int64_t nnz;
    const int64_t *tmpl_ptr;       /* ntmpl + 1 */
    const int32_t *tmpl_col;       /* nnz       */
    const double  *tmpl_w;         /* nnz       */

    /* velocity stage per direction d < dim */
    int32_t vel_nslot;             /* HF_V_NSLOT_NEWT or HF_V_NSLOT_VE         */
    const int32_t  *vel_slots[3];  /* vel_nslot * nfacet[d], slot-major        */
    const uint32_t *vel_flags[3];  /* nfacet[d]                                */
    const uint16_t *vel_delta[3];  /* nfacet[d]: index into delta              */

    /* divergence stage */
    const int32_t  *div_slots;     /* HF_P_NSLOT * ncell                       */
    const uint16_t *cell_delta;    /* ncell: index into delta                  */

    /* Poisson matrix (global ids == cell ids on one rank), constant per mesh */
    int64_t pnnz;
    const int64_t *p_ptr;          /* ncell + 1 */
    const int32_t *p_col;          /* pnnz      */
    const double  *p_val;          /* pnnz      */
    const double  *p_brhs;         /* ncell: boundary part of each row's rhs   */
    int32_t pin_row;               /* desingularised row, -1 if none           */
    double  pin_value;             /* get_pressure at the pinned cell centre   */

    /* viscoelastic cell stage (flowtype == HF_VISCOELASTIC) */
    int32_t cell_nslot;            /* HF_C_NSLOT(dim) or 0                     */
    const int32_t  *cell_slots;    /* cell_nslot * ncell                       */
    const uint32_t *cell_flags;    /* ncell                                    */

    /* Batches.  ninst > 0 concatenates ninst independent cases of the same
     * dim and flow type: instance i owns cells [cell_off[i], cell_off[i+1])
     * and facets [facet_off[d][i], facet_off[d][i+1]); every slot code, row
     * base and Poisson column is already a global index; each instance has its
     * own parameters and pressure pin.  ninst == 0 is one case described by
     * par, pin_row and pin_value. */
    int32_t ninst;
    const hf_params *inst_par;     /* ninst                                    */
    const int32_t *cell_off;       /* ninst + 1                                */
    const int32_t *facet_off[3];   /* ninst + 1 per direction                  */
    const int32_t *inst_pin;       /* ninst: pinned cell (global id) or -1     */
    const double  *inst_pin_value; /* ninst                                    */
} hf_program;

/* ------------------------------------------------------------------ */
/* step engine                                                         */
/* ------------------------------------------------------------------ */
typedef struct hf_case hf_case;

typedef struct hf_options {
    int32_t precision;        /* HF_PREC_FP64 / HF_PREC_MIXED                 */
    int32_t poisson;          /* HF_POISSON_*                                 */
    double  poisson_rtol;     /* relative residual target (reference: 1e-10)  */
    double  poisson_atol;     /* absolute residual target (reference: 1e-10)  */
    int32_t poisson_maxit;    /* iteration cap; 0 = 20000                      */
    int32_t device;           /* CUDA device ordinal                          */
    int32_t precond;          /* HF_PRECOND_*                                 */
    int32_t eager;            /* 0: each step is one CUDA graph launch; 1:    */
                              /* kernels launched one by one with a host loop */
                              /* over the iterations (kernel profilers)       */
    int32_t tuning;           /* 0: before the first step, time the velocity- */
                              /* and cell-stage kernels at a few block sizes  */
                              /* on this case and keep the fastest (results   */
                              /* do not depend on it); 1: built-in sizes      */
} hf_options;

typedef struct hf_stats {
    int64_t steps;            /* steps taken since create                      */
    int32_t last_iters;       /* Poisson iterations of the last step (inner)   */
    int32_t last_outer;       /* refinement sweeps of the last step (mixed:    */
                              /* the most of any instance; plain: 1)           */
    double  last_residual;    /* relative true residual of the last solve      */
    int64_t total_iters;      /* all Poisson iterations since create           */
    int64_t kernel_launches;  /* kernels launched by hf_case_step so far       */
    double  device_bytes;     /* HBM held by this case                         */
} hf_stats;

/* Replaces higflow_solver_step / _viscoelastic for one case.
 * hf_case_create copies the program to the device; the program memory can be
 * freed afterwards.  Fields start at zero; set them with hf_case_set_field. */
int  hf_case_create(const hf_program *prog, const hf_options *opt, hf_case **out);
int  hf_case_set_field(hf_case *c, int32_t field, int32_t comp, const double *host, int64_t n);
int  hf_case_get_field(hf_case *c, int32_t field, int32_t comp, double *host, int64_t n);
/* Advance nsteps time steps (each one the full reference sub-step order) and
 * wait for them; returns the first failed Poisson solve among them.  With the
 * CG solver each step is one CUDA graph launch on the case stream (the first
 * call captures the graphs). */
int  hf_case_step(hf_case *c, int32_t nsteps);
/* The same without waiting: the steps are queued on the case stream and a
 * failure is reported by the next hf_case_synchronize (or hf_case_step). */
int  hf_case_step_async(hf_case *c, int32_t nsteps);
int  hf_case_stats(hf_case *c, hf_stats *out);
int  hf_case_synchronize(hf_case *c);
void hf_case_destroy(hf_case *c);

/* Poisson solver of a case: method (HF_PRECOND_AMG / HF_PRECOND_JACOBI for CG,
 * -1 for BiCGStab), number of levels and, per level up to max_levels, rows and
 * non-zeros of A, P and R summed over the instances.  With AMG the levels are
 * the concatenated multigrid levels followed by one entry for the dense
 * coarsest solves of all instances (rows = sum cn, nnz_a = sum cn^2). */
int  hf_case_solver_info(hf_case *c, int32_t *method, int32_t *nlev, int64_t *rows, int64_t *nnz_a,
                         int64_t *nnz_p, int64_t *nnz_r, int32_t max_levels);

/* The block sizes the case launches its tuned kernels with (see
 * hf_options.tuning): blocks[0] velocity-stage rows (k_vrows), [1] facet
 * kernel (k_velocity), [2] cell stage (k_ve_cell); n >= 3. */
int  hf_case_launch_shapes(hf_case *c, int32_t *blocks, int32_t n);

/* Kernels per step outside the Poisson iterations, and per loop body of the
 * iterations (one body = two CG iterations). */
int  hf_case_launch_counts(hf_case *c, int32_t *per_step, int32_t *per_body);

/* Batches: number of instances, and the last step's Poisson result of one
 * instance (iterations, all sweeps together; refinement sweeps (mixed form;
 * 1 for the plain form); status; relative residual ||r|| / ||b||). */
int  hf_case_instances(hf_case *c, int32_t *ninst);
int  hf_case_instance_result(hf_case *c, int32_t inst, int32_t *iters, int32_t *outer, int32_t *status,
                             double *residual);

/* Poisson iterations of every instance summed over all steps so far (n = ninst). */
int  hf_case_instance_iters(hf_case *c, int64_t *total_iters, int32_t n);

/* Adaptive time step (higflow_adjust_timestep, higflow/src/hig-flow-timestep.c:
 * 115-139), each instance on its own CFL number: CFL = dt * max over cells of
 * sum_d |(u_l + u_r)/2| / (face area normal to d); dt <- min(min(0.1/(CFL +
 * 1e-12), 1.1) dt, 32 dt0), dt0 = the instance's dt at create.  Writes each
 * instance's CFL and new dt (n = ninst; either array may be null); the next
 * steps use the new dt.  HF_ERR_UNSUPPORTED for the semi-implicit velocity,
 * whose system matrix holds dt. */
int  hf_case_adjust_timestep(hf_case *c, double *cfl, double *dt, int32_t n);

/* Set each instance's time step (n = ninst) for the next steps, as a case main
 * loop does when it changes ns->par.dt (higflow_adjust_timestep,
 * hig-flow-timestep.c:115-139, or a restart); the instances' parameters go to
 * the device on every call (it waits for the case's stream).
 * HF_ERR_UNSUPPORTED for the semi-implicit velocity when dt changes (its
 * system matrix holds dt; an unchanged dt is accepted and not copied). */
int  hf_case_set_timestep(hf_case *c, const double *dt, int32_t n);

/* Per-instance step limits (no counterpart in the reference, which runs one
 * case per job): instance i takes steps[i] more steps and is then frozen (no
 * kernel changes its fields) while the others go on; steps[i] < 0: no limit.
 * n = ninst.  Each frozen instance's fields stay those of its last step, so
 * its result is the same as when it runs alone for steps[i] steps.  Needs the
 * CG Poisson path and an explicit velocity scheme (HF_ERR_UNSUPPORTED
 * otherwise).  Once limits are set, an instance whose step fails (a NaN, a
 * Poisson solve that does not converge) is frozen after that step and the
 * others go on; the step call still returns the first failure. */
int  hf_case_set_step_limits(hf_case *c, const int64_t *steps, int32_t n);

/* Under step limits: each instance's first failed step's status (0: none so
 * far; HF_ERR_NAN, HF_ERR_NOT_CONVERGED), n = ninst.  Waits for the case's
 * stream. */
int  hf_case_instance_failures(hf_case *c, int32_t *status, int32_t n);

/* The CUDA stream every kernel of this case runs on (a cudaStream_t). */
int  hf_case_stream(hf_case *c, void **stream);

/* Per-phase device time: with profiling on, each phase of hf_case_step is
 * bracketed by CUDA events on the case stream; times accumulate (ms) with the
 * number of kernel launches per phase until the next hf_case_profile call. */
enum {
    HF_PHASE_VE_CELL = 0,       /* viscoelastic cell stage                 */
    HF_PHASE_VELOCITY = 1,      /* intermediate velocity                   */
    HF_PHASE_POISSON_INIT = 2,  /* divergence rhs + first residual         */
    HF_PHASE_POISSON_ITER = 3,  /* Krylov iterations                       */
    HF_PHASE_FINAL = 4,         /* final velocity and pressure             */
    HF_PHASE_VELOCITY_ROWS = 5, /* within HF_PHASE_VELOCITY: its stencil   */
                                /* rows (k_vrows) alone; CG path only      */
    HF_PHASE_VE_CELL_MAIN = 6,  /* within HF_PHASE_VE_CELL: its main       */
                                /* kernel (k_ve_cell) alone; CG path only  */
    HF_NPHASE = 7
};
int  hf_case_profile(hf_case *c, int32_t enable);
int  hf_case_phase_times(hf_case *c, double *ms, int64_t *launches, int32_t n);

/* Device memory the engine would hold for a program (admission control). */
int  hf_case_device_bytes(const hf_program *prog, const hf_options *opt, int64_t *bytes);

/* Last error message of the calling thread (static storage). */
const char *hf_last_error(void);

/* ------------------------------------------------------------------ */
/* serving: independent cases stepping concurrently on one device,    */
/* one engine case per request (no counterpart in the reference, which */
/* runs one case per job).  For requests that can share a batch, the   */
/* continuous-batching server (higflow_b200/serve.py) groups them into */
/* batch cases with per-instance step limits instead; this server is   */
/* for requests that cannot batch (the semi-implicit velocity forms).  */
/* ------------------------------------------------------------------ */
typedef struct hf_server hf_server;

typedef struct hf_server_options {
    double  hbm_budget_gb;    /* device memory the admitted cases may hold; 0 = 150 */
    int32_t max_active;       /* cases being created or stepped at once; 0 = 64     */
    int32_t chunk_steps;      /* steps queued per case per dispatch; 0 = 16         */
    int32_t setup_threads;    /* host threads creating admitted cases; 0 = 8        */
    int32_t device;           /* CUDA device ordinal                               */
} hf_server_options;

typedef struct hf_field_data {
    int32_t field, comp;      /* HF_FIELD_*, component                           */
    const double *data;       /* host values, copied at submit                   */
    int64_t n;
} hf_field_data;

typedef struct hf_server_counts {
    int64_t submitted, completed, failed, queued, active;
    int64_t reserved_bytes;   /* device memory held or reserved by admitted cases */
    int64_t cell_steps;       /* cells x steps of the completed requests          */
    double  seconds;          /* since hf_server_create                           */
} hf_server_counts;

/* Requests are admitted in arrival order while their device memory fits the
 * budget, created on host threads, then stepped on their own CUDA streams
 * (chunk_steps graph launches at a time) until done; fields stay on the device
 * until hf_server_release.  Each request is an engine case of its own, so its
 * result is the same alone and in any mix. */
int  hf_server_create(const hf_server_options *opt, hf_server **out);
/* Queue a case (program, options, initial fields, steps); copies everything. */
int  hf_server_submit(hf_server *s, const hf_program *prog, const hf_options *opt, int32_t nsteps,
                      const hf_field_data *fields, int32_t nfields, int64_t *id);
/* Wait for a request (timeout_ms < 0: until done); HF_ERR_TIMEOUT if still
 * running.  status: the request's own result; queue_s: submit to admission;
 * total_s: submit to completion (time to solution). */
int  hf_server_wait(hf_server *s, int64_t id, int32_t timeout_ms, int32_t *status, double *queue_s,
                    double *total_s);
int  hf_server_get_field(hf_server *s, int64_t id, int32_t field, int32_t comp, double *host, int64_t n);
int  hf_server_release(hf_server *s, int64_t id);
int  hf_server_stats(hf_server *s, hf_server_counts *out);
/* Drops requests not yet admitted, waits for the admitted ones, frees all. */
void hf_server_destroy(hf_server *s);
const char *hf_server_last_error(void);

/* ------------------------------------------------------------------ */
/* linear-solver engine: one entry point per _solver_vtable slot       */
/* (higtree/src/solver.h:42-87).  Row/column indices are global ids in */
/* [first_gid, first_gid + size).                                      */
/* ------------------------------------------------------------------ */
typedef struct hf_slv hf_slv;

int  hf_slv_create(int32_t first_gid, int32_t size, hf_slv **out);             /* _slv_create_petsc */
int  hf_slv_set_maxnonzeros(hf_slv *s, int32_t maxnz);                         /* set_maxnonzeros   */
int  hf_slv_set_Ai(hf_slv *s, int32_t i, int32_t numjs, const int32_t *j, const double *v); /* set_Ai */
int  hf_slv_set_bi(hf_slv *s, int32_t i, double v);                            /* set_bi            */
int  hf_slv_add_bi(hf_slv *s, int32_t i, double v);                            /* add_bi            */
int  hf_slv_set_xi(hf_slv *s, int32_t i, double v);                            /* set_xi            */
int  hf_slv_set_x(hf_slv *s, const double *x);                                 /* set_x             */
int  hf_slv_get_xi(hf_slv *s, int32_t i, double *v);                           /* get_xi            */
int  hf_slv_get_x(hf_slv *s, double *x);                                       /* get_x             */
int  hf_slv_get_x_scatter(hf_slv *s, int32_t size, const int32_t *idx, double *x); /* get_x_scatter */
int  hf_slv_assemble_matrix(hf_slv *s);                                        /* assemble_matrix   */
int  hf_slv_assemble_rhs(hf_slv *s);                                           /* assemble_rhs      */
int  hf_slv_assemble_output(hf_slv *s);                                        /* assemble_output   */
int  hf_slv_set_tolerances(hf_slv *s, double rtol, double atol, int32_t maxit);
int  hf_slv_solve(hf_slv *s);                                                  /* solve             */
int  hf_slv_result(hf_slv *s, int32_t *iterations, double *residual, int32_t *converged);
void hf_slv_destroy(hf_slv *s);                                                /* destroy           */

/* No counterpart in the reference.  The hf_slv_solve iteration (Jacobi-
 * preconditioned BiCGStab from the given x until ||b - A x|| <= max(rtol ||b||,
 * atol)) on an n-row CSR system whose arrays (ptr: n+1, col/val: ptr[n], b, x:
 * n) already live in device memory of the current device, queued on `stream`
 * and waited for.  It allocates nothing: every work vector sits in one static
 * device buffer of 65536 rows (about 4.7 MB), for callers that cannot allocate
 * once running (an HBM budget fixed at start-up, or solves on one stream while
 * other streams of the device are busy, which cudaMalloc/cudaFree would stall).
 * Larger systems are rejected with HF_ERR_INVALID.  The buffer's device address
 * is looked up (cudaGetSymbolAddress, which may load the module) by the first
 * call on each device and kept; that first call should come before any stream
 * capture.  A call that fails with a CUDA error waits for its queued kernels
 * when the stream still answers and drops the kept address; a device reset
 * (cudaDeviceReset) between calls is not supported.  Each call clears the
 * buffer's scalars before it starts.  Calls that overlap (other threads or
 * streams on the same device) share the buffer and race: serialise them. */
int  hf_slv_solve_device_noalloc(int32_t n, const int32_t *ptr, const int32_t *col, const double *val,
                                 const double *b, double *x, double rtol, double atol, int32_t maxit,
                                 void *stream, int32_t *iterations, double *residual);

/* The Mittag-Leffler function E_{alpha,beta}(z) that the GPTT model's M term
 * takes (replaces mlfv, hig-flow-mittag-leffler.h:22 / .c:117), evaluated on
 * the current device at n points: z and out are host arrays of 2n doubles,
 * real and imaginary parts interleaved.  fi: accuracy digits, 1..8 (the model
 * passes 6).  0 < alpha <= 5, beta <= 5 (the range the reference's evaluation
 * accepts); otherwise HF_ERR_INVALID.  Real parts follow the reference; the
 * imaginary part of the asymptotic form's leading term is the true one (the
 * reference's has the wrong sign there). */
int  hf_mittag_leffler(double alpha, double beta, const double *z, int64_t n, int32_t fi, double *out);

#ifdef __cplusplus
}
#endif

#endif

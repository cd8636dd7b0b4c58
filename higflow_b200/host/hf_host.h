/*
 * HigFlow host of the drop-in: builds a HigFlow case the way a case main
 * program does (higflow/example2d_Newt/ns-example-2d.c:159-230) and records
 * its step program with the binding's flattener (hf_flatten), so that the
 * stencils the GPU engine runs are HigTree's own, bit for bit.
 *
 * Compiled against the case's HigFlow headers with the same -DDIM as the
 * case.  In this image it is linked with the reference HigTree/HigFlow
 * sources compiled in place (higflow_b200/host/Makefile) into
 * higflow_b200/lib/libhigflow_host{2,3}d.so.
 *
 * A case is described by legacy text inputs (<name>.domain, <name>.bc, read by
 * higflow_initialize_domain, hig-flow-ic.c:11, and
 * higflow_initialize_boundaries, hig-flow-bc.c:572) and by hfh_params, whose
 * boundary and initial values feed the callbacks a case file would define.
 */
#ifndef HF_HOST_H
#define HF_HOST_H

#include <stdint.h>

#include "higflow_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define HFH_MAXBC 16

/* Case description: controllers and parameters of higflow_solver
 * (hig-flow-kernel.h:108-214, 425-457) plus the callback data. */
typedef struct hfh_params {
    int32_t flowtype, projtype, convecdiscrtype, secondconvecdiscrtype;
    int32_t ve_model, ve_convecdiscrtype, kernel;  /* kernel: HF_KERNEL_* */
    int32_t nbc;
    double Re, dt, t0;
    double De, beta, kernel_tol, alpha, epsilon, xi;
    /* boundary velocity for bc id b, component d:
     *   bc_u[b][d] + bc_upar[b][d] * (1 - ((x[bc_tdim[b]] - bc_c[b]) / bc_h[b])^2) */
    double bc_u[HFH_MAXBC][3];
    double bc_upar[HFH_MAXBC][3];
    int32_t bc_tdim[HFH_MAXBC];
    double bc_c[HFH_MAXBC], bc_h[HFH_MAXBC];
    double bc_p[HFH_MAXBC];
    double k_init[3][3];        /* initial kernel tensor (get_tensor) */
    int32_t tempdiscrtype;      /* HF_EXPLICIT_EULER ... HF_SEMI_IMPLICIT_BDF2 */
    int32_t pad_;
    double L2_fene, lambda_fene, E_fene;
    int32_t ve_discrtype;       /* HF_VE_EXPLICIT / HF_VE_IMPLICIT */
    int32_t pad2_;
    double alpha_gptt, beta_gptt;
    double src_t;               /* cell source term = src_t * t (0: no source) */
} hfh_params;

struct higflow_solver;

/* Build the case (domain, boundaries, properties, solver) from
 * <nameload>.domain / <nameload>.bc; *ns_out is a higflow_solver.  The params
 * are copied and stay the case's callback data; hfh_select makes a case's
 * data current before reference code that evaluates callbacks runs for it. */
int  hfh_build(const char *nameload, const hfh_params *p, struct higflow_solver **ns_out);
void hfh_select(struct higflow_solver *ns);
void hfh_destroy(struct higflow_solver *ns);

/* Build, record the step program (hf_flatten) and destroy: the program of the
 * case described by the inputs.  Free it with hfh_program_free. */
int  hfh_record(const char *nameload, const hfh_params *p, hf_program **out);
void hfh_program_free(hf_program *prog);
const char *hfh_error(void);
int  hfh_dim(void);

/* The reference prints progress through stdout; a host that hands programs to
 * another process keeps stdout clean (on by default). */
void hfh_set_quiet(int on);
void hfh_quiet_begin(void);
void hfh_quiet_end(void);

#ifdef __cplusplus
}
#endif

#endif

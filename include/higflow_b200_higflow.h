/*
 * higflow_b200 — HigFlow-facing drop-in binding.
 *
 * These entry points take HigFlow's own solver object and are compiled against
 * HigFlow's headers (higflow/src/hig-flow-kernel.h) with the same -DDIM as
 * libhigflow.  They sit between a case's main loop and the GPU engine declared
 * in higflow_b200.h:
 *
 *   hf_flatten       walks the reference meshes once and records every stencil
 *                    query of one step into an hf_program (host memory)
 *   hf_attach        flattens, uploads program and current fields to the GPU
 *   hf_step          one GPU time step; replaces higflow_solver_step
 *                    (higflow/src/hig-flow-step.c:1363) and
 *                    higflow_solver_step_viscoelastic
 *                    (hig-flow-step-viscoelastic.c:2091)
 *   hf_sync_to_host  copies the device fields back into ns->dp*->values so
 *                    HigFlow's printers and savers see them
 *   hf_sync_to_device copies ns->dp*->values (state and sources) to the
 *                    device, after higflow_load_properties
 *                    (higflow/src/hig-flow-io.c:5716) or a host-side edit
 *   hf_detach        syncs and frees the GPU state
 *   hf_solver_step   void wrapper with the reference's calling convention;
 *                    aborts with a message on a non-zero status, as the
 *                    reference does on errors (higtree/src/utils.h:46-52)
 */
#ifndef HIGFLOW_B200_HIGFLOW_H
#define HIGFLOW_B200_HIGFLOW_H

#include "higflow_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

struct higflow_solver;

int  hf_flatten(struct higflow_solver *ns, hf_program **out);
void hf_program_free(hf_program *p);
/* reason for the last non-zero hf_flatten status (static storage) */
const char *hf_flatten_error(void);

int  hf_attach(struct higflow_solver *ns, const hf_options *opt);
int  hf_step(struct higflow_solver *ns);
int  hf_sync_to_host(struct higflow_solver *ns);
int  hf_sync_to_device(struct higflow_solver *ns);
/* higflow_adjust_timestep on the GPU state (hf_case_adjust_timestep); sets
 * ns->par.dt */
int  hf_adjust_timestep(struct higflow_solver *ns);
void hf_detach(struct higflow_solver *ns);
void hf_solver_step(struct higflow_solver *ns);

#ifdef __cplusplus
}
#endif

#endif

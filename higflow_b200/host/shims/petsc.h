/*
 * PETSc stand-in for the HigFlow host build and the oracle build.  The
 * reference's utils.c only initialises and finalises PETSc; its Poisson solves
 * go through the solver vtable, which the host build gives to the GPU solver
 * engine (hf_host_solver.c) and the oracle to its own CPU engine.
 */
#ifndef HF_ORACLE_PETSC_SHIM_H
#define HF_ORACLE_PETSC_SHIM_H
typedef int PetscErrorCode;
PetscErrorCode PetscInitialize(int *argc, char ***argv, const char *file, const char *help);
PetscErrorCode PetscFinalize(void);
#endif

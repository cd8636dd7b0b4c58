/*
 * PETSc stand-in for the oracle build (test infrastructure).  The reference's
 * utils.c only initialises and finalises PETSc; its Poisson solves go through
 * the solver vtable, which the oracle's own CPU engine implements.
 */
#ifndef HF_ORACLE_PETSC_SHIM_H
#define HF_ORACLE_PETSC_SHIM_H
typedef int PetscErrorCode;
PetscErrorCode PetscInitialize(int *argc, char ***argv, const char *file, const char *help);
PetscErrorCode PetscFinalize(void);
#endif

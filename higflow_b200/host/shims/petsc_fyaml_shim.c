/*
 * Definitions for the PETSc and libfyaml stand-ins (HigFlow host build and
 * oracle build; neither library is in this image).
 */
#include <stdio.h>
#include <stdlib.h>
#include "petsc.h"
#include "libfyaml.h"

PetscErrorCode PetscInitialize(int *argc, char ***argv, const char *file, const char *help)
{
    (void)argc; (void)argv; (void)file; (void)help;
    return 0;
}

PetscErrorCode PetscFinalize(void) { return 0; }

static void no_yaml(const char *fn)
{
    fprintf(stderr, "single-rank build: %s is not available (cases are built without YAML input)\n", fn);
    abort();
}

struct fy_document *fy_document_build_from_file(const struct fy_parse_cfg *cfg, const char *file)
{
    (void)cfg; (void)file;
    no_yaml("fy_document_build_from_file");
    return NULL;
}

void fy_document_destroy(struct fy_document *fyd) { (void)fyd; }

int fy_document_scanf(struct fy_document *fyd, const char *fmt, ...)
{
    (void)fyd; (void)fmt;
    no_yaml("fy_document_scanf");
    return 0;
}

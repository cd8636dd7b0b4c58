/*
 * AMR text-format reader for the HigFlow host build and the oracle build.
 *
 * higtree/src/higtree-io.c cannot be compiled here (it needs HDF5), so the
 * three reader entry points the reference calls on the step-setup path are
 * restated from it:
 *   higio_read_amr_info       higtree-io.c:269-293  (bbox, levels, patches)
 *   higio_read_from_amr_info  higtree-io.c:97-153   (uniform first level,
 *                                                    2x refinement of patches)
 *   higio_read_from_amr       higtree-io.c:155-161
 */
#include <assert.h>
#include <stdio.h>
#include <stdlib.h>
#include "higtree-io.h"
#include "utils.h"

higio_amr_info *higio_read_amr_info(FILE *fd)
{
    higio_amr_info *mi = calloc(1, sizeof *mi);
    for (int dim = 0; dim < DIM; dim++) {
        if (fscanf(fd, "%lf", &mi->l[dim]) != 1) abort();
        if (fscanf(fd, "%lf", &mi->h[dim]) != 1) abort();
    }
    if (fscanf(fd, "%d", &mi->numlevels) != 1) abort();
    mi->levels = calloc((size_t)mi->numlevels, sizeof *mi->levels);
    for (int l = 0; l < mi->numlevels; l++) {
        __higio_level_info *lv = &mi->levels[l];
        lv->level = l;
        for (int dim = 0; dim < DIM; dim++)
            if (fscanf(fd, "%lf", &lv->delta[dim]) != 1) abort();
        if (fscanf(fd, "%d", &lv->numpatches) != 1) abort();
        lv->patches = calloc((size_t)lv->numpatches, sizeof *lv->patches);
        for (int p = 0; p < lv->numpatches; p++) {
            for (int dim = 0; dim < DIM; dim++)
                if (fscanf(fd, "%d", &lv->patches[p].initcell[dim]) != 1) abort();
            for (int dim = 0; dim < DIM; dim++)
                if (fscanf(fd, "%d", &lv->patches[p].patchsize[dim]) != 1) abort();
        }
    }
    return mi;
}

void higio_amr_info_destroy(higio_amr_info *mi)
{
    for (int l = 0; l < mi->numlevels; l++) free(mi->levels[l].patches);
    free(mi->levels);
    free(mi);
}

hig_cell *higio_read_from_amr_info(higio_amr_info *mi)
{
    hig_cell *root = hig_create_root(mi->l, mi->h);
    hig_refine_uniform(root, mi->levels[0].patches[0].patchsize);

    int two[DIM];
    for (int i = 0; i < DIM; i++) two[i] = 2;
    for (int l = 1; l < mi->numlevels; l++) {
        __higio_level_info *lv = &mi->levels[l];
        for (int p = 0; p < lv->numpatches; p++) {
            __higio_patch_info *pa = &lv->patches[p];
            Point init;
            for (int i = 0; i < DIM; i++) init[i] = lv->delta[i] * pa->initcell[i] + mi->l[i];
            int k[DIM];
            for (int i = 0; i < DIM; i++) k[i] = 0;
            for (;;) {
                Point pt;
                for (int i = 0; i < DIM; i++) pt[i] = init[i] + lv->delta[i] * k[i];
                hig_cell *c = hig_get_cell_with_point(root, pt);
                Point cd;
                hig_get_delta(c, cd);
                int fine_enough = 1;
                for (int i = 0; i < DIM; i++)
                    if (FLT_LT(lv->delta[i], cd[i])) { fine_enough = 0; break; }
                if (!fine_enough) hig_refine_uniform(c, two);
                int i = 0;
                while (i < DIM && k[i] + 2 >= pa->patchsize[i] - 1) { k[i] = 0; i++; }
                if (i < DIM) k[i] += 2; else break;
            }
        }
    }
    return root;
}

hig_cell *higio_read_from_amr(FILE *fd)
{
    higio_amr_info *mi = higio_read_amr_info(fd);
    hig_cell *root = higio_read_from_amr_info(mi);
    higio_amr_info_destroy(mi);
    return root;
}

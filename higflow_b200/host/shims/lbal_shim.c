/*
 * Single-rank load balancer for the HigFlow host build and the oracle build.
 *
 * Stands in for higtree/src/lbal.c (Zoltan-based).  On one rank every input
 * tree stays local, in insertion order, and no tree is fringe, which is what
 * higflow_partition_domain (higflow/src/hig-flow-kernel.c:1298-1345) consumes.
 */
#include <stdlib.h>
#include <string.h>
#include "lbal.h"

load_balancer *lb_create(MPI_Comm comm, unsigned num_groups)
{
    load_balancer *lb = calloc(1, sizeof *lb);
    lb->group = comm;
    lb->num_groups = num_groups ? num_groups : 1;
    return lb;
}

void lb_add_input_tree(load_balancer *lb, hig_cell *tree, bool managed, unsigned group)
{
    struct _lb_input_tree *t = calloc(1, sizeof *t);
    t->tree = tree;
    t->group = group;
    t->managed = managed;
    /* append, keeping insertion order */
    struct _lb_input_tree **pp = &lb->trees;
    while (*pp) pp = &(*pp)->next;
    *pp = t;
    lb->num_in_higs++;
}

void lb_calc_partition(load_balancer *lb, partition_graph *pg)
{
    (void)pg;
    lb->num_out_higs = lb->num_in_higs;
    lb->output = calloc(lb->num_out_higs ? lb->num_out_higs : 1, sizeof *lb->output);
    lb->out_higs_group_start = calloc(lb->num_groups + 1, sizeof(size_t));
    /* stable grouping: trees of group g, in insertion order */
    size_t k = 0;
    for (unsigned g = 0; g < lb->num_groups; g++) {
        lb->out_higs_group_start[g] = k;
        for (struct _lb_input_tree *t = lb->trees; t; t = t->next) {
            if (t->group == g) {
                lb->output[k].tree = t->tree;
                lb->output[k].group = g;
                k++;
            }
        }
    }
    lb->out_higs_group_start[lb->num_groups] = k;
}

size_t lb_get_num_local_trees(load_balancer *lb) { return lb->num_out_higs; }

hig_cell *lb_get_local_tree(load_balancer *lb, size_t idx, unsigned *group)
{
    if (group) *group = lb->output[idx].group;
    return lb->output[idx].tree;
}

unsigned lb_get_num_local_trees_in_group(load_balancer *lb, unsigned group)
{
    return (unsigned)(lb->out_higs_group_start[group + 1] - lb->out_higs_group_start[group]);
}

hig_cell *lb_get_local_tree_in_group(load_balancer *lb, size_t group_idx, unsigned group)
{
    return lb->output[lb->out_higs_group_start[group] + group_idx].tree;
}

void lb_destroy(load_balancer *lb)
{
    /* Trees handed to the domain stay alive; only the bookkeeping is freed. */
    struct _lb_input_tree *t = lb->trees;
    while (t) {
        struct _lb_input_tree *n = t->next;
        free(t);
        t = n;
    }
    free(lb->output);
    free(lb->out_higs_group_start);
    free(lb);
}

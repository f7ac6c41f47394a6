/* cds_oracle.h -- CPU restatement of the reference k-clique densest-subgraph
 * pipeline (wajidmanzoor/CDS, cpuCode/c++).  TEST INFRASTRUCTURE ONLY: the
 * checker for tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg.  Nothing in the product links or calls it.
 *
 * Graphs are passed as symmetric CSR: off[n+1] (uint64), adj[off[n]] (uint32),
 * rows sorted, no self-loops, no duplicates.
 */
#ifndef CDS_ORACLE_H
#define CDS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Reads the adjacency-list format exactly as cpuCode/c++/src/graph.cpp:9-52
 * does (header "n m", then "v nbr nbr ..." lines, self-loops dropped) and
 * returns a CSR whose rows keep the file's order.  *off_out / *adj_out are
 * malloc'd; free them with oracle_free.  Returns 0 or -1. */
int oracle_read_adjlist(const char *path, uint32_t *n_out, uint64_t **off_out,
                        uint32_t **adj_out);
void oracle_free(void *p);

/* k-clique count and per-vertex clique degree (cpuCode/c++/src/helpers.cpp:
 * 317-511).  clique_degree may be NULL.  Returns |Psi| or -1 on error. */
int64_t oracle_count_cliques(uint32_t n, const uint64_t *off, const uint32_t *adj,
                             uint32_t k, int64_t *clique_degree);

/* Number of k-cliques whose first vertex in the listing order (the root the
 * enumeration starts from) has an id u with u % stride == phase: a bounded,
 * seeded sample of the listing work (stride 1 counts every clique). */
int64_t oracle_count_cliques_sampled(uint32_t n, const uint64_t *off, const uint32_t *adj,
                                     uint32_t k, uint32_t stride, uint32_t phase);

/* Number of k-cliques whose members all have in_set[v] != 0. */
int64_t oracle_count_in_set(uint32_t n, const uint64_t *off, const uint32_t *adj,
                            uint32_t k, const uint8_t *in_set);

/* Sequential clique-core peel (cpuCode/c++/src/helpers.cpp:16-150).  Row i
 * (0-based) of the outputs describes the (i+1)-th removal: the vertex, its
 * clique degree at removal, and the number of cliques left afterwards.
 * core[v] = running maximum of the removal degree (the clique-core number).
 * Any output pointer may be NULL.  Returns |Psi| or -1. */
int64_t oracle_peel(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t k,
                    uint32_t *order, int64_t *removal_degree, int64_t *cliques_left,
                    int64_t *core);

typedef struct oracle_result {
  int64_t total_cliques;   /* |Psi| of the whole graph                       */
  int64_t core_threshold;  /* k' = ceil(best prefix density)                  */
  int64_t core_size;       /* vertices of the densest (k',Psi)-core           */
  int64_t core_cliques;    /* cliques inside that core                        */
  int64_t max_core;        /* largest clique-core number                      */
  int64_t pruned_edges;    /* core edges inside >= 1 core clique              */
  int64_t n_components;    /* connected components of the pruned core        */
  int64_t flows;           /* max-flow solves performed                       */
  int64_t num;             /* cliques inside the answer set                   */
  int64_t den;             /* size of the answer set                          */
} oracle_result;

/* Whole pipeline with exact arithmetic.  in_set[n] receives the answer set
 * (1 = member).  Returns 0 or -1. */
int oracle_solve(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t k,
                 oracle_result *res, uint8_t *in_set);

#ifdef __cplusplus
}
#endif
#endif
